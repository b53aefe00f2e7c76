"""Host-side logic of the serving benchmark, with no GPU: the request stream
(deterministic for a seed; two-set joins pair sets of equal d; one eps per
set and neighbour target), the open-loop replay (results in request order,
Poisson arrivals at the offered rate, every request waited for) and the
latency summary, driven through a stand-in server."""
import threading
import time

import numpy as np
import pytest

from hilbertjoin_b200 import serving


class FakeServer:
    """submit/wait with a fixed service time; the count encodes the request."""

    def __init__(self, service_s=0.0):
        self.service_s = service_s
        self.lock = threading.Lock()
        self.submits = []
        self.reqs = {}

    def submit(self, a, b, eps):
        with self.lock:
            rid = len(self.submits)
            self.submits.append(time.perf_counter())
            self.reqs[rid] = (a, b, eps)
        return rid

    def wait(self, rid, timeout_ms=-1.0):
        a, b, eps = self.reqs[rid]
        if self.service_s:
            time.sleep(self.service_s)
        return {"status": 0, "count": a * 1000 + (-1 if b is None else b), "latency_ms": 1.0 + rid,
                "candidate_pairs": 10}


def small_stream(seed=5):
    return serving.make_workload(n_requests=60, n_sets=10, seed=seed, n_lo=200, n_hi=3000)


def test_stream_is_deterministic_and_consistent():
    sets, reqs = small_stream()
    sets2, reqs2 = small_stream()
    assert reqs == reqs2
    assert all(np.array_equal(s["x"], t["x"]) for s, t in zip(sets, sets2))
    assert small_stream(seed=6)[1] != reqs
    for r in reqs:
        a = sets[r["a"]]
        assert a["x"].shape == (a["n"], a["d"]) and a["x"].dtype == np.float32
        assert a["d"] in serving.DIMS and 200 <= a["n"] <= 3000
        assert r["nbr"] in (8, 16, 32, 64, 128) and r["eps"] > 0
        assert r["eps"] == a["eps"][r["nbr"]]  # one eps per set and target
        if r["b"] is not None:
            assert r["b"] != r["a"] and sets[r["b"]]["d"] == a["d"]
    assert any(r["b"] is None for r in reqs) and any(r["b"] is not None for r in reqs)


def test_replay_all_at_once_keeps_request_order():
    _, reqs = small_stream()
    ids = [100 + i for i in range(10)]
    out, wall = serving._replay(FakeServer(), ids, reqs, rate=0)
    assert len(out) == len(reqs) and wall >= 0
    for r, o in zip(reqs, out):
        assert o["count"] == ids[r["a"]] * 1000 + (-1 if r["b"] is None else ids[r["b"]])


def test_replay_open_loop_offers_the_rate():
    reqs = [{"a": 0, "b": None, "eps": 0.1}] * 300
    srv = FakeServer()
    rate = 3000.0
    out, wall = serving._replay(srv, [7], reqs, rate=rate, seed=4)
    assert len(out) == 300 and all(o["status"] == 0 for o in out)
    gaps = np.diff(srv.submits)
    # exponential inter-arrival times with mean 1/rate (sleep granularity adds a little)
    assert 0.5 / rate < gaps.mean() < 3.0 / rate, gaps.mean()
    assert wall >= 0.5 * len(reqs) / rate


def test_summary_percentiles():
    res = [{"status": 0, "latency_ms": float(v), "candidate_pairs": 5} for v in range(1, 101)]
    s = serving._summary(res, 2.0)
    assert s["requests"] == 100 and s["ok"] and s["requests_per_s"] == 50.0
    assert s["p50_ms"] == pytest.approx(50.5) and s["p99_ms"] == pytest.approx(99.01)
    assert s["candidate_pairs_per_s"] == 250.0
    res[3]["status"] = 5
    assert not serving._summary(res, 2.0)["ok"]
