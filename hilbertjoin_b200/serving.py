"""Join serving: resident point sets, a thread-safe request queue, admission
against a device-memory budget, and concurrent execution of admitted joins
(the native loop in csrc/hj_server.cu, bound here with ctypes).

    srv = Server(form="auto", memory_budget_bytes=40 << 30, max_inflight=8)
    a = srv.upload(points_a)                 # stays on the device
    rid = srv.submit(a, None, eps)           # self-join; submit(a, b, eps) for A x B
    res = srv.wait(rid)                      # {"count", "status", "latency_ms", ...}

`run_benchmark` replays the serving workload (Poisson arrivals, mixed self and
two-set joins of uneven n, d and eps) and reports throughput and p50/p99
latency next to the plain FP64 path serving one request at a time.
"""
from __future__ import annotations

import ctypes
import json
import threading
import time

import numpy as np

from . import FORMS, HJError, Result, ServerOpts, lib
from . import workloads as W


def _bind():
    L = lib()
    if getattr(L, "_hj_server_bound", False):
        return L
    P, U64, U32, I, D = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_double
    sigs = {
        "hj_server_opts_init": (None, [ctypes.POINTER(ServerOpts)]),
        "hj_server_create": (I, [ctypes.POINTER(ServerOpts), ctypes.POINTER(P)]),
        "hj_server_destroy": (I, [P]),
        "hj_set_upload": (I, [P, P, I, U64, U32, ctypes.POINTER(U64)]),
        "hj_set_release": (I, [P, U64]),
        "hj_submit": (I, [P, U64, U64, D, ctypes.POINTER(U64)]),
        "hj_poll": (I, [P, U64, ctypes.POINTER(I), ctypes.POINTER(Result)]),
        "hj_wait": (I, [P, U64, D, ctypes.POINTER(Result)]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    L._hj_server_bound = True
    return L


def _result_dict(r: Result) -> dict:
    return {"count": int(r.count), "status": int(r.status), "form_used": int(r.form_used),
            "queue_ms": r.queue_ms, "run_ms": r.run_ms, "latency_ms": r.latency_ms,
            "candidate_pairs": int(r.candidate_pairs), "band_pairs": int(r.band_pairs)}


class Server:
    def __init__(self, form="auto", memory_budget_bytes: int = 40 << 30, max_inflight: int = 8, device=None,
                 batch_max: int = 1, block_centring: bool = False):
        """batch_max > 1 (tensor-core forms): a free worker runs up to batch_max
        queued requests as one batch (one persistent launch). block_centring:
        the requests' FP16 joins may switch to per-block centring (admission
        then counts its buffers); otherwise they use one global centre."""
        L = _bind()
        o = ServerOpts()
        L.hj_server_opts_init(ctypes.byref(o))
        o.memory_budget_bytes = int(memory_budget_bytes)
        o.max_inflight = int(max_inflight)
        o.batch_max = int(batch_max)
        o.block_centring = int(bool(block_centring))
        o.device = -1 if device is None else int(device)
        o.form = FORMS[form] if isinstance(form, str) else int(form)
        h = ctypes.c_void_p()
        rc = L.hj_server_create(ctypes.byref(o), ctypes.byref(h))
        if rc != 0:
            raise HJError(rc, "hj_server_create failed")
        self._h = h
        self._L = L

    def upload(self, points) -> int:
        x = np.ascontiguousarray(np.asarray(points))
        if x.dtype not in (np.float32, np.float64):
            x = x.astype(np.float32)
        sid = ctypes.c_uint64(0)
        rc = self._L.hj_set_upload(self._h, x.ctypes.data_as(ctypes.c_void_p), x.itemsize, x.shape[0], x.shape[1],
                                   ctypes.byref(sid))
        if rc != 0:
            raise HJError(rc, "hj_set_upload failed")
        return int(sid.value)

    def release(self, set_id: int) -> None:
        rc = self._L.hj_set_release(self._h, set_id)
        if rc != 0:
            raise HJError(rc, "hj_set_release failed")

    def submit(self, a: int, b, eps: float) -> int:
        rid = ctypes.c_uint64(0)
        rc = self._L.hj_submit(self._h, a, 0 if b is None else b, float(eps), ctypes.byref(rid))
        if rc != 0:
            raise HJError(rc, "hj_submit rejected the request")
        return int(rid.value)

    def poll(self, rid: int):
        done = ctypes.c_int(0)
        r = Result()
        rc = self._L.hj_poll(self._h, rid, ctypes.byref(done), ctypes.byref(r))
        if rc != 0:
            raise HJError(rc, "hj_poll failed")
        return _result_dict(r) if done.value else None

    def wait(self, rid: int, timeout_ms: float = -1.0) -> dict:
        r = Result()
        rc = self._L.hj_wait(self._h, rid, float(timeout_ms), ctypes.byref(r))
        if rc != 0:
            raise HJError(rc, "hj_wait failed")
        return _result_dict(r)

    def close(self) -> None:
        if self._h:
            self._L.hj_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ------------------------------------------------------------------ workload

DIMS = (8, 16, 32, 64, 128)


def make_workload(n_requests: int = 2000, n_sets: int = 48, seed: int = 5, n_lo: int = 1000, n_hi: int = 500_000,
                  self_frac: float = 0.7, nbr_lo: float = 8, nbr_hi: float = 128):
    """The serving stream: a pool of point sets (n log-uniform in [n_lo, n_hi], d
    from DIMS, uniform [0,1) or a 16-component Gaussian mixture, FP32) that stay
    resident, and requests drawing a self-join (self_frac) or a two-set join of
    two pool sets of equal d, with eps for a mean neighbour count log-uniform in
    [nbr_lo, nbr_hi]. Returns (sets, requests); requests are dicts with keys
    a, b (None for self), eps."""
    rng = np.random.default_rng(seed)
    sets = []
    for i in range(n_sets):
        d = DIMS[i % len(DIMS)]
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        if rng.random() < 0.5:
            x = W.uniform(n, d, 1000 + i, dtype=np.float32)
            kind = "uniform"
        else:
            x = W.gmm(n, d, 1000 + i, components=16, dtype=np.float32)
            kind = "gmm16"
        sets.append({"x": x, "n": n, "d": d, "kind": kind, "eps": {}})
    by_d = {d: [i for i, s in enumerate(sets) if s["d"] == d] for d in DIMS}
    reqs = []
    for _ in range(n_requests):
        a = int(rng.integers(n_sets))
        nbr = float(np.exp(rng.uniform(np.log(nbr_lo), np.log(nbr_hi))))
        tgt = min((8, 16, 32, 64, 128), key=lambda t: abs(np.log(t / nbr)))
        b = None
        if rng.random() >= self_frac and len(by_d[sets[a]["d"]]) > 1:
            b = int(rng.choice([i for i in by_d[sets[a]["d"]] if i != a]))
        s = sets[a]
        if tgt not in s["eps"]:
            s["eps"][tgt] = W.calibrate_eps(s["x"], s["n"], tgt, sample=1500)
        reqs.append({"a": a, "b": b, "eps": s["eps"][tgt], "nbr": tgt})
    return sets, reqs


def _replay(srv: Server, ids, reqs, rate: float, seed: int = 1):
    """Open-loop replay with Poisson arrivals at `rate` requests/s (rate <= 0: all
    at once). Returns (results in request order, wall seconds)."""
    rng = np.random.default_rng(seed)
    rids = [None] * len(reqs)
    t0 = time.perf_counter()

    def submitter():
        t_next = time.perf_counter()
        for i, r in enumerate(reqs):
            if rate > 0:
                t_next += rng.exponential(1.0 / rate)
                dt = t_next - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
            rids[i] = srv.submit(ids[r["a"]], None if r["b"] is None else ids[r["b"]], r["eps"])

    th = threading.Thread(target=submitter)
    th.start()
    out = [None] * len(reqs)
    for i in range(len(reqs)):
        while rids[i] is None:
            time.sleep(0.0005)
        out[i] = srv.wait(rids[i])
    th.join()
    return out, time.perf_counter() - t0


def _summary(res, wall):
    lat = np.array([r["latency_ms"] for r in res])
    ok = all(r["status"] == 0 for r in res)
    pairs = sum(r["candidate_pairs"] for r in res)
    return {"requests": len(res), "ok": ok, "wall_s": wall, "requests_per_s": len(res) / wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "candidate_pairs_per_s": pairs / wall}


def run_benchmark(n_requests: int = 2000, form: str = "auto", max_inflight: int = 8, baseline_requests: int = 200,
                  seed: int = 5, budget: int = 40 << 30, n_hi: int = 500_000, batch_max: int = 8) -> dict:
    sets, reqs = make_workload(n_requests, seed=seed, n_hi=n_hi)
    out = {"workload": f"{n_requests} requests, 70% self / 30% A x B, n log-U[1e3, {n_hi:.0e}], d in {DIMS}, "
                       "uniform or 16-GMM FP32, eps for 8-128 neighbours, sets resident", "form": form}
    with Server(form=form, memory_budget_bytes=budget, max_inflight=max_inflight) as srv:
        ids = [srv.upload(s["x"]) for s in sets]
        _replay(srv, ids, reqs[:16], 0)  # warm-up
        res, wall = _replay(srv, ids, reqs, 0)
        cap = _summary(res, wall)
        out["saturated"] = cap
        counts = [r["count"] for r in res]
    if batch_max > 1:  # the same stream with queued requests grouped into batches
        with Server(form=form, memory_budget_bytes=budget, max_inflight=max_inflight, batch_max=batch_max) as srv:
            ids = [srv.upload(s["x"]) for s in sets]
            _replay(srv, ids, reqs[:16], 0)
            res_bt, wall_bt = _replay(srv, ids, reqs, 0)
            if [r["count"] for r in res_bt] != counts:
                raise RuntimeError("batched and unbatched servers disagree")
            out[f"saturated_batch_max_{batch_max}"] = _summary(res_bt, wall_bt)
    with Server(form="plain", memory_budget_bytes=budget, max_inflight=1) as srv:
        ids = [srv.upload(s["x"]) for s in sets]
        _replay(srv, ids, reqs[:4], 0)
        k = min(baseline_requests, len(reqs))
        res_b, wall_b = _replay(srv, ids, reqs[:k], 0)
        base = _summary(res_b, wall_b)
        assert [r["count"] for r in res_b] == counts[:k], "plain and tensor-core servers disagree"
        out["baseline_plain_one_at_a_time"] = base
        # open loop at 80 % of the baseline's capacity, on both servers
        rate = 0.8 * base["requests_per_s"]
        res_bo, wall_bo = _replay(srv, ids, reqs[:k], rate, seed=2)
        out["baseline_open_loop"] = dict(_summary(res_bo, wall_bo), offered_rate=rate)
    with Server(form=form, memory_budget_bytes=budget, max_inflight=max_inflight) as srv:
        ids = [srv.upload(s["x"]) for s in sets]
        res_o, wall_o = _replay(srv, ids, reqs[:k], rate, seed=2)
        out["open_loop_same_rate"] = dict(_summary(res_o, wall_o), offered_rate=rate)
        rate2 = 0.8 * cap["requests_per_s"]
        res_o2, wall_o2 = _replay(srv, ids, reqs, rate2, seed=3)
        out["open_loop_80pct_capacity"] = dict(_summary(res_o2, wall_o2), offered_rate=rate2)
    out["throughput_ratio_vs_plain"] = cap["requests_per_s"] / base["requests_per_s"]
    return out


if __name__ == "__main__":
    print(json.dumps(run_benchmark()))
