"""Serving: resident sets, concurrent admitted joins, admission control. Each
request's count in the mix equals the count of the same join run alone (exact
integers: the pipeline is deterministic and requests share no state)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200
    return hilbertjoin_b200


@pytest.mark.parametrize("form,batch_max", [("tf32", 1), ("plain", 1), ("fp16", 8)])
def test_results_alone_equal_results_in_the_mix(hj, form, batch_max):
    from hilbertjoin_b200 import serving
    sets, reqs = serving.make_workload(n_requests=60, n_sets=10, seed=11, n_hi=40_000)
    alone = []
    for r in reqs:
        a = sets[r["a"]]["x"]
        if r["b"] is None:
            alone.append(hj.self_join_count(a, r["eps"], form=form))
        else:
            alone.append(hj.join_count(a, sets[r["b"]]["x"], r["eps"], form=form))
    with serving.Server(form=form, max_inflight=6, batch_max=batch_max) as srv:
        ids = [srv.upload(s["x"]) for s in sets]
        rids = [srv.submit(ids[r["a"]], None if r["b"] is None else ids[r["b"]], r["eps"]) for r in reqs]
        mix = [srv.wait(i) for i in rids]
    assert all(m["status"] == 0 for m in mix)
    assert [m["count"] for m in mix] == alone


def test_admission_budget_and_release(hj):
    from hilbertjoin_b200 import serving
    x = np.random.default_rng(1).random((20000, 16)).astype(np.float32)
    with serving.Server(form="tf32", memory_budget_bytes=8 << 20, max_inflight=2) as srv:
        s = srv.upload(x)
        with pytest.raises(hj.HJError) as e:  # larger than the whole budget
            srv.submit(s, None, 0.5)
        assert e.value.status == 8
    with serving.Server(form="tf32", memory_budget_bytes=1 << 30, max_inflight=2) as srv:
        s = srv.upload(x)
        rid = srv.submit(s, None, 0.5)
        srv.release(s)  # freed once its request finishes
        r = srv.wait(rid)
        assert r["status"] == 0 and r["count"] == hj.self_join_count(x, 0.5, form="tf32")
        with pytest.raises(hj.HJError):
            srv.submit(s, None, 0.5)


def test_poll_until_done(hj):
    import time
    from hilbertjoin_b200 import serving
    x = np.random.default_rng(2).random((30000, 8)).astype(np.float32)
    with serving.Server(form="tf32") as srv:
        s = srv.upload(x)
        rid = srv.submit(s, None, 0.2)
        t0 = time.time()
        res = None
        while res is None and time.time() - t0 < 60:
            res = srv.poll(rid)
            time.sleep(0.001)
        assert res is not None and res["count"] == hj.self_join_count(x, 0.2)


def test_device_memory_stays_within_budget(hj):
    """A budget that admits only a few of these requests at a time: while 24
    joins of uneven size run through 8 workers, the device memory the server
    takes (free memory before the requests minus its lowest value during them)
    stays within the budget plus 256 MB of slack (per-context counters, events
    and the kernels' code loaded on first use). Workers' buffers are charged
    against the budget and freed when nothing else fits."""
    import threading
    import time
    import torch
    from hilbertjoin_b200 import serving
    from hilbertjoin_b200 import workloads as W
    budget = 700 << 20
    sizes = [150_000, 60_000, 100_000, 20_000, 150_000, 80_000]
    xs = [W.uniform(n, 32, 300 + i, dtype=np.float32) for i, n in enumerate(sizes)]
    eps = [W.calibrate_eps(x, x.shape[0], 32, sample=2000) for x in xs]
    with serving.Server(form="fp16", memory_budget_bytes=budget, max_inflight=8) as srv:
        ids = [srv.upload(x) for x in xs]
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        low = [free0]
        done = threading.Event()

        def sample():
            while not done.is_set():
                low[0] = min(low[0], torch.cuda.mem_get_info()[0])
                time.sleep(0.002)

        th = threading.Thread(target=sample)
        th.start()
        try:
            rids = [srv.submit(ids[i % len(xs)], None, eps[i % len(xs)]) for i in range(24)]
            res = [srv.wait(r) for r in rids]
        finally:
            done.set()
            th.join()
    assert all(r["status"] == 0 for r in res)
    for i in range(len(xs)):
        assert res[i]["count"] == hj.self_join_count(xs[i], eps[i], form="fp16")
    used = free0 - low[0]
    assert used <= budget + (256 << 20), (used >> 20, budget >> 20)
