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
