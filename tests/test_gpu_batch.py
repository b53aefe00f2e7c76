"""Batched joins: many joins of uneven n, d and eps in one persistent
tensor-core launch (hj_batch_*). Each job's count must equal the count of the
same join run alone (which the parity tests tie to the oracle), in every
tensor-core form, on repeated runs, and when a run is captured into a CUDA
graph and replayed."""
import numpy as np
import pytest

import oracle as O
from hilbertjoin_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200 as hj
    from hilbertjoin_b200 import batching as B
    return torch, hj, B


def make_jobs(torch, seed=0, dtype=np.float32):
    """A mixed batch: self-joins and two-set joins, n from 700 to 40k,
    d from 3 to 200, uniform and clustered data, 8 to 64 neighbours."""
    rng = np.random.default_rng(seed)
    spec = [(700, None, 3, "u"), (5000, None, 8, "g"), (12000, 9000, 16, "u"), (3001, None, 33, "u"),
            (40000, None, 64, "u"), (20000, 4000, 64, "g"), (2500, None, 100, "u"), (6000, 6000, 128, "g"),
            (1500, None, 200, "u"), (9000, None, 28, "g")]
    jobs, host = [], []
    for i, (na, nb, d, kind) in enumerate(spec):
        gen = (lambda n, s: W.uniform(n, d, s, dtype=dtype)) if kind == "u" else \
            (lambda n, s: W.gmm(n, d, s, components=8, dtype=dtype))
        a = gen(na, 100 + i)
        b = gen(nb, 200 + i) if nb else None
        nbr = float(rng.choice([8, 16, 32, 64]))
        eps = W.calibrate_eps(a, na, nbr) if b is None else W.calibrate_eps_join(a, b, nb, nbr)
        host.append((a, b, eps))
        jobs.append((torch.from_numpy(a).cuda(), None if b is None else torch.from_numpy(b).cuda(), eps))
    return jobs, host


def alone(hj, job, form):
    """The job run on its own in the given form ("plain": the FP64 form)."""
    a, b, eps = job
    return hj.self_join_count(a, eps, form=form) if b is None else hj.join_count(a, b, eps, form=form)


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
def test_batch_counts_equal_joins_alone(env, form):
    torch, hj, B = env
    jobs, host = make_jobs(torch)
    got, st = B.batch_count(jobs, form=form, return_stats=True)
    want = [alone(hj, j, "plain") for j in jobs]
    assert got == want
    assert st["work_items"] > 0 and st["candidate_pairs"] > 0
    # two small ones against the oracle directly
    a, _, eps = host[0]
    assert got[0] == O.self_count_brute(a.astype(np.float64), eps)
    a, b, eps = host[2]
    assert got[2] == O.join_count_brute(a.astype(np.float64), b.astype(np.float64), eps)


def test_batch_repeated_runs_and_graph_replay(env):
    torch, hj, B = env
    jobs, _ = make_jobs(torch, seed=1)
    want = [alone(hj, j, "fp16") for j in jobs]
    with B.Batch(jobs, form="fp16") as b:
        assert b.counts() == want  # planning ran it once
        b.run()
        b.run()
        assert b.counts() == want
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            b.run(stream=s)
        for _ in range(3):
            g.replay()
        torch.cuda.synchronize()
        assert b.counts() == want
        del g


def test_batch_with_fp64_routed_job_and_fp64_inputs(env):
    """A job whose eps^2 is tiny against its squared norms goes to the FP64
    kernel inside the batch; FP64 inputs; ref_compat applies to every job."""
    torch, hj, B = env
    rng = np.random.default_rng(7)
    far = rng.random((3000, 16)) * 1000.0
    jobs = [(torch.from_numpy(far).cuda(), None, 0.5),
            (torch.from_numpy(rng.random((4000, 24))).cuda(), None, 0.35),
            (torch.from_numpy(rng.random((2000, 24))).cuda(), torch.from_numpy(rng.random((3001, 24))).cuda(), 0.4)]
    got, st = B.batch_count(jobs, form="fp16", return_stats=True)
    assert st["fp64_items"] > 0
    assert got == [alone(hj, j, "plain") for j in jobs]
    assert got[0] == O.self_count_brute(far, 0.5)
    rc = B.batch_count(jobs, form="tf32", ref_compat=True)
    want = [hj.self_join_count(jobs[0][0], 0.5, ref_compat=True), hj.self_join_count(jobs[1][0], 0.35, ref_compat=True),
            hj.join_count(jobs[2][0], jobs[2][1], 0.4, ref_compat=True)]
    assert rc == want


def test_batch_rejects_bad_jobs(env):
    torch, hj, B = env
    x = torch.rand(100, 300, device="cuda")
    with pytest.raises(hj.HJError):
        B.batch_count([(x, None, 0.1)])
    with pytest.raises(hj.HJError):
        B.batch_count([(torch.rand(10, 4, device="cuda"), None, 0.1)], form="plain")


def test_item_chunk_and_tuned_batches_are_exact(env):
    torch, hj, B = env
    from hilbertjoin_b200 import autotune
    x = torch.from_numpy(W.gmm(30000, 24, 5, components=8, dtype=np.float32)).cuda()
    eps = W.calibrate_eps(x.cpu().numpy(), 30000, 24)
    want = hj.self_join_count(x, eps)
    for chunk in (1, 7, 64, 300):
        for form in ("fp16", "tf32"):
            assert hj.self_join_count(x, eps, form=form, item_chunk=chunk) == want
    jobs, _ = make_jobs(torch, seed=3)
    assert B.batch_count(jobs, tuned=True) == [alone(hj, j, "plain") for j in jobs]
    assert autotune.config_for(24)["form"] in autotune.FORMS
    with pytest.raises(hj.HJError):
        hj.self_join_count(x, eps, form="fp16", item_chunk=5000)
