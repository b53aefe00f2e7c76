"""GPU parity: the engine (called through its C ABI) against the CPU oracle.

Every form must return exactly the oracle's count: the FP64 direct-difference
pair test, inclusive at eps. The golden fixtures also pin the reference's own
counts (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle
from tests.golden.make_golden import make

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_counts.json")))["cases"]
FORMS = ["plain", "tf32", "bf16x3", "fp16"]


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200
    return hilbertjoin_b200


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
@pytest.mark.parametrize("form", FORMS)
def test_golden(hj, case, form):
    x = make(case)
    if case["kind"] == "self":
        got = hj.self_join_count(x, case["eps"], form=form)
        got_ref = hj.self_join_count(x, case["eps"], form=form, ref_compat=True)
    else:
        b = make(dict(case, seed=case["seed_b"], n=case["m"]))
        got = hj.join_count(x, b, case["eps"], form=form)
        got_ref = hj.join_count(x, b, case["eps"], form=form, ref_compat=True)
    assert got == case["oracle_count"]
    assert got_ref == case["oracle_count_tail_drop"]
    if case["ref_valid"]:
        assert got == case["ref_count"]


RAGGED = [(1, 3), (2, 1), (63, 5), (64, 8), (65, 7), (127, 2), (1000, 9), (3001, 17), (4097, 33)]


@pytest.mark.parametrize("n,d", RAGGED)
@pytest.mark.parametrize("form", FORMS)
def test_self_ragged(hj, n, d, form):
    rng = np.random.default_rng(n * 131 + d)
    x = rng.random((n, d))
    for eps in (0.05, 0.3, 0.9):
        assert hj.self_join_count(x, eps, form=form) == oracle.self_count_brute(x, eps), eps


@pytest.mark.parametrize("d", [1, 2, 3, 4, 6, 8, 12, 31, 64, 100, 128])
@pytest.mark.parametrize("form", FORMS)
def test_self_dims(hj, d, form):
    rng = np.random.default_rng(d)
    x = rng.random((2500, d))
    eps = float(np.sqrt(d) * 0.18)
    assert hj.self_join_count(x, eps, form=form) == oracle.self_count_brute(x, eps)


@pytest.mark.parametrize("na,nb,d", [(1000, 3000, 8), (3000, 1000, 20), (1, 500, 4), (777, 1, 5), (2048, 2048, 64)])
@pytest.mark.parametrize("form", FORMS)
def test_join_shapes(hj, na, nb, d, form):
    """Includes nB > nA, where the reference itself crashes."""
    rng = np.random.default_rng(na + nb + d)
    a, b = rng.random((na, d)), rng.random((nb, d))
    eps = float(np.sqrt(d) * 0.2)
    assert hj.join_count(a, b, eps, form=form) == oracle.join_count_brute(a, b, eps)


@pytest.mark.parametrize("form", FORMS)
def test_clustered_and_duplicates(hj, form):
    from hilbertjoin_b200 import workloads as W
    x = W.gmm(6000, 12, 3)
    x = np.concatenate([x, x[:500]])  # exact duplicates: distance 0, always counted
    eps = 0.05
    assert hj.self_join_count(x, eps, form=form) == oracle.self_count_brute(x, eps)


@pytest.mark.parametrize("form", FORMS)
def test_eps_extremes(hj, form):
    rng = np.random.default_rng(11)
    x = rng.random((700, 6))
    n = x.shape[0]
    assert hj.self_join_count(x, 1e-9, form=form) == 0
    assert hj.self_join_count(x, 100.0, form=form) == n * (n - 1) // 2
    assert hj.join_count(x, x[:300], 100.0, form=form) == n * 300


@pytest.mark.parametrize("form", FORMS)
def test_lattice_ties(hj, form):
    """Exact ties at eps follow the direct-difference FP64 test (inclusive); for
    the tensor-core forms every tie lands in the band and is re-evaluated."""
    from hilbertjoin_b200 import workloads as W
    for levels, step in ((3, 0.1), (5, 0.25), (4, 0.3)):
        x = W.lattice(3000, 6, levels, step=step, levels=levels)
        assert hj.self_join_count(x, step, form=form) == oracle.self_count_brute(x, step)


@pytest.mark.parametrize("active_dims", [0, 1, 2, 3, 4, 5])
def test_active_dims_change_work_only(hj, active_dims):
    rng = np.random.default_rng(5)
    x = rng.random((5000, 10))
    ref = oracle.self_count_brute(x, 0.35)
    c, st = hj.self_join_count(x, 0.35, active_dims=active_dims, return_stats=True)
    assert c == ref
    assert st["candidate_pairs"] >= c


@pytest.mark.parametrize("form", FORMS)
def test_fp32_input(hj, form):
    rng = np.random.default_rng(3)
    x = rng.random((3000, 16)).astype(np.float32)
    eps = 0.6
    assert hj.self_join_count(x, eps, form=form) == oracle.self_count_brute(x.astype(np.float64), eps)
    b = rng.random((2000, 16)).astype(np.float32)
    assert hj.join_count(x, b, eps, form=form) == \
        oracle.join_count_brute(x.astype(np.float64), b.astype(np.float64), eps)


@pytest.mark.parametrize("form", ["tf32", "bf16x3", "fp16"])
def test_tc_signed_and_scaled_data(hj, form):
    """Mixed-sign coordinates and large magnitudes exercise the band bound."""
    rng = np.random.default_rng(8)
    x = (rng.random((3000, 24)) * 2.0 - 1.0) * 1000.0
    eps = 1500.0
    assert hj.self_join_count(x, eps, form=form) == oracle.self_count_brute(x, eps)
    y = rng.random((2000, 24)) * 1e-3 + 5.0
    eps = 1.1e-3
    assert hj.self_join_count(y, eps, form=form) == oracle.self_count_brute(y, eps)


def test_torch_device_input(hj):
    import torch
    rng = np.random.default_rng(4)
    x = rng.random((3000, 24))
    eps = 0.9
    ref = oracle.self_count_brute(x, eps)
    assert hj.self_join_count(torch.from_numpy(x).cuda(), eps) == ref
    assert hj.self_join_count(torch.from_numpy(x).float().cuda(), eps) == \
        oracle.self_count_brute(x.astype(np.float32).astype(np.float64), eps)


def test_ego_sort_matches_oracle(hj):
    """The device EGO order is the oracle's stable lexicographic cell order, bit for bit."""
    import ctypes
    from hilbertjoin_b200 import workloads as W
    for x, eps in ((np.random.default_rng(1).random((5000, 7)), 0.2), (W.gmm(4000, 28, 2), 0.03),
                   (W.lattice(3000, 5, 9, levels=4), 0.1), (np.random.default_rng(2).random((4000, 64)), 0.2)):
        x = np.ascontiguousarray(x)
        perm = np.zeros(x.shape[0], dtype=np.uint64)
        srt = np.zeros_like(x)
        o = hj.Opts()
        hj.lib().hj_opts_init(ctypes.byref(o))
        st = hj.lib().hj_ego_sort
        st.restype = ctypes.c_int
        st.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_void_p]
        r = st(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], eps, ctypes.byref(o),
               perm.ctypes.data_as(ctypes.c_void_p), srt.ctypes.data_as(ctypes.c_void_p))
        assert r == 0
        assert np.array_equal(perm, oracle.ego_order(x, eps))
        assert np.array_equal(srt, x[perm.astype(np.int64)])


def test_invalid_inputs(hj):
    x = np.random.default_rng(0).random((100, 4))
    with pytest.raises(hj.HJError) as e:
        hj.self_join_count(x, -1.0)
    assert e.value.status == 1
    y = x.copy()
    y[3, 2] = np.nan
    with pytest.raises(hj.HJError) as e:
        hj.self_join_count(y, 0.1)
    assert e.value.status == 1
    assert hj.self_join_count(x[:0], 0.1) == 0


def test_reference_signature_dropins(hj):
    by = {c["name"]: c for c in GOLDEN}
    c = by["self_uniform_d16"]
    x = make(c)
    before = x.copy()
    cnt, st, it, lp = hj.test_ego_loop3_macro(x, c["eps"], 14)
    assert cnt == c["ref_count"]
    assert np.array_equal(x, before)  # the input is not permuted (the reference's is)
    c = by["join_uniform_d20"]
    a = make(c)
    b = make(dict(c, seed=c["seed_b"], n=c["m"]))
    cnt, *_ = hj.test_ego_loop3_noself(a, b, c["eps"])
    assert cnt == c["ref_count"]


def test_medium_sparse_config_shape(hj):
    """The repository example's shape (uniform, d=64, eps=0.2) at n=50k: no pairs,
    and the stripes prune most of the grid."""
    x = np.random.default_rng(1).random((50_000, 64))
    c, st = hj.self_join_count(x, 0.2, return_stats=True)
    assert c == 0
    assert st["loadpercent"] < 60.0


@pytest.mark.parametrize("form", ["plain", "tf32"])
@pytest.mark.parametrize("K", [2, 3, 4])
def test_shards_sum_to_full_count(hj, form, K):
    """The device shard selection (equal-load ranges of the work list) partitions the
    work: the shard counts sum to the oracle's brute-force count."""
    import oracle
    from hilbertjoin_b200 import workloads as W
    x = W.gmm(20000, 16, 5)
    eps = 0.08
    want = oracle.self_count_brute(x, eps)
    parts = [hj.self_join_count(x, eps, form=form, shard=(k, K)) for k in range(K)]
    assert sum(parts) == want
    assert sum(1 for p in parts if p > 0) >= 2  # the work really is split
    a, b = W.uniform(6000, 8, 1), W.uniform(5000, 8, 2)
    want_j = oracle.join_count_brute(a, b, 0.3)
    assert sum(hj.join_count(a, b, 0.3, form=form, shard=(k, K)) for k in range(K)) == want_j
