"""Pair materialisation (hj_self_join_pairs / hj_join_pairs) against the oracle's
brute-force pair lists: the same (i, j) input-index pairs, in the same sorted
order, bit for bit. The reference's counterpart is its compiled-out
join_pair queue (hilbertjoin/egojoin.h:32-35,
hilbertjoin/test_ego_loop3_queue.cpp:19-37); the pair test is the count
path's, so the list length must equal the count of every form."""
import ctypes

import numpy as np
import pytest

import oracle as O
from hilbertjoin_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200 as hj
    return hj


SELF_CASES = [  # n, d, target neighbours, dtype, seed
    (1, 4, 8, np.float64, 1),
    (2, 3, 8, np.float64, 2),
    (777, 1, 16, np.float64, 3),
    (3001, 3, 16, np.float64, 4),
    (5000, 8, 32, np.float32, 5),
    (4099, 33, 24, np.float64, 6),
    (6000, 64, 64, np.float32, 7),
    (2500, 128, 16, np.float64, 8),
    (2100, 129, 16, np.float32, 9),   # above 128: B tiles in 64-dim chunks
    (1900, 256, 16, np.float64, 10),
]


@pytest.mark.parametrize("n,d,nbr,dtype,seed", SELF_CASES)
def test_self_pairs_match_oracle(hj, n, d, nbr, dtype, seed):
    x = W.uniform(n, d, seed, dtype=dtype)
    eps = W.calibrate_eps(x, n, nbr) if n > 2 else 0.5
    got, st = hj.self_join_pairs(x, eps, return_stats=True)
    want = O.self_pairs_brute(x.astype(np.float64), eps, cap_hint=len(got) + 1)
    assert got.dtype == np.uint64 and got.shape == want.shape
    assert np.array_equal(got, want)
    assert st["form_used"] == "plain_fp64"
    assert len(got) == hj.self_join_count(x, eps)


JOIN_CASES = [  # nA, nB, d, target, dtype, seed
    (1, 500, 6, 8, np.float64, 11),
    (300, 1, 6, 8, np.float64, 12),
    (2000, 3333, 12, 16, np.float64, 13),
    (4100, 900, 40, 32, np.float32, 14),
    (1500, 1500, 100, 16, np.float64, 15),
    (1200, 1700, 200, 16, np.float32, 16),
]


@pytest.mark.parametrize("na,nb,d,nbr,dtype,seed", JOIN_CASES)
def test_join_pairs_match_oracle(hj, na, nb, d, nbr, dtype, seed):
    a = W.uniform(na, d, seed, dtype=dtype)
    b = W.uniform(nb, d, seed + 100, dtype=dtype)
    eps = W.calibrate_eps_join(a, b, nb, nbr) if min(na, nb) > 1 else 0.6
    got = hj.join_pairs(a, b, eps)
    want = O.join_pairs_brute(a.astype(np.float64), b.astype(np.float64), eps, cap_hint=len(got) + 1)
    assert np.array_equal(got, want)
    assert len(got) == hj.join_count(a, b, eps)


def test_pairs_clustered_duplicates_and_ties(hj):
    rng = np.random.default_rng(21)
    # 600 copies of one point: every pair qualifies (distance 0)
    x = np.repeat(rng.random((1, 10)), 600, axis=0)
    got = hj.self_join_pairs(x, 1e-3)
    assert len(got) == 600 * 599 // 2
    assert np.array_equal(got, O.self_pairs_brute(x, 1e-3, cap_hint=len(got)))
    # a lattice with spacing eps: exact ties at distance eps count (<= eps^2)
    g = np.stack(np.meshgrid(*[np.arange(12) * 0.25] * 3, indexing="ij"), -1).reshape(-1, 3)
    got = hj.self_join_pairs(g, 0.25)
    assert np.array_equal(got, O.self_pairs_brute(g, 0.25))
    # Gaussian mixture: dense clusters next to empty space
    y = W.gmm(8000, 16, 22, components=8)
    eps = W.calibrate_eps(y, 8000, 48)
    assert np.array_equal(hj.self_join_pairs(y, eps), O.self_pairs_brute(y, eps))


def test_pairs_are_deterministic_and_consistent_with_all_forms(hj):
    x = W.uniform(20000, 32, 31, dtype=np.float32)
    eps = W.calibrate_eps(x, 20000, 40)
    p1 = hj.self_join_pairs(x, eps)
    p2 = hj.self_join_pairs(x, eps)
    assert np.array_equal(p1, p2)
    for form in ("plain", "tf32", "bf16x3", "fp16"):
        assert hj.self_join_count(x, eps, form=form) == len(p1)


def test_pairs_capacity_contract(hj):
    """More pairs than capacity: nothing written, exact total reported,
    status 10; capacity 0 with a NULL buffer asks for the number."""
    x = W.uniform(3000, 8, 41)
    eps = W.calibrate_eps(x, 3000, 16)
    full = hj.self_join_pairs(x, eps)
    k = len(full)
    assert k > 10
    L = hj.lib()
    o = hj._opts("plain", None, False, None, None)
    cnt = ctypes.c_uint64(0)
    rc = L.hj_self_join_pairs(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], eps, ctypes.byref(o), None,
                              0, ctypes.byref(cnt), None)
    assert rc == hj.ERR_CAPACITY and cnt.value == k
    buf = np.full((k - 1, 2), 7, dtype=np.uint64)
    rc = L.hj_self_join_pairs(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], eps, ctypes.byref(o),
                              buf.ctypes.data_as(ctypes.c_void_p), k - 1, ctypes.byref(cnt), None)
    assert rc == hj.ERR_CAPACITY and cnt.value == k
    assert np.all(buf == 7)  # untouched
    with pytest.raises(hj.HJError):
        hj.self_join_pairs(x, eps, capacity=k - 1)
    assert np.array_equal(hj.self_join_pairs(x, eps, capacity=k), full)


def test_pairs_empty_inputs_and_no_pairs(hj):
    assert hj.self_join_pairs(np.zeros((0, 4)), 0.1).shape == (0, 2)
    assert hj.join_pairs(np.zeros((5, 4)), np.zeros((0, 4)), 0.1).shape == (0, 2)
    x = W.uniform(2000, 5, 51)
    assert hj.self_join_pairs(x, 1e-9).shape == (0, 2)


def test_pairs_ref_compat_drops_the_ego_tail(hj):
    """ref_compat: only the first 8*floor(n/8) EGO-sorted points take part."""
    n = 2003
    x = W.uniform(n, 6, 61)
    eps = W.calibrate_eps(x, n, 16)
    keep = O.ego_order(x, eps)[: n // 8 * 8]
    sub = O.self_pairs_brute(x[keep], eps)
    m = np.sort(keep[sub.astype(np.int64)], axis=1)  # back to input indices, i < j
    want = m[np.lexsort((m[:, 1], m[:, 0]))]
    got = hj.self_join_pairs(x, eps, ref_compat=True)
    assert np.array_equal(got, want)


def test_pairs_shards_partition_the_list(hj):
    x = W.uniform(30000, 16, 71, dtype=np.float32)
    eps = W.calibrate_eps(x, 30000, 32)
    full = hj.self_join_pairs(x, eps)
    parts = [hj.self_join_pairs(x, eps, shard=(k, 3)) for k in range(3)]
    cat = np.concatenate(parts)
    cat = cat[np.lexsort((cat[:, 1], cat[:, 0]))]
    assert np.array_equal(cat, full)


def test_pairs_medium_size_properties(hj):
    """200k x 16: too large for the brute-force pair list, so check the
    properties: count equals the tensor-core count, sorted and unique, i < j,
    every listed pair within eps (oracle dist2), per-row degrees of a sample
    equal the oracle's row counts."""
    n, d = 200_000, 16
    x = W.gmm(n, d, 81, components=16, dtype=np.float32)
    eps = W.calibrate_eps(x, n, 24)
    p = hj.self_join_pairs(x, eps)
    assert len(p) == hj.self_join_count(x, eps, form="tf32")
    assert np.all(p[:, 0] < p[:, 1])
    key = p[:, 0] * np.uint64(n) + p[:, 1]
    assert np.all(key[1:] > key[:-1])
    x64 = x.astype(np.float64)
    rng = np.random.default_rng(3)
    for k in rng.integers(0, len(p), 2000):
        i, j = int(p[k, 0]), int(p[k, 1])
        assert O.dist2(x64[i], x64[j]) <= eps * eps
    rows = rng.integers(0, n, 64).astype(np.uint64)
    deg = np.bincount(p[:, 0].astype(np.int64), minlength=n) + np.bincount(p[:, 1].astype(np.int64), minlength=n)
    assert np.array_equal(deg[rows.astype(np.int64)].astype(np.uint64), O.self_row_counts(x64, eps, rows))


def test_pairs_reject_large_d(hj):
    """The plain FP64 kernel, which lists the pairs, covers d <= 256."""
    with pytest.raises(hj.HJError):
        hj.self_join_pairs(np.zeros((10, 257)), 0.1)
    with pytest.raises(hj.HJError):
        hj.self_join_count(np.zeros((10, 257)), 0.1, form="plain")
