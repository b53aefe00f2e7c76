"""Per-block centring of the FP16 tensor-core operands (HJ_CENTRING_BLOCK):
every 128-rank block of the EGO order is stored as an FP16 centre plus FP16
residuals, with the centre cross terms and the column's norm as extra K
columns. The counts must be
the FP64 counts on every input, including pairs exactly at eps and the
clustered data that the global centre sends to the FP64 kernel; the estimates
must sit inside a bound that scales with the residuals."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200
    return hilbertjoin_b200


def exact_dist2(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    out = np.empty((a.shape[0], b.shape[0]))
    for i0 in range(0, a.shape[0], 128):
        out[i0:i0 + 128] = ((a[i0:i0 + 128, None, :] - b[None, :, :]) ** 2).sum(-1)
    return out


def tight_clusters(n, d, seed, k=12, sigma=0.004, dtype=np.float32):
    """k clusters of spread sigma with means spread over [0, 1)^d: eps near the
    cluster-mate distances is far below the spread of the data."""
    rng = np.random.default_rng(seed)
    means = rng.random((k, d))
    lab = rng.integers(0, k, n)
    return (means[lab] + sigma * rng.standard_normal((n, d))).astype(dtype)


def eps_for(x, nbrs, seed=0):
    from hilbertjoin_b200 import workloads as W
    return W.calibrate_eps(x, x.shape[0], nbrs, sample=min(4000, x.shape[0]))


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
@pytest.mark.parametrize("n,d", [(20000, 28), (9000, 64), (12000, 8), (5003, 3), (3001, 1), (1000 + 37, 16)])
def test_self_counts_block_forced(hj, n, d, form):
    x = tight_clusters(n, d, 100 + d)
    eps = eps_for(x, 40)
    want = oracle.self_count_brute(x.astype(np.float64), eps)
    got, st = hj.self_join_count(x, eps, form=form, centring="block", return_stats=True)
    assert got == want, (n, d, form, got, want)
    assert st["tc_centring"] == "block"
    assert st["form_used"] == "tc_" + form


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_join_counts_block_forced(hj, dtype, form):
    a = tight_clusters(7001, 20, 5, dtype=dtype)
    b = tight_clusters(9100, 20, 5, dtype=dtype)[::-1].copy()
    eps = eps_for(a, 30)
    want = oracle.join_count_brute(a.astype(np.float64), b.astype(np.float64), eps)
    got, st = hj.join_count(a, b, eps, form=form, centring="block", return_stats=True)
    assert got == want
    assert st["tc_centring"] == "block"


def test_uniform_and_dense_block_forced(hj):
    """Uniform data, sparse and dense eps (the dense case: one cell, blocks in
    norm order rather than cluster order, residuals as large as the data)."""
    rng = np.random.default_rng(77)
    x = rng.random((8000, 24)).astype(np.float32)
    for eps in (0.35, 0.9, 2.5):
        want = oracle.self_count_brute(x.astype(np.float64), eps)
        assert hj.self_join_count(x, eps, form="fp16", centring="block") == want, eps


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
def test_lattice_ties_at_eps(hj, form):
    """Points on a 0.125 lattice (exact in binary): many pairs lie exactly at
    eps, where only the FP64 test decides; every such pair must reach the band
    (or be certain) and the count must be the FP64 count."""
    rng = np.random.default_rng(3)
    x = (rng.integers(0, 9, (6000, 6)) * 0.125 + 3.0).astype(np.float64)
    for eps in (0.125, 0.25, np.sqrt(2) * 0.125, 0.375):
        want = oracle.self_count_brute(x, eps)
        assert hj.self_join_count(x, eps, form=form, centring="block") == want, eps
        assert hj.self_join_count(x.astype(np.float32), eps, form=form, centring="block") == \
            oracle.self_count_brute(x.astype(np.float32).astype(np.float64), eps), eps


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
def test_scaling_and_offsets(hj, form):
    """Offsets far from zero and a dim whose range dwarfs the others (FP16
    subnormal residuals)."""
    rng = np.random.default_rng(9)
    y = tight_clusters(6000, 16, 9, dtype=np.float64) + 1e9
    eps = eps_for(y - 1e9, 40)
    assert hj.self_join_count(y, eps, form=form, centring="block") == oracle.self_count_brute(y, eps)
    z = rng.random((5000, 10))
    z[:, 0] *= 1e6
    z[:, 1:] *= 1e-3
    for eps in (3e3, 4e4):
        assert hj.self_join_count(z, eps, form=form, centring="block") == oracle.self_count_brute(z, eps)


def test_auto_picks_block_for_clustered_small_eps(hj):
    """With one global centre the clustered data's band is wider than eps^2/2
    and its items would run on the FP64 kernel: auto centring switches to
    blocks, keeps them on the tensor cores, and stays exact. The headline-like
    dense uniform case keeps the global centre."""
    from hilbertjoin_b200 import workloads as W
    x = W.gmm(60000, 28, 4, components=16, dtype=np.float32)
    eps = eps_for(x, 60)
    want = oracle.self_count_brute(x.astype(np.float64), eps)
    g, st_g = hj.self_join_count(x, eps, form="fp16", centring="global", return_stats=True)
    a, st_a = hj.self_join_count(x, eps, form="fp16", return_stats=True)
    assert g == want and a == want
    assert st_g["tc_centring"] == "global" and st_g["fp64_items"] > 0
    assert st_a["tc_centring"] == "block"
    assert st_a["fp64_items"] < st_g["fp64_items"]
    u = W.uniform(20000, 64, 22, dtype=np.float32)
    eps_u = W.calibrate_eps(u, 20000, 32)
    cu, st_u = hj.self_join_count(u, eps_u, form="fp16", return_stats=True)
    assert st_u["tc_centring"] == "global"
    assert cu == oracle.self_count_brute(u.astype(np.float64), eps_u)


def test_shards_sum_block(hj):
    x = tight_clusters(15000, 28, 44)
    eps = eps_for(x, 40)
    want = oracle.self_count_brute(x.astype(np.float64), eps)
    parts = [hj.self_join_count(x, eps, form="fp16", centring="block", shard=(k, 3)) for k in range(3)]
    assert sum(parts) == want


def test_ref_compat_block(hj):
    x = tight_clusters(4099, 12, 8)
    eps = eps_for(x, 30)
    plain = hj.self_join_count(x, eps, form="plain", ref_compat=True)
    assert hj.self_join_count(x, eps, form="fp16", centring="block", ref_compat=True) == plain


def test_unsupported_combinations(hj):
    x = tight_clusters(2000, 65, 1)
    with pytest.raises(hj.HJError):
        hj.self_join_count(x, 0.05, form="fp16", centring="block")
    y = tight_clusters(2000, 8, 1)
    with pytest.raises(hj.HJError):
        hj.self_join_count(y, 0.05, form="fp16", centring=7)
    # the plain form ignores the option
    assert hj.self_join_count(y, 0.05, form="plain", centring="block") == \
        oracle.self_count_brute(y.astype(np.float64), 0.05)


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
def test_estimates_all_pairs_loose_bound(hj, form):
    """Every pair estimated (one cell): the error stays within the bound of
    the residual model with the loosest residual, the diameter of the data's
    bounding box, and the estimates are real tensor-core results."""
    rng = np.random.default_rng(12)
    for d in (5, 28, 64):
        a = (rng.standard_normal((600, d)) * 2.0 + 5.0).astype(np.float32)
        b = (rng.standard_normal((800, d)) * 2.0 + 5.0).astype(np.float32)
        est = hj.tc_estimates(a, b, form, centring="block").astype(np.float64)
        ex = exact_dist2(a, b)
        both = np.concatenate([a, b]).astype(np.float64)
        half = 0.5 * (both.max(0) - both.min(0))
        R = float(np.sqrt((half ** 2).sum()))  # |c| <= R (centres inside the box)
        H = 2.0 * R                             # |h| <= diameter of the box
        g, kstep = (4, 8) if form == "tf32" else (8, 16)
        dp = -(-(d + 3) // g) * g                 # block width of the operand rows
        kpad = -(-(3 * dp) // kstep) * kstep      # product terms the MMAs sum
        if form == "bf16x3":
            kpad *= 3                             # three products per K step
        S = 1.5 * (H * H + 2 * H * R)           # cross terms and the folded q / 2
        rho = 2 * 2.0 ** -11 * H
        bound = 2 * kpad * 2.0 ** -22 * S + 2 * rho * np.sqrt(ex) + rho * rho + 1e-5 * (1 + ex)
        assert np.isfinite(est).all()
        assert (np.abs(est - ex) <= bound).all(), (d, float((np.abs(est - ex) / bound).max()))
        assert np.abs(est - ex).max() > 0


def test_estimates_tighter_than_global_on_clusters(hj):
    """Clustered data at a small eps: over the pairs of the work list the block
    estimates are far closer to the exact distances than the global-centre
    ones (the residuals are about sigma sqrt(d), the global norms about 1)."""
    x = tight_clusters(4000, 28, 31, k=6)
    y = tight_clusters(4000, 28, 31, k=6)[::-1].copy()
    eps = eps_for(x, 40)
    eb, st_b = hj.tc_estimates(x, y, "fp16", centring="block", eps=eps, return_stats=True)
    eg, st_g = hj.tc_estimates(x, y, "fp16", centring="global", eps=eps, return_stats=True)
    assert st_b["tc_centring"] == "block"
    ex = exact_dist2(x, y)
    # the bound grows with the distance (2 rho |a - b|): compare near eps
    near = ex <= 4 * eps * eps
    mb = np.isfinite(eb) & near
    mg = np.isfinite(eg) & near
    assert mb.sum() > 1000
    err_b = np.abs(eb[mb].astype(np.float64) - ex[mb])
    # the global run routes most items to FP64 (no estimates there); compare
    # where it has estimates
    if mg.sum() > 0:
        err_g = np.abs(eg[mg].astype(np.float64) - ex[mg]).max()
        assert err_b.max() * 8 < err_g, (err_b.max(), err_g)
    # items on the tensor cores have a band below eps^2 / 2 (blocks that
    # straddle two clusters have large residuals); typical pairs far below
    assert err_b.max() < eps * eps, (err_b.max(), eps)
    assert np.quantile(err_b, 0.99) < 0.02 * eps * eps, (np.quantile(err_b, 0.99), eps)


def test_server_block_centring_switch(hj):
    """The server runs its FP16 joins with one global centre unless asked for
    block centring; with it, clustered requests at a small eps switch to block
    centres. Counts equal the oracle's either way."""
    from hilbertjoin_b200 import serving
    x = tight_clusters(30000, 28, 61)
    eps = eps_for(x, 40)
    want = oracle.self_count_brute(x.astype(np.float64), eps)
    for block in (False, True):
        with serving.Server(form="fp16", max_inflight=2, block_centring=block) as srv:
            sid = srv.upload(x)
            res = [srv.wait(srv.submit(sid, None, eps)) for _ in range(2)]
        assert all(r["status"] == 0 and r["count"] == want for r in res), (block, res)
