"""Tensor-core forms: the dist^2 estimate of every pair stays inside the error
bound that decides which pairs are re-evaluated in FP64 (the exactness of the
count rests on it), and the band logic returns the FP64 count."""
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


def bound_constants(hj, form, a, b):
    _, st = hj.join_count(a, b, 1e-6, form=form, return_stats=True)
    return st["band_halfwidth_rel"]


@pytest.mark.parametrize("form", ["tf32", "bf16x3", "fp16"])
@pytest.mark.parametrize("d,kind", [(4, "u"), (20, "u"), (32, "u"), (64, "u"), (100, "u"), (128, "u"),
                                    (64, "signed"), (28, "gmm")])
def test_estimates_within_bound(hj, form, d, kind):
    rng = np.random.default_rng(d * 7 + len(kind))
    if kind == "u":
        a, b = rng.random((700, d)), rng.random((900, d))
    elif kind == "signed":
        a, b = rng.standard_normal((700, d)) * 3.0, rng.standard_normal((900, d)) * 3.0
    else:
        from hilbertjoin_b200 import workloads as W
        a, b = W.gmm(700, d, 1), W.gmm(900, d, 2)
    a = a.astype(np.float32)
    b = b.astype(np.float32)
    est = hj.tc_estimates(a, b, form).astype(np.float64)
    ex = exact_dist2(a, b)
    # the engine shifts the tensor-core operands by the midpoint of the
    # coordinate range of both sets; its bound is in the shifted norms
    both = np.concatenate([a, b]).astype(np.float64)
    center = 0.5 * both.min(0) + 0.5 * both.max(0)
    na = ((a.astype(np.float64) - center) ** 2).sum(1)
    nb = ((b.astype(np.float64) - center) ** 2).sum(1)
    c_rel = bound_constants(hj, form, a, b)
    bound = c_rel * (na[:, None] + nb[None, :])
    ratio = np.abs(est - ex) / bound
    assert np.isfinite(est).all()
    assert ratio.max() < 1.0, (form, d, kind, float(ratio.max()))
    # the estimate is a real tensor-core result, not a copy of the FP64 value
    assert np.abs(est - ex).max() > 0


@pytest.mark.parametrize("form", ["tf32", "bf16x3", "fp16"])
def test_band_pairs_are_rechecked(hj, form):
    """eps set at the median distance puts many pairs in the band; the count is
    still the FP64 count and the reported max error respects the bound."""
    rng = np.random.default_rng(21)
    x = rng.random((4000, 32)).astype(np.float32)
    d2 = exact_dist2(x[:500], x[500:1500])
    eps = float(np.sqrt(np.median(d2)))
    c, st = hj.self_join_count(x, eps, form=form, return_stats=True)
    assert c == oracle.self_count_brute(x.astype(np.float64), eps)
    assert st["band_pairs"] > 0
    assert st["max_abs_err_band"] <= st["band_halfwidth_rel"] * 2 * 32 * 1.0


def test_forms_agree_dense(hj):
    """The dense single-cell regime of the headline configuration, at a size the
    oracle still covers: all forms give the FP64 count."""
    from hilbertjoin_b200 import workloads as W
    x = W.uniform(20000, 64, 22, dtype=np.float32)
    eps = W.calibrate_eps(x, 20000, 32)
    want = oracle.self_count_brute(x.astype(np.float64), eps)
    for form in ("plain", "tf32", "bf16x3", "fp16"):
        assert hj.self_join_count(x, eps, form=form) == want, form


@pytest.mark.parametrize("d", [160, 256])
def test_wide_ill_conditioned_routes_to_fp64(hj, d):
    """Two unit-variance clusters 1000 apart in every dim, at d > 128: the
    centred squared norms (~d * 500^2) dwarf eps^2 (~2d), so the tensor-core
    bound is far too wide and the work items are routed to the plain FP64
    kernel, which runs d > 128 by 64-dim chunks of the B tiles. Counts stay the
    FP64 counts."""
    rng = np.random.default_rng(1017)

    def pts(n):
        return (1000.0 * rng.integers(0, 2, n)[:, None] + rng.standard_normal((n, d))).astype(np.float32)

    a, b = pts(2939), pts(2917)
    s = a[:400].astype(np.float64)
    eps = float(np.sqrt(np.quantile(exact_dist2(s, s)[np.triu_indices(400, 1)], 0.1)))
    want_j = oracle.join_count_brute(a.astype(np.float64), b.astype(np.float64), eps)
    want_s = oracle.self_count_brute(a.astype(np.float64), eps)
    _, plain_j = hj.join_count(a, b, eps, form="plain", return_stats=True)
    _, plain_s = hj.self_join_count(a, eps, form="plain", return_stats=True)
    for form in ("fp16", "tf32", "bf16x3", "plain"):
        got, st = hj.join_count(a, b, eps, form=form, return_stats=True)
        assert got == want_j, form
        got_s, st_s = hj.self_join_count(a, eps, form=form, return_stats=True)
        assert got_s == want_s, form
        if form != "plain":
            # every item routed: the join runs on the plain form's finer work list
            assert st["fp64_items"] > 0 and st_s["fp64_items"] > 0, form
            assert st["candidate_pairs"] == plain_j["candidate_pairs"], form
            assert st_s["candidate_pairs"] == plain_s["candidate_pairs"], form


def test_fp16_scaling_extremes(hj):
    """FP16 operands are scaled so the largest centred coordinate lands in
    [2^14, 2^15): a dim whose range dwarfs the others drives the small ones
    into FP16 subnormals (covered by the bound's absolute term), and offsets
    far from zero are removed by the centring. Counts stay the FP64 counts."""
    rng = np.random.default_rng(44)
    x = rng.random((4000, 12))
    x[:, 0] *= 1e6
    x[:, 1:] *= 1e-3
    for eps in (2e3, 5e4):
        assert hj.self_join_count(x, eps, form="fp16") == oracle.self_count_brute(x, eps)
    y = rng.random((3000, 20)) + 1e12
    eps = float(np.sqrt(np.median(exact_dist2(y[:300] - 1e12, y[300:900] - 1e12)))) * 0.5
    assert hj.self_join_count(y, eps, form="fp16") == oracle.self_count_brute(y, eps)
    z = rng.standard_normal((3000, 40)) * 1e-9
    eps = 4e-9
    assert hj.self_join_count(z, eps, form="fp16") == oracle.self_count_brute(z, eps)


def test_auto_form_picks_by_size_and_stays_exact(hj):
    """auto: the plain FP64 form for small joins (na * nb * d <= 2e10, where its
    fewer stages are faster), FP16 above; the count is the plain form's."""
    from hilbertjoin_b200 import workloads as W
    small = W.uniform(5000, 16, 61, dtype=np.float32)
    eps_s = W.calibrate_eps(small, 5000, 16)
    c, st = hj.self_join_count(small, eps_s, form="auto", return_stats=True)
    assert st["form_used"] == "plain_fp64" and c == hj.self_join_count(small, eps_s)
    big = W.uniform(60000, 16, 62, dtype=np.float32)
    eps_b = W.calibrate_eps(big, 60000, 16)
    c, st = hj.self_join_count(big, eps_b, form="auto", return_stats=True)
    assert st["form_used"] == "tc_fp16" and c == hj.self_join_count(big, eps_b)
    wide = W.uniform(3000, 200, 63, dtype=np.float32)  # d > 128: auto takes FP16 at any size
    eps_w = W.calibrate_eps(wide, 3000, 16)
    c, st = hj.self_join_count(wide, eps_w, form="auto", return_stats=True)
    assert st["form_used"] == "tc_fp16" and c == hj.self_join_count(wide, eps_w)


def _cancellation_sets(d, n_a, n_b, seed):
    """Mixed-sign coordinates of equal magnitude c with small noise: every A
    point has a random sign pattern; half of the B points copy an A point's
    signs on the first d/2 dims and flip them on the rest, so that their dot
    product climbs to about +c^2 d/2 and cancels back to about 0 -- the
    accumulator's running sum peaks far above the result. The other B points
    are random. Centring (per-dim midpoint) leaves the patterns as they are."""
    rng = np.random.default_rng(seed)
    c = 3.0
    sa = rng.choice([-1.0, 1.0], size=(n_a, d))
    sb = rng.choice([-1.0, 1.0], size=(n_b, d))
    pick = rng.integers(0, n_a, size=n_b // 2)
    sb[: n_b // 2, : d // 2] = sa[pick, : d // 2]
    sb[: n_b // 2, d // 2:] = -sa[pick, d // 2:]
    a = c * sa + 0.05 * rng.standard_normal((n_a, d))
    b = c * sb + 0.05 * rng.standard_normal((n_b, d))
    return a.astype(np.float32), b.astype(np.float32), pick


@pytest.mark.parametrize("form", ["tf32", "bf16x3", "fp16"])
def test_estimates_within_bound_under_cancellation(hj, form):
    """K = 256 (d = 256), mixed signs, the running sum of the dot product far
    above its result: every estimate stays within the derived bound. The largest
    |error| / bound ratio is printed for the record."""
    d = 256
    a, b, _ = _cancellation_sets(d, 500, 600, 7)
    est = hj.tc_estimates(a, b, form).astype(np.float64)
    ex = exact_dist2(a, b)
    both = np.concatenate([a, b]).astype(np.float64)
    center = 0.5 * both.min(0) + 0.5 * both.max(0)
    na = ((a.astype(np.float64) - center) ** 2).sum(1)
    nb = ((b.astype(np.float64) - center) ** 2).sum(1)
    c_rel = bound_constants(hj, form, a, b)
    ratio = np.abs(est - ex) / (c_rel * (na[:, None] + nb[None, :]))
    print(f"cancellation d={d} form={form}: max |err|/bound = {ratio.max():.4f}")
    assert np.isfinite(est).all()
    assert ratio.max() < 1.0, (form, float(ratio.max()))


@pytest.mark.parametrize("form", ["tf32", "bf16x3", "fp16"])
def test_count_exact_under_cancellation(hj, form):
    """eps^2 at the median distance of the cancelling pairs: those pairs sit at
    the band; the count is the FP64 oracle's."""
    d = 256
    a, b, pick = _cancellation_sets(d, 1500, 1600, 8)
    d2 = ((a[pick[:300]].astype(np.float64) - b[:300].astype(np.float64)) ** 2).sum(1)
    eps = float(np.sqrt(np.median(d2)))
    want = oracle.join_count_brute(a.astype(np.float64), b.astype(np.float64), eps)
    got, st = hj.join_count(a, b, eps, form=form, return_stats=True)
    assert got == want, (form, got, want, st["band_pairs"], st["fp64_items"])
