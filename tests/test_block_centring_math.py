"""The algebra of per-block centring, checked on the CPU with numpy (FP16
rounding by numpy's float16, products exact in FP64): the operand rows
[h | h | c m | h a] read as the windows B = [0, 3dp) and A = [dp, 4dp) give
w = x'_i.x'_j - c_i.c_j - q_j / 2 for the stored points x' = c + h; the three
FP16 pieces of q / 2 reproduce it to 2^-33; and s = q_i + |c_i - c_j|^2 - 2 w
is within the linear bound 2 rho dist + rho^2 (rho = 2^-11 (|h_i| + |h_j|) +
the subnormal floor) of the exact distance, for d = 1 .. 64. The BF16x3 form
(hi + lo pairs, three products per term) is checked the same way with
rho = 2^-17 (|h_i| + |h_j|) and the dropped lo.lo products below 2^-16 S."""
import numpy as np
import pytest

F16 = np.float16


def f16(v):
    return np.asarray(v, dtype=np.float64).astype(F16).astype(np.float64)


def bc_rows(x):
    """Block-centred rows of points x (already sorted into 128-point blocks)."""
    n, d = x.shape
    g = 0.5 * x.min(0) + 0.5 * x.max(0)
    scale = 2.0 ** (14 - np.floor(np.log2(np.abs(x - g).max())) - 5)
    X = (x - g) * scale
    assert np.abs(X).max() < 2 ** 10
    dp = -(-(d + 3) // 8) * 8
    blocks = -(-n // 128)
    R = np.zeros((blocks * 128, 4 * dp))
    q = np.zeros(blocks * 128)
    cent = np.zeros((blocks, d))
    for b in range(blocks):
        r0, r1 = b * 128, min(n, b * 128 + 128)
        Xb = X[r0:r1]
        c = f16(0.5 * Xb.min(0) + 0.5 * Xb.max(0))
        h = f16(Xb - c)
        cent[b] = c
        qq = (h * h).sum(1) + 2 * (h * c).sum(1)
        v1 = 0.5 * qq
        m1 = f16(v1 * 2.0 ** -15)
        v2 = v1 - m1 * 2.0 ** 15
        m2 = f16(v2 * 2.0 ** -4)
        v3 = v2 - m2 * 2.0 ** 4
        m3 = f16(v3 * 2.0 ** 7)
        rem = v1 - (m1 * 2.0 ** 15 + m2 * 2.0 ** 4 + m3 * 2.0 ** -7)
        assert (np.abs(rem) <= 2.0 ** -33 * np.abs(qq) + 2.0 ** -32).all()
        for m in (m1, m2, m3):
            assert np.abs(m).max() < 2 ** 12
        R[r0:r1, 0:d] = h
        R[r0:r1, dp:dp + d] = h
        R[r0:r1, 2 * dp:2 * dp + d] = c
        R[r0:r1, 2 * dp + d] = m1
        R[r0:r1, 2 * dp + d + 1] = m2
        R[r0:r1, 2 * dp + d + 2] = m3
        R[r0:r1, 3 * dp:3 * dp + d] = h
        R[r0:r1, 3 * dp + d:3 * dp + d + 3] = [-2.0 ** 15, -2.0 ** 4, -2.0 ** -7]
        q[r0:r1] = qq
    assert (f16(R) == R).all()  # every stored value is an FP16 value
    return X, R, q, cent, dp


@pytest.mark.parametrize("d", [1, 3, 8, 28, 29, 61, 64])
def test_windows_give_the_distance(d):
    rng = np.random.default_rng(d)
    k = 5
    means = rng.random((k, d))
    lab = np.repeat(np.arange(k), 128)  # one cluster per 128-point block, as EGO order tends to give
    x = means[lab] + 0.004 * rng.standard_normal((lab.size, d))
    X, R, q, cent, dp = bc_rows(x)
    n = x.shape[0]
    Rz = np.concatenate([R, np.zeros((R.shape[0], 64))], 1)  # the copy's zero fill past the row end
    A = Rz[:n, dp:4 * dp]
    B = Rz[:n, 0:3 * dp]
    w = A @ B.T
    bi = np.arange(n) // 128
    D = ((cent[bi][:, None, :] - cent[bi][None, :, :]) ** 2).sum(-1)
    s = q[:n, None] + D - 2 * w
    ex = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    hn = np.sqrt(((X - cent[bi]) ** 2).sum(1))
    rho = 2.0 ** -11 * (hn[:, None] + hn[None, :]) + 2 * np.sqrt(d) * 2.0 ** -25
    bound = 2 * rho * np.sqrt(ex) + rho * rho + 1e-9 * (1 + ex)
    assert (np.abs(s - ex) <= bound).all(), float((np.abs(s - ex) / bound).max())
    # the bound is not vacuous: the residuals are small against the data
    assert np.median(hn) < 0.1 * np.abs(X).max()


def rn8(v):
    """Round to nearest even with 8 significant bits (BF16 in its normal range)."""
    m, e = np.frexp(np.asarray(v, dtype=np.float64))
    return np.ldexp(np.rint(np.ldexp(m, 8)), e - 8)


def pair(v):
    """The BF16 hi + lo pair of v (lo = BF16 of the exact remainder)."""
    hi = rn8(v)
    return hi, rn8(v - hi)


def bc_rows_bf16(x):
    """The same rows for the BF16x3 form: every value a hi + lo pair, q / 2 in
    three pair-valued pieces against constants -1."""
    n, d = x.shape
    g = 0.5 * x.min(0) + 0.5 * x.max(0)
    scale = 2.0 ** (14 - np.floor(np.log2(np.abs(x - g).max())) - 5)
    X = (x - g) * scale
    dp = -(-(d + 3) // 8) * 8
    blocks = -(-n // 128)
    Rh = np.zeros((blocks * 128, 4 * dp))
    Rl = np.zeros_like(Rh)
    q = np.zeros(blocks * 128)
    cent = np.zeros((blocks, d))
    for b in range(blocks):
        r0, r1 = b * 128, min(n, b * 128 + 128)
        Xb = X[r0:r1]
        ch, cl = pair(0.5 * Xb.min(0) + 0.5 * Xb.max(0))
        c = ch + cl
        hh, hl = pair(Xb - c)
        h = hh + hl
        cent[b] = c
        qq = (h * h).sum(1) + 2 * (h * c).sum(1)
        pieces, v = [], 0.5 * qq
        for _ in range(3):
            ph, pl = pair(v)
            pieces.append((ph, pl))
            v = v - (ph + pl)
        assert (np.abs(v) <= 2.0 ** -45 * np.abs(qq) + 2.0 ** -60).all()
        for R, part in ((Rh, 0), (Rl, 1)):
            hv, cv = (hh, ch) if part == 0 else (hl, cl)
            R[r0:r1, 0:d] = hv
            R[r0:r1, dp:dp + d] = hv
            R[r0:r1, 2 * dp:2 * dp + d] = cv
            for t in range(3):
                R[r0:r1, 2 * dp + d + t] = pieces[t][part]
            R[r0:r1, 3 * dp:3 * dp + d] = hv
        Rh[r0:r1, 3 * dp + d:3 * dp + d + 3] = -1.0
        q[r0:r1] = qq
    assert (rn8(Rh) == Rh).all() and (rn8(Rl) == Rl).all()  # every stored value is a BF16 value
    return X, Rh, Rl, q, cent, dp


@pytest.mark.parametrize("d", [1, 3, 28, 64])
def test_bf16x3_windows_within_the_pair_bound(d):
    """BF16x3: the three MMAs (hi.hi + hi.lo + lo.hi) give s within
    2 rho dist + rho^2 + 2 * 2^-16 S of the exact distance, rho = 2^-17 (|h_i| +
    |h_j|): the pair keeps 17 bits and the dropped lo.lo products stay below
    2^-16 of S = sum |A_k B_k|."""
    rng = np.random.default_rng(100 + d)
    k = 4
    means = rng.random((k, d))
    lab = np.repeat(np.arange(k), 128)
    x = means[lab] + 0.004 * rng.standard_normal((lab.size, d))
    X, Rh, Rl, q, cent, dp = bc_rows_bf16(x)
    n = x.shape[0]
    pad = np.zeros((Rh.shape[0], 64))
    Rh, Rl = np.concatenate([Rh, pad], 1), np.concatenate([Rl, pad], 1)
    Ah, Al = Rh[:n, dp:4 * dp], Rl[:n, dp:4 * dp]
    Bh, Bl = Rh[:n, 0:3 * dp], Rl[:n, 0:3 * dp]
    w = Ah @ Bh.T + Ah @ Bl.T + Al @ Bh.T
    S = np.abs(Ah + Al) @ np.abs(Bh + Bl).T
    bi = np.arange(n) // 128
    D = ((cent[bi][:, None, :] - cent[bi][None, :, :]) ** 2).sum(-1)
    s = q[:n, None] + D - 2 * w
    ex = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    hn = np.sqrt(((X - cent[bi]) ** 2).sum(1))
    rho = 1.001 * 2.0 ** -17 * (hn[:, None] + hn[None, :])
    bound = 2 * rho * np.sqrt(ex) + rho * rho + 2 * 1.001 * 2.0 ** -16 * S + 1e-9 * (1 + ex)
    ratio = np.abs(s - ex) / bound
    assert (ratio <= 1).all(), float(ratio.max())
    print(f"d={d}: max |s - dist2| / bound = {ratio.max():.3f}")
    if d <= 3:
        # where the representation terms dominate, radii of 2^-18 (the constants
        # before the correction) are exceeded by some pairs
        old = rho * np.sqrt(ex) + (rho / 2) ** 2 + 2 * 2.0 ** -18 * S + 1e-9 * (1 + ex)
        assert (np.abs(s - ex) > old).any()


def _trunc(x, e):
    unit = np.ldexp(1.0, e - 24)
    return np.trunc(x / unit) * unit


def _mma_model(acc, prods):
    """One tensor-core step of the accumulation model (Fasi et al. 2021): the
    accumulator and the exact products aligned to the largest exponent and
    truncated to 24 bits, summed, the sum truncated to FP32."""
    terms = np.concatenate([acc[..., None], prods], axis=-1)
    _, e = np.frexp(np.abs(terms).max(-1))
    tot = _trunc(terms, e[..., None]).sum(-1)
    _, e2 = np.frexp(np.abs(tot))
    return _trunc(tot, e2)


def _bc_tau_model(form, d, dp, eps_op, xa, ca, pa, xb, cb, qb, D):
    """bc_constants and bc_tau restated (FP64 here; the kernel rounds the
    constants up to FP32)."""
    cols = 3 * dp
    K = -(-cols // 16) * 16 * (3 if form == "bf16x3" else 1)
    kp21 = 2 * K * 2.0 ** -22 + (2 * 1.001 * 2.0 ** -16 if form == "bf16x3" else 0.0)
    rho_u = 1.001 * 2.0 ** (-17 if form == "bf16x3" else -11)
    floor = (2.0 ** -25 if form == "fp16" else 2.0 ** -134) + 2.0 ** -37
    rho_c = 2 * np.sqrt(d) * floor
    u_norm, u_d = 2.0 ** -23 + 2.0 ** -33, 16 * 2.0 ** -24
    theta = 2 * (d + 2) * 2.0 ** -53 * eps_op ** 2 + 2.0 ** -29
    S = xa * (xb + cb) + ca * xb + 0.5005 * qb
    rho = rho_u * (xa + xb) + 2 * rho_c
    E = kp21 * S + u_norm * (pa + qb) + u_d * D
    return 1.25 * (2 * E + 2 * eps_op * rho + 2 * rho * rho + theta)


@pytest.mark.parametrize("form", ["fp16", "bf16x3"])
@pytest.mark.parametrize("d", [3, 28, 64])
def test_emulated_kernel_classification_is_sound(form, d):
    """End to end under the accumulation model: the block-centred rows, the
    MMAs emulated step by step (16 products per step; BF16x3 as hi.hi, hi.lo,
    lo.hi per K step into one accumulator), s in FP32 terms, and the band
    half-width tau of bc_constants / bc_tau. Every pair the band calls certain
    ("s + tau <= eps^2" inside, "s - tau > eps^2" outside) is on that side of
    eps^2 by the exact distance, and most pairs near eps are certain."""
    rng = np.random.default_rng(7 * d + (form == "bf16x3"))
    k = 2
    means = rng.random((k, d))
    lab = np.repeat(np.arange(k), 128)
    x = means[lab] + 0.004 * rng.standard_normal((lab.size, d))
    if form == "fp16":
        X, R, q, cent, dp = bc_rows(x)
        Rh, Rl = R, np.zeros_like(R)
    else:
        X, Rh, Rl, q, cent, dp = bc_rows_bf16(x)
    n = x.shape[0]
    cols = 3 * dp
    K = -(-cols // 16) * 16
    pad = np.zeros((Rh.shape[0], K + 64))
    Rh, Rl = np.concatenate([Rh, pad], 1), np.concatenate([Rl, pad], 1)
    Ah, Al = Rh[:n, dp:dp + K], Rl[:n, dp:dp + K]
    Bh, Bl = Rh[:n, 0:K], Rl[:n, 0:K]
    passes = [(Ah, Bh)] if form == "fp16" else [(Ah, Bh), (Ah, Bl), (Al, Bh)]
    w = np.zeros((n, n))
    for s0 in range(0, K, 16):
        for P, Q in passes:
            prods = P[:, None, s0:s0 + 16] * Q[None, :, s0:s0 + 16]  # exact in FP64
            w = _mma_model(w, prods)
    bi = np.arange(n) // 128
    cA = cent[bi]
    D = ((cA[:, None, :] - cA[None, :, :]) ** 2).sum(-1)
    q32 = q[:n].astype(np.float32).astype(np.float64)
    s = q32[:, None] + D.astype(np.float32).astype(np.float64) - 2 * w
    ex = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    h = X - cA
    hn = np.sqrt((h * h).sum(1))
    cn = np.sqrt((cent * cent).sum(1))
    qa = np.abs(q[:n])
    blocks = n // 128
    xb = np.array([hn[b * 128:(b + 1) * 128].max() for b in range(blocks)])[bi]
    qb = np.array([qa[b * 128:(b + 1) * 128].max() for b in range(blocks)])[bi]
    same = bi[:, None] == bi[None, :]
    eps2 = float(np.quantile(ex[same & (ex > 0)], 0.3))  # many pairs near eps
    eps_op = np.sqrt(eps2)
    tau = _bc_tau_model(form, d, dp, eps_op, hn[:, None], cn[bi][:, None], qa[:, None], xb[None, :],
                        cn[bi][None, :], qb[None, :], D)
    inside = s + tau <= eps2
    outside = s - tau > eps2
    assert not (inside & (ex > eps2)).any()
    assert not (outside & (ex <= eps2)).any()
    near = np.abs(ex - eps2) < 0.5 * eps2
    assert (inside | outside)[near].mean() > 0.5, float((inside | outside)[near].mean())
