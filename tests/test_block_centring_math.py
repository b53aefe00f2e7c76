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
