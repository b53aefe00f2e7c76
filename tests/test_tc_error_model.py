"""The error model behind the tensor-core band, checked on the CPU (the
hardware is checked against the whole bound by tests/test_gpu_tc.py and
tests/test_gpu_block_centring.py).

1. Accumulation. The engine budgets the FP32 accumulation of a K-term dot at
   K * 2^-22 * S, S = sum |a_k b_k|, following the model that Fasi, Higham,
   Mikaitis and Pranesh measured for NVIDIA tensor cores (PeerJ Computer Science
   7:e330, 2021): each hardware step adds k exact products to the accumulator
   after aligning all k + 1 terms to the largest exponent and truncating them to
   24 bits, then truncates the sum to FP32. The emulation below follows that
   model for step sizes k = 2..16 on cancelling and random inputs.
2. Operand rounding. FP16 and TF32 keep 11 significant bits (2^-11 relative per
   operand); the BF16 hi/lo split of an FP32 value drops lo*lo and the split's
   residue, below 3.1 * 2^-16 of |a_k b_k|.
"""
import math

import numpy as np
import pytest

ACC = 2.0 ** -22


def trunc_bits(x, e, bits=24):
    """x truncated toward zero to a multiple of 2^(e - bits) (exact in FP64)."""
    unit = np.ldexp(1.0, e - bits)
    return np.trunc(x / unit) * unit


def tc_dot(prods, k):
    """Model of the tensor core's sum of the product terms prods[:, K] (exact
    values), k per step, FP32 accumulator. Returns the result per row."""
    trials, K = prods.shape
    acc = np.zeros(trials)
    for s in range(0, K, k):
        terms = np.concatenate([acc[:, None], prods[:, s:s + k]], axis=1)
        m = np.abs(terms).max(axis=1)
        _, e = np.frexp(m)  # |term| < 2^e
        aligned = trunc_bits(terms, e[:, None])
        tot = aligned.sum(axis=1)  # exact: fewer than 2^30 units of 2^(e-24)
        _, e2 = np.frexp(np.abs(tot))
        acc = trunc_bits(tot, e2)
    return acc


def fp16_values(rng, shape, spread=6):
    return (rng.standard_normal(shape) * np.ldexp(1.0, rng.integers(-spread, spread, shape))).astype(
        np.float16).astype(np.float64)


@pytest.mark.parametrize("k", [2, 4, 8, 16])
@pytest.mark.parametrize("K", [16, 64, 96, 256, 768])
def test_accumulation_within_K_2m22_S(k, K):
    rng = np.random.default_rng(1000 * k + K)
    trials = 400
    a = fp16_values(rng, (trials, K))
    b = fp16_values(rng, (trials, K))
    # half the rows cancel: the second half of the terms nearly undoes the
    # first, so the running sum climbs far above the result
    h, c = K // 2, trials // 2
    a[:c, h:2 * h] = a[:c, :h]
    b[:c, h:2 * h] = (-b[:c, :h] * (1.0 + 2.0 ** -8 * rng.standard_normal((c, h)))).astype(
        np.float16).astype(np.float64)
    prods = a * b  # FP16 x FP16: 22 significant bits, exact in FP64
    exact = np.array([math.fsum(r) for r in prods])  # correctly rounded: within 2^-53 S
    S = np.abs(prods).sum(axis=1)
    got = tc_dot(prods, k)
    err = np.abs(got - exact)
    bound = K * ACC * S + 2.0 ** -52 * S
    ratio = (err / np.where(bound > 0, bound, 1.0)).max()
    print(f"k={k} K={K}: max |err| / (K 2^-22 S) = {ratio:.4f}")
    assert (err <= bound).all(), ratio
    # the model is not vacuous: truncation errors show up on the cancelling rows
    assert err[: trials // 2].max() > 0


def bf16_rn(f):
    """FP32 -> BF16 round to nearest even (finite inputs), as FP32."""
    u = np.asarray(f, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def tf32_rn(f):
    """FP32 -> TF32 (10 stored mantissa bits) round to nearest even, as FP32."""
    u = np.asarray(f, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0xFFF + ((u >> 13) & 1)) & 0xFFFFE000
    return u.astype(np.uint32).view(np.float32)


def test_bf16x3_split_drops_below_3_1_2m16():
    rng = np.random.default_rng(7)
    n = 200_000
    a = (rng.standard_normal(n) * np.ldexp(1.0, rng.integers(-30, 30, n))).astype(np.float32)
    b = (rng.standard_normal(n) * np.ldexp(1.0, rng.integers(-30, 30, n))).astype(np.float32)
    ah = bf16_rn(a)
    bh = bf16_rn(b)
    al = bf16_rn(a - ah)  # a - ah is exact in FP32
    bl = bf16_rn(b - bh)
    A, B = a.astype(np.float64), b.astype(np.float64)
    Ah, Al, Bh, Bl = (v.astype(np.float64) for v in (ah, al, bh, bl))
    three = Ah * Bh + Ah * Bl + Al * Bh  # each product exact in FP64 (16 bits)
    rel = np.abs(three - A * B) / np.abs(A * B)
    print(f"bf16x3: max dropped / |ab| = {rel.max() / 2.0 ** -16:.3f} * 2^-16")
    assert rel.max() <= 3.1 * 2.0 ** -16
    assert rel.max() > 0.5 * 2.0 ** -16  # the bound is near the worst case


@pytest.mark.parametrize("kind", ["fp16", "tf32"])
def test_11_bit_operands(kind):
    rng = np.random.default_rng(11)
    n = 200_000
    if kind == "fp16":
        # FP16's normal range [2^-14, 2^15): the engine scales its operands below
        # 2^15; values under 2^-14 are charged an absolute error instead
        x = rng.choice([-1.0, 1.0], (2, n)) * rng.uniform(1, 2, (2, n)) * np.ldexp(1.0, rng.integers(-14, 15, (2, n)))
        r = x.astype(np.float16).astype(np.float64)
    else:
        x = (rng.standard_normal((2, n)) * np.ldexp(1.0, rng.integers(-60, 60, (2, n)))).astype(np.float32)
        r = tf32_rn(x).astype(np.float64)
        x = x.astype(np.float64)
    u = 2.0 ** -11
    rel_op = np.abs(r - x) / np.abs(x)
    assert rel_op.max() <= u
    rel_prod = np.abs(r[0] * r[1] - x[0] * x[1]) / np.abs(x[0] * x[1])
    assert rel_prod.max() <= 2 * u + u * u


def test_fp16_subnormal_absolute_error():
    """Below 2^-14 FP16 is subnormal: the rounding error is absolute, at most
    half the spacing 2^-24, which the FP16 band charges per product term."""
    rng = np.random.default_rng(13)
    v = rng.uniform(-1, 1, 200_000) * 2.0 ** -14
    err = np.abs(v.astype(np.float16).astype(np.float64) - v)
    assert err.max() <= 2.0 ** -25
    assert err.max() > 0.9 * 2.0 ** -25


def rn_sig_bits(v, p):
    """v rounded to nearest (ties to even) to p significant bits (FP64 emulation)."""
    m, e = np.frexp(v)
    return np.ldexp(np.rint(np.ldexp(m, p)), e - p)


def test_bf16_pair_from_fp64_keeps_17_bits():
    """The block-centred BF16x3 operands: hi = bf16(v), lo = bf16(v - hi) from
    FP64. The pair keeps v to 2^-17 |v| (the rho_u of that form), and
    |lo| <= 2^-8 |v|, so a dropped lo*lo product is below 2^-16 of |v w|."""
    rng = np.random.default_rng(17)
    n = 1_000_000
    v = rng.uniform(-1, 1, n) * np.ldexp(1.0, rng.integers(-20, 10, n))
    w = rng.uniform(-1, 1, n) * np.ldexp(1.0, rng.integers(-20, 10, n))
    vh = rn_sig_bits(v, 8)
    vl = rn_sig_bits(v - vh, 8)
    wh = rn_sig_bits(w, 8)
    wl = rn_sig_bits(w - wh, 8)
    res = np.abs(v - vh - vl) / np.abs(v)
    assert res.max() <= 2.0 ** -17 and res.max() > 0.9 * 2.0 ** -17
    lolo = np.abs(vl * wl) / np.abs((vh + vl) * (wh + wl))
    assert lolo.max() <= 1.001 * 2.0 ** -16 and lolo.max() > 0.9 * 2.0 ** -16
    # the emulation is CUDA's rounding for values in BF16's normal range
    x32 = v.astype(np.float32)
    assert np.array_equal(rn_sig_bits(x32.astype(np.float64), 8), bf16_rn(x32).astype(np.float64))


@pytest.mark.parametrize("form", ["bf16x3", "tf32", "fp16"])
@pytest.mark.parametrize("d", [3, 28, 64, 256])
def test_global_centre_operand_terms(form, d):
    """The one-centre forms without the accumulation term: centred FP64 values,
    FP32 norms, operands as the gather writes them (TF32 and BF16 from the FP32
    value, FP16 from FP64 after an exact power-of-two scale), products summed
    exactly. |s - dist2| stays within the operand part of c_rel (|a|^2 + |b|^2):
    1.25 (p + 14 2^-24 + d 2^-50) with p = 2 2^-11 + 2^-22 (TF32, FP16) or
    3.1 2^-16 (BF16x3)."""
    rng = np.random.default_rng(d + {"bf16x3": 0, "tf32": 1000, "fp16": 2000}[form])
    n = 300
    x = rng.standard_normal((n, d)) * np.ldexp(1.0, rng.integers(-3, 4, d)) + rng.uniform(-50, 50, d)
    c = x - (0.5 * x.min(0) + 0.5 * x.max(0))
    if form == "fp16":
        s_exp = 14 - int(np.floor(np.log2(np.abs(c).max())))
        c = np.ldexp(c, s_exp)  # exact
        ops = (c.astype(np.float16).astype(np.float64),)
    else:
        f = c.astype(np.float32)
        if form == "tf32":
            ops = (tf32_rn(f).astype(np.float64),)
        else:
            hi = bf16_rn(f)
            ops = (hi.astype(np.float64), bf16_rn(f - hi).astype(np.float64))
    norms = (c * c).sum(1).astype(np.float32).astype(np.float64)
    if len(ops) == 1:
        dot = ops[0] @ ops[0].T
    else:
        hi, lo = ops
        dot = hi @ hi.T + hi @ lo.T + lo @ hi.T
    s = norms[:, None] + norms[None, :] - 2 * dot
    ex = ((c[:, None, :] - c[None, :, :]) ** 2).sum(-1)
    u24 = 2.0 ** -24
    p = 2 * 2.0 ** -11 + 2.0 ** -22 if form != "bf16x3" else 3.1 * 2.0 ** -16
    c_rel = 1.25 * (p + 2 * u24 + 12 * u24 + d * 2.0 ** -50)
    bound = c_rel * (norms[:, None] + norms[None, :])
    ratio = np.abs(s - ex) / bound
    print(f"{form} d={d}: max |s - dist2| / operand bound = {ratio.max():.3f}")
    assert ratio.max() <= 1.0, float(ratio.max())
    assert ratio.max() > 0.01  # the operand part is not vacuous
