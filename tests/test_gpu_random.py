"""Randomised parity sweep: seeded random joins -- sizes, dimensions, data
kinds, eps, forms and options drawn at random -- each checked against the
oracle's brute-force count (exact integers). Complements the hand-picked
cases with combinations nobody thought of."""
import numpy as np
import pytest

import oracle as O
from hilbertjoin_b200 import workloads as W

pytestmark = pytest.mark.gpu

N_CASES = 48


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200 as hj
    return hj


def draw(rng, n, d, kind):
    if kind == "uniform":
        return rng.random((n, d))
    if kind == "gmm":
        return W.gmm(n, d, int(rng.integers(1 << 30)), components=int(rng.integers(1, 12)))
    if kind == "lattice":
        return 0.25 * rng.integers(0, 6, size=(n, d)).astype(np.float64)
    # offset and scaled: large coordinates, small spread
    return 1e4 + rng.random((n, d)) * float(rng.choice([1e-3, 1.0, 50.0]))


def case(i):
    rng = np.random.default_rng(1000 + i)
    d = int(rng.choice([1, 2, 3, 5, 8, 13, 16, 28, 33, 64, 65, 100, 128, 129, 200, 256]))  # every form: d <= 256
    kind = str(rng.choice(["uniform", "gmm", "lattice", "offset"]))
    self_join = rng.random() < 0.6
    na = int(rng.integers(1, 4000))
    nb = int(rng.integers(1, 3000))
    a = draw(rng, na, d, kind)
    b = None if self_join else draw(rng, nb, d, kind)
    if rng.random() < 0.5:
        a = a.astype(np.float32)
        b = None if b is None else b.astype(np.float32)
    # eps: from a sample's pair distances (0.1% .. 30% quantile), or a lattice step
    s = a[: min(na, 400)].astype(np.float64)
    d2 = ((s[:, None, :] - s[None, :, :]) ** 2).sum(-1)[np.triu_indices(len(s), 1)] if len(s) > 1 else np.ones(1)
    q = float(rng.choice([0.001, 0.01, 0.05, 0.3]))
    eps = float(np.sqrt(np.quantile(d2, q))) if d2.size else 1.0
    if kind == "lattice" and rng.random() < 0.5:
        eps = 0.25 * float(rng.integers(1, 4))  # exact ties at eps
    eps = max(eps, 1e-6)
    form = str(rng.choice(["tf32", "fp16", "bf16x3", "auto", "plain"]))
    opts = {"active_dims": int(rng.integers(0, 6)), "item_chunk": int(rng.choice([0, 1, 5, 64]))}
    if rng.random() < 0.3:
        opts["reorder_dims"] = True
    return a, b, eps, form, opts


@pytest.mark.parametrize("i", range(N_CASES))
def test_random_case_matches_oracle(hj, i):
    a, b, eps, form, opts = case(i)
    if b is None:
        got = hj.self_join_count(a, eps, form=form, **opts)
        want = O.self_count_brute(a.astype(np.float64), eps)
    else:
        got = hj.join_count(a, b, eps, form=form, **opts)
        want = O.join_count_brute(a.astype(np.float64), b.astype(np.float64), eps)
    assert got == want, (i, a.shape, None if b is None else b.shape, eps, form, opts)
