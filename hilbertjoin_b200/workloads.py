"""Seeded synthetic point sets for the epsilon-join benchmarks and tests.

No dataset ships with the engine and the reference's paper datasets are not
reachable, so every workload is generated from a seed with the shapes, sizes
and value distributions of the benchmark configurations:

* ``uniform``: i.i.d. U[0,1) coordinates (the reference's own default data,
  util/dataIo.cpp:4-33, there drawn with MKL's MCG31 generator; here with
  numpy's PCG64 from the seed);
* ``gmm``: a clustered mixture -- component means U[0,1)^d, isotropic sigma
  log-uniform in [sigma_lo, sigma_hi], weights Dirichlet(1), clipped to [0,1);
* ``lattice``: coordinates on a grid of step ``step`` (exact ties at eps),
  used to pin the tie semantics of the pair test.

``calibrate_eps`` picks eps so that the mean number of neighbours per point is
a target, from a 10,000-point sample of the same set.
"""
from __future__ import annotations

import numpy as np

ONE_BELOW = np.nextafter(1.0, 0.0)


def uniform(n: int, d: int, seed: int, dtype=np.float64) -> np.ndarray:
    x = np.random.default_rng(seed).random((n, d))
    return x.astype(dtype) if dtype != np.float64 else x


def gmm(n: int, d: int, seed: int, components: int = 64, sigma_lo: float = 0.005, sigma_hi: float = 0.05,
        dtype=np.float64) -> np.ndarray:
    rng = np.random.default_rng(seed)
    means = rng.random((components, d))
    sig = np.exp(rng.uniform(np.log(sigma_lo), np.log(sigma_hi), size=components))
    w = rng.dirichlet(np.ones(components))
    comp = rng.choice(components, size=n, p=w)
    x = means[comp] + sig[comp, None] * rng.standard_normal((n, d))
    x = np.clip(x, 0.0, ONE_BELOW)
    return x.astype(dtype) if dtype != np.float64 else x


def lattice(n: int, d: int, seed: int, step: float = 0.1, levels: int = 10) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return step * rng.integers(0, levels, size=(n, d)).astype(np.float64)


def _pair_dist2_sample(x: np.ndarray) -> np.ndarray:
    """All unordered pairwise squared distances of x (FP64 Gram form, by blocks).
    Only used to pick eps; the result is rounded to 7 digits by the callers."""
    x = np.asarray(x, dtype=np.float64)
    m = x.shape[0]
    nrm = (x * x).sum(1)
    out = []
    blk = 1024
    for i0 in range(0, m, blk):
        a = x[i0:i0 + blk]
        d2 = nrm[i0:i0 + blk, None] + nrm[None, :] - 2.0 * (a @ x.T)
        ii = np.arange(i0, i0 + a.shape[0])[:, None]
        jj = np.arange(m)[None, :]
        out.append(d2[jj > ii])
    return np.concatenate(out) if out else np.zeros(0)


def calibrate_eps(x: np.ndarray, n_total: int, mean_neighbours: float, sample: int = 10_000) -> float:
    """eps such that a point has about `mean_neighbours` neighbours within eps
    in a set of `n_total` points drawn like x, estimated from the first `sample`
    points: eps = sqrt(quantile(dist^2, mean_neighbours / (n_total - 1))).
    Rounded to 7 significant digits so that the value is reproducible."""
    s = np.asarray(x[:sample], dtype=np.float64)
    d2 = _pair_dist2_sample(s)
    q = min(1.0, mean_neighbours / max(1, n_total - 1))
    k = max(0, min(d2.size - 1, int(np.floor(q * d2.size))))
    v = np.partition(d2, k)[k]
    return float(f"{np.sqrt(v):.7g}")


def calibrate_eps_join(a: np.ndarray, b: np.ndarray, nb_total: int, mean_neighbours: float,
                       sample: int = 4_000) -> float:
    """eps for about `mean_neighbours` B-partners per point of A."""
    sa = np.asarray(a[:sample], dtype=np.float64)
    sb = np.asarray(b[:sample], dtype=np.float64)
    d2 = ((sa[:, None, :] - sb[None, :, :]) ** 2).sum(-1).ravel()
    q = min(1.0, mean_neighbours / max(1, nb_total))
    k = max(0, min(d2.size - 1, int(np.floor(q * d2.size))))
    v = np.partition(d2, k)[k]
    return float(f"{np.sqrt(v):.7g}")


# The benchmark configurations at their stated sizes. Every set is regenerated
# from its seed; `eps` is either the configuration's stated value or calibrated
# (and rounded to 7 digits) from the first points of the same set.
CONFIGS = {
    "cfg1_self_200k_d64": dict(kind="self", gen="uniform", dtype="f64", n=200_000, d=64, seed=1, eps=0.2),
    "cfg2_join_200k_d20": dict(kind="join", gen="uniform", dtype="f32", n=200_000, m=200_000, d=20, seed=2,
                               seed_b=3, eps=0.2),
    "cfg2_join_200k_d20_nbrs20": dict(kind="join", gen="uniform", dtype="f32", n=200_000, m=200_000, d=20, seed=2,
                                      seed_b=3, nbrs=20),
    "cfg3_self_1M_d64_nbrs32": dict(kind="self", gen="uniform", dtype="f32", n=1_000_000, d=64, seed=22, nbrs=32),
    "cfg4_self_4M_d28_gmm64_nbrs100": dict(kind="self", gen="gmm", dtype="f32", n=4_000_000, d=28, seed=4,
                                           components=64, nbrs=100),
}


def config_sets(name: str):
    """(A, B or None, eps) of a benchmark configuration; A and B in the
    configuration's storage type (float32 or float64)."""
    c = CONFIGS[name]
    dt = np.float32 if c["dtype"] == "f32" else np.float64
    if c["gen"] == "uniform":
        a = uniform(c["n"], c["d"], c["seed"], dtype=dt)
    else:
        a = gmm(c["n"], c["d"], c["seed"], components=c["components"], dtype=dt)
    b = uniform(c["m"], c["d"], c["seed_b"], dtype=dt) if c["kind"] == "join" else None
    if "eps" in c:
        eps = c["eps"]
    elif b is None:
        eps = calibrate_eps(a, c["n"], c["nbrs"])
    else:
        eps = calibrate_eps_join(a, b, c["m"], c["nbrs"])
    return a, b, eps
