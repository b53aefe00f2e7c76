"""The oracle's dimension costs (CPU, no GPU) against the histogram formula of
the reference's outputStatistics (hilbertjoin/egojoin.cpp:553-558):
cost = sum h(h-1)/2 + sum h[c-1] h[c] over the sampled cells of one dim."""
import numpy as np
import pytest

import oracle as O


def _hist_cost(x, eps):
    n = x.shape[0]
    S = min(n, 8192)
    idx = (np.arange(S, dtype=np.uint64) * np.uint64(n) // np.uint64(S)).astype(np.int64)
    cells = np.floor(x[idx] / eps)
    out = []
    for t in range(x.shape[1]):
        v, h = np.unique(cells[:, t], return_counts=True)
        hm = dict(zip(v.tolist(), h.tolist()))
        cost = sum(c * (c - 1) // 2 for c in h.tolist())
        cost += sum(hm.get(a - 1, 0) * b for a, b in zip(v.tolist(), h.tolist()))
        out.append(cost)
    return np.array(out, dtype=np.uint64)


@pytest.mark.parametrize("n,scales,eps", [(500, [1, 0.1, 3], 0.05), (20000, [1, 0.1, 5, 0.01, 2, 1], 0.05),
                                          (9000, [10, -4, 0.5, 1e-3], 0.3)])
def test_dim_costs_equal_histogram_formula(n, scales, eps):
    x = np.random.default_rng(n).random((n, len(scales))) * np.array(scales, dtype=np.float64)
    assert np.array_equal(O.dim_costs(x, eps), _hist_cost(x, eps))


def test_dim_order_is_ascending_cost_with_index_ties():
    x = np.zeros((100, 4))
    x[:, 2] = np.arange(100)  # one point per cell: the cheapest dim
    rd = O.dim_order(x, 0.5)
    # dims 0, 1, 3 tie (all points in one cell) and keep their index order
    assert rd.tolist() == [1, 2, 0, 3]
