"""The oracle's pair lists (CPU, no GPU): their length is the oracle's count,
they are sorted by (i, j), self pairs have i < j, and every listed pair and
no other satisfies the pair test (checked against a numpy restatement of the
FMA chain on small inputs)."""
import numpy as np

import oracle as O


def _np_pairs(a, b, eps, self_join):
    out = []
    for i in range(a.shape[0]):
        for j in range(i + 1 if self_join else 0, b.shape[0]):
            if O.dist2(a[i], b[j]) <= eps * eps:
                out.append((i, j))
    return np.array(out, dtype=np.uint64).reshape(-1, 2)


def test_self_pairs_small_exact():
    x = np.random.default_rng(1).random((300, 5))
    eps = 0.2
    got = O.self_pairs_brute(x, eps, cap_hint=1)  # exercises the regrow path
    assert np.array_equal(got, _np_pairs(x, x, eps, True))
    assert len(got) == O.self_count_brute(x, eps)


def test_join_pairs_small_exact():
    rng = np.random.default_rng(2)
    a, b = rng.random((200, 4)), rng.random((170, 4))
    got = O.join_pairs_brute(a, b, 0.15)
    assert np.array_equal(got, _np_pairs(a, b, 0.15, False))
    assert len(got) == O.join_count_brute(a, b, 0.15)


def test_pairs_sorted_and_counted_at_medium_size():
    x = np.random.default_rng(3).random((6000, 12))
    eps = 0.45
    p = O.self_pairs_brute(x, eps)
    assert len(p) == O.self_count_brute(x, eps) > 0
    assert np.all(p[:, 0] < p[:, 1])
    key = p[:, 0] * np.uint64(len(x)) + p[:, 1]
    assert np.all(key[1:] > key[:-1])
