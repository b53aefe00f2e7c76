"""The CPU oracle checked against the golden fixtures, which hold counts of the
hilbertJoin reference built from its own sources (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle
from tests.golden.make_golden import make

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_counts.json")))["cases"]


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_oracle_matches_golden(case):
    x = make(case)
    if case["kind"] == "self":
        brute = oracle.self_count_brute(x, case["eps"])
        ego, cand = oracle.self_count_ego(x, case["eps"], 3)
        ego_tail, _ = oracle.self_count_ego(x, case["eps"], 3, tail_drop=True)
        n = x.shape[0]
        assert cand <= n * (n - 1) // 2
    else:
        b = make(dict(case, seed=case["seed_b"], n=case["m"]))
        brute = oracle.join_count_brute(x, b, case["eps"])
        ego, _ = oracle.join_count_ego(x, b, case["eps"], 2)
        ego_tail, _ = oracle.join_count_ego(x, b, case["eps"], 2, tail_drop=True)
    assert brute == case["oracle_count"]
    assert ego == brute
    assert ego_tail == case["oracle_count_tail_drop"]
    if case["ref_valid"]:
        # inside the reference's valid domain the reference itself agrees
        assert case["ref_count"] == case["oracle_count"]


def test_golden_documents_reference_limits():
    by = {c["name"]: c for c in GOLDEN}
    # ties at exactly eps: norm expansion (reference) vs direct difference (oracle)
    assert by["self_lattice_d8_ties"]["ref_count"] != by["self_lattice_d8_ties"]["oracle_count"]
    # d < 8: the reference's bounds miss pairs
    assert by["self_uniform_d4"]["ref_count"] < by["self_uniform_d4"]["oracle_count"]
    # n % 8 != 0: the reference drops the last n % 8 EGO-sorted points
    t = by["self_uniform_tail_n4005"]
    assert t["ref_count"] == t["oracle_count_tail_drop"] < t["oracle_count"]


@pytest.mark.parametrize("active_dims", [0, 1, 2, 3, 4])
def test_stripes_only_change_work(active_dims):
    x = np.random.default_rng(5).random((3000, 12))
    brute = oracle.self_count_brute(x, 0.45)
    c, cand = oracle.self_count_ego(x, 0.45, active_dims)
    assert c == brute


def test_ego_order_is_stable_lexicographic():
    x = np.random.default_rng(9).random((2000, 5))
    eps = 0.3
    perm = oracle.ego_order(x, eps).astype(np.int64)
    cells = oracle.cells(x, eps)[perm]
    for r in range(1, len(perm)):
        a, b = cells[r - 1], cells[r]
        nz = np.nonzero(a != b)[0]
        if nz.size:
            assert a[nz[0]] < b[nz[0]]
        else:
            assert perm[r - 1] < perm[r]  # ties keep input order


@pytest.mark.skipif(oracle.pick_ref_binary() is None, reason="reference binary not built on this host")
def test_reference_egosort_agrees_with_cell_function():
    """The reference's own epsilonGridOrdering output is an EGO order under the
    oracle's cell function floor(x/eps), and a permutation of the input rows."""
    x = np.random.default_rng(3).random((3000, 8))
    eps = 0.25
    s = oracle.ref_ego_sorted(x, eps)
    assert np.array_equal(np.sort(s.view("V64").ravel()), np.sort(x.view("V64").ravel()))
    c = oracle.cells(s, eps)
    for r in range(1, c.shape[0]):
        nz = np.nonzero(c[r - 1] != c[r])[0]
        if nz.size:
            assert c[r - 1][nz[0]] < c[r][nz[0]]


def test_fma_pair_semantics():
    a = np.array([0.3, 0.0])
    b = np.array([0.2, 0.0])
    df = 0.3 - 0.2
    assert oracle.dist2(a, b) == np.float64(df) * np.float64(df)
    # the pair test is inclusive: a pair at exactly eps counts
    x = np.array([[0.0, 0.0], [0.5, 0.0]])
    assert oracle.self_count_brute(x, 0.5) == 1


CONFIGS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config_counts.json")))["configs"]


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_fixture_reference_equals_oracle(name):
    """At the benchmark configurations' stated sizes the reference built from its
    own sources and the oracle return the same count (tests/golden/
    make_config_golden.py), and the fixture's eps is the one the workload
    generator derives now."""
    from hilbertjoin_b200 import workloads as W
    c = CONFIGS[name]
    assert c["ref_count"] == c["oracle_count"], name
    spec = W.CONFIGS[name]
    if "eps" in spec:
        assert c["eps"] == spec["eps"]
    elif name.startswith("cfg4"):
        pytest.skip("regenerating the 4M-point set is left to the GPU test")
    else:
        _, _, eps = W.config_sets(name)
        assert c["eps"] == eps
