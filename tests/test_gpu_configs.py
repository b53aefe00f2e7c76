"""Parity at the benchmark configurations' stated sizes.

Every configuration of ``hilbertjoin_b200.workloads.CONFIGS`` (200k x 64
self-join at eps 0.2, the 200k x 200k x 20 two-set join at eps 0.2 and at an
eps for ~20 partners, the 1M x 64 dense self-join, the 4M x 28 clustered
self-join) runs in every distance form and must return the FP64 oracle's count
recorded in tests/golden/config_counts.json (made by make_config_golden.py:
brute force over all pairs, or the oracle's EGO + stripe count for the 4M
set). The same file records the reference's own count on each configuration;
it must equal the oracle's there as well (checked on the CPU in
test_oracle_golden.py)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_counts.json")
FORMS = ["plain", "fp16", "tf32", "bf16x3"]


def _fixtures():
    if not os.path.exists(GOLDEN):
        return {}
    with open(GOLDEN) as f:
        return json.load(f)["configs"]


FIX = _fixtures()


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    import hilbertjoin_b200 as hj
    return hj


_cache = {}


def _sets(name):
    """Device copies of a configuration's sets (kept for the module)."""
    import torch
    if name not in _cache:
        _cache.clear()
        from hilbertjoin_b200 import workloads as W
        a, b, eps = W.config_sets(name)
        assert eps == FIX[name]["eps"]
        _cache[name] = (torch.from_numpy(a).cuda(), None if b is None else torch.from_numpy(b).cuda(), eps)
    return _cache[name]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", sorted(FIX))
def test_config_count_equals_oracle(hj, name, form):
    a, b, eps = _sets(name)
    want = FIX[name]["oracle_count"]
    if b is None:
        got, st = hj.self_join_count(a, eps, form=form, return_stats=True)
    else:
        got, st = hj.join_count(a, b, eps, form=form, return_stats=True)
    assert got == want, (name, form, got, want, st["form_used"], st["fp64_items"])
    if name.startswith("cfg4") and form != "plain":
        # eps far below the spread of the clustered data: the join switches to
        # block centres and keeps the work on the tensor cores
        assert st["tc_centring"] == "block", (form, st["tc_centring"], st["fp64_items"])
