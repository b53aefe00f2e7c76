"""The entry point's smoke check (one small self-join and one two-set join in
every form against the oracle) runs as part of the GPU suite."""
import pytest

pytestmark = pytest.mark.gpu


def test_graft_entry_smoke():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import __graft_entry__
    __graft_entry__.smoke()
