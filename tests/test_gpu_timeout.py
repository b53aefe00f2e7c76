"""The bounded device waits of the tensor-core kernel, made to run out.

hj_debug_set_wait_gate makes the kernel's epilogue wait on a device barrier
that nothing arrives on. The wait gives up after the gate's time, the kernel
raises its timeout error, the other roles stop, every copy and MMA already
issued is drained, the tensor memory is freed, and the call returns
HJ_ERR_TIMEOUT. Afterwards the same process runs the same join normally: the
context stays usable. No fault, trap or hang is involved."""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hj():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200 as hj
    L = hj.lib()
    L.hj_debug_set_wait_gate.restype = ctypes.c_int
    L.hj_debug_set_wait_gate.argtypes = [ctypes.c_uint64]
    return hj


@pytest.mark.parametrize("form", ["fp16", "tf32", "bf16x3"])
def test_wait_runs_out_then_the_next_call_succeeds(hj, form):
    from hilbertjoin_b200 import workloads as W
    x = W.uniform(6000, 32, 3, dtype=np.float32)
    eps = W.calibrate_eps(x, 6000, 16)
    want = oracle.self_count_brute(x.astype(np.float64), eps)
    L = hj.lib()
    assert L.hj_debug_set_wait_gate(50_000_000) == 0  # 50 ms
    try:
        with pytest.raises(hj.HJError) as e:
            hj.self_join_count(x, eps, form=form)
        assert e.value.status == 4  # HJ_ERR_TIMEOUT
    finally:
        assert L.hj_debug_set_wait_gate(0) == 0
    assert hj.self_join_count(x, eps, form=form) == want
    assert hj.self_join_count(x, eps, form="plain") == want


def test_gate_longer_than_the_wait_limit_is_rejected(hj):
    assert hj.lib().hj_debug_set_wait_gate(3_000_000_000) == 1
