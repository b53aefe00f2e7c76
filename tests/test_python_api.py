"""The Python mirror of the C ABI, checked without a GPU: names of forms and
centring modes, shapes, dimension and dtype agreement, and that rejections
by the library arrive as HJError with the library's status and message.
Calls that pass every check reach the library, which answers
HJ_ERR_NO_DEVICE where no GPU is present."""
import numpy as np
import pytest

import hilbertjoin_b200 as hj


def _no_gpu():
    import torch
    return not torch.cuda.is_available()


def test_unknown_form_and_centring_names():
    x = np.zeros((8, 3))
    with pytest.raises(ValueError, match="unknown form 'int8'"):
        hj.self_join_count(x, 0.1, form="int8")
    with pytest.raises(ValueError, match="unknown centring 'local'"):
        hj.self_join_count(x, 0.1, form="fp16", centring="local")
    with pytest.raises(ValueError, match="unknown form"):
        hj.join_count(x, x, 0.1, form="fp8")


def test_shapes_and_dimensions():
    with pytest.raises(ValueError, match="2-D"):
        hj.self_join_count(np.zeros(10), 0.1)
    with pytest.raises(ValueError, match="same dimension"):
        hj.join_count(np.zeros((4, 3)), np.zeros((4, 5)), 0.1)
    with pytest.raises(ValueError, match="2-D"):
        hj.self_join_pairs(np.zeros((2, 2, 2)), 0.1)


def test_mixed_device_and_host_inputs():
    class FakeCuda:  # stands for a CUDA tensor without touching a device
        __module__ = "torch.fake"
        is_cuda = True

    with pytest.raises(ValueError, match="both be CUDA tensors or both host arrays"):
        hj.join_count(FakeCuda(), np.zeros((4, 3)), 0.1)
    with pytest.raises(ValueError, match="both be CUDA tensors or both host arrays"):
        hj.join_count(np.zeros((4, 3)), FakeCuda(), 0.1)


def test_library_rejection_carries_status_and_message():
    with pytest.raises(hj.HJError) as e:
        hj.self_join_count(np.zeros((8, 3)), 0.0)
    assert e.value.status == 1 and "eps" in str(e.value)
    with pytest.raises(hj.HJError) as e:
        hj.join_count(np.zeros((8, 1100)), np.zeros((8, 1100)), 0.5)
    assert e.value.status == 1 and "d must be" in str(e.value)


@pytest.mark.skipif(not _no_gpu(), reason="a device is present")
def test_valid_calls_reach_the_library():
    # integer and FP32 inputs are accepted (integers widened to FP64); the
    # library then reports that no device is present
    for x in (np.arange(24, dtype=np.int32).reshape(8, 3), np.zeros((8, 3), np.float32)):
        with pytest.raises(hj.HJError) as e:
            hj.self_join_count(x, 0.5, form="fp16", centring="block")
        assert e.value.status in (3, 6)
    with pytest.raises(hj.HJError) as e:
        hj.join_count(np.zeros((8, 3), np.float32), np.zeros((5, 3)), 0.5)  # b cast to a's dtype
    assert e.value.status in (3, 6)
