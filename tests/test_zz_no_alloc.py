"""The allocation-free EGO sort entry point, called through the C ABI.

hj_ego_sort_device_noalloc serves callers that cannot call cudaMalloc during
their run (an application whose memory pool owns the device, a latency-critical
stream that must not pay cudaMalloc's implicit synchronisation): it keeps all
its temporaries in a fixed 32 MiB array inside the library. Its output must be
the permutation the allocating entry point hj_ego_sort returns (integers, so
exactly equal), on two calls in a row, since the calls share that array.
This file sorts last so that a failure here comes after every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hilbertjoin_b200 as hj
    L = hj.lib()
    f = L.hj_ego_sort_device_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_void_p]
    return torch, hj, f


CASES = [(40_000, 12, 0.12, np.float64, 1), (25_000, 7, 0.2, np.float32, 2), (30_000, 64, 0.3, np.float64, 3)]


@pytest.mark.parametrize("n,d,eps,dtype,seed", CASES)
def test_noalloc_matches_allocating_sort_twice(env, n, d, eps, dtype, seed):
    torch, hj, f = env
    x = np.random.default_rng(seed).random((n, d)).astype(dtype)
    want, _ = hj.ego_sort(x.astype(np.float64), eps)  # the allocating entry point
    xd = torch.from_numpy(x).cuda()
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(-1)
        torch.cuda.synchronize()
        rc = f(ctypes.c_void_p(xd.data_ptr()), x.itemsize, n, d, eps, ctypes.c_void_p(out.data_ptr()),
               ctypes.c_void_p(stream))
        torch.cuda.synchronize()
        assert rc == 0
        got = out.cpu().numpy().view(np.uint32).astype(np.uint64)
        assert np.array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_its_array(env):
    torch, hj, f = env
    xd = torch.zeros((4, 8), dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    # 50M points need far more than the fixed array: rejected before any kernel runs
    rc = f(ctypes.c_void_p(xd.data_ptr()), 8, 50_000_000, 8, 0.1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
