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


def test_noalloc_takes_no_device_memory(env):
    """After a first call (which looks up the array's address and loads the
    kernels), further calls leave the device's free memory unchanged."""
    torch, hj, f = env
    n, d, eps = 30_000, 16, 0.15
    x = np.random.default_rng(11).random((n, d))
    xd = torch.from_numpy(x).cuda()
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = (ctypes.c_void_p(xd.data_ptr()), 8, n, d, eps, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert f(*args) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert f(*args) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_back_to_back_on_one_stream(env):
    """Two different inputs queued one after the other on one non-default
    stream, with no host synchronisation of ours in between: calls on one
    stream are ordered, so both outputs are right although they share the
    array."""
    torch, hj, f = env
    s = torch.cuda.Stream()
    n1, n2, d = 20_000, 27_000, 9
    x1 = np.random.default_rng(21).random((n1, d))
    x2 = np.random.default_rng(22).random((n2, d)) * 3.0
    want1, _ = hj.ego_sort(x1, 0.11)
    want2, _ = hj.ego_sort(x2, 0.29)
    with torch.cuda.stream(s):
        xd1, xd2 = torch.from_numpy(x1).cuda(), torch.from_numpy(x2).cuda()
        o1 = torch.full((n1,), -1, dtype=torch.int32, device="cuda")
        o2 = torch.full((n2,), -1, dtype=torch.int32, device="cuda")
    sp = ctypes.c_void_p(s.cuda_stream)
    assert f(ctypes.c_void_p(xd1.data_ptr()), 8, n1, d, 0.11, ctypes.c_void_p(o1.data_ptr()), sp) == 0
    assert f(ctypes.c_void_p(xd2.data_ptr()), 8, n2, d, 0.29, ctypes.c_void_p(o2.data_ptr()), sp) == 0
    s.synchronize()
    assert np.array_equal(o1.cpu().numpy().view(np.uint32).astype(np.uint64), want1)
    assert np.array_equal(o2.cpu().numpy().view(np.uint32).astype(np.uint64), want2)


def test_noalloc_failure_sets_message(env):
    torch, hj, f = env
    xd = torch.zeros((4, 8), dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = f(ctypes.c_void_p(xd.data_ptr()), 8, 50_000_000, 8, 0.1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"scratch" in hj.lib().hj_last_error()
