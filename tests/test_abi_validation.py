"""Argument checks of the C ABI, called the way a C caller of the reference
would call it after switching (ctypes on lib/libhj.so, plain pointers and
sizes). Every check runs before a device is touched, so these run with or
without a GPU: each bad argument returns HJ_ERR_INVALID_ARG (or
HJ_ERR_UNSUPPORTED) and a message in hj_last_error(), never a crash, and a
later call replaces the message."""
import ctypes
import math

import numpy as np
import pytest

OK, INVALID, UNSUPPORTED = 0, 1, 7


@pytest.fixture(scope="module")
def L():
    import hilbertjoin_b200 as hj
    return hj.lib()


@pytest.fixture(scope="module")
def pts():
    return np.zeros((16, 4))


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def last(L):
    return L.hj_last_error().decode()


def self_count(L, pts, n, d, eps, count=True):
    c = ctypes.c_uint64(77)
    return L.hj_self_join_count(P(pts) if pts is not None else None, n, d, eps, None,
                                ctypes.byref(c) if count else None, None)


@pytest.mark.parametrize("d,msg", [(0, "d must be"), (1025, "d must be")])
def test_dimension_range(L, pts, d, msg):
    assert self_count(L, pts, 4, d, 0.1) == INVALID
    assert msg in last(L)


@pytest.mark.parametrize("eps", [0.0, -1.0, math.inf, math.nan])
def test_eps_must_be_positive_and_finite(L, pts, eps):
    assert self_count(L, pts, 16, 4, eps) == INVALID
    assert "eps" in last(L)


def test_size_limit_checked_before_reading(L, pts):
    # n above the limit is rejected before the (small) buffer is read
    assert self_count(L, pts, 1 << 31, 4, 0.1) == INVALID
    assert "2^31" in last(L)


def test_null_pointers(L, pts):
    assert self_count(L, pts, 16, 4, 0.1, count=False) == INVALID
    assert "null" in last(L)
    assert self_count(L, None, 16, 4, 0.1) == INVALID
    c = ctypes.c_uint64()
    assert L.hj_join_count(P(pts), 16, None, 5, 4, 0.1, None, ctypes.byref(c), None) == INVALID
    assert L.hj_join_count_f32(P(pts), 16, None, 5, 4, 0.1, None, ctypes.byref(c), None) == INVALID
    perm = np.zeros(16, np.uint64)
    assert L.hj_ego_sort(None, 16, 4, 0.1, None, P(perm), None) == INVALID
    assert L.hj_ego_sort(P(pts), 16, 4, 0.1, None, None, None) == INVALID
    assert L.hj_dim_order(P(pts), 16, 4, 0.1, None, None, None) == INVALID


def test_pair_output_arguments(L, pts):
    n_pairs = ctypes.c_uint64()
    # a capacity without a buffer
    assert L.hj_self_join_pairs(P(pts), 16, 4, 0.1, None, None, 10, ctypes.byref(n_pairs), None) == INVALID
    # no place for the total
    out = np.zeros(20, np.uint64)
    assert L.hj_self_join_pairs(P(pts), 16, 4, 0.1, None, P(out), 10, None, None) == INVALID
    # pair output runs the plain FP64 form, d <= 256
    wide = np.zeros((4, 300))
    assert L.hj_self_join_pairs(P(wide), 4, 300, 0.1, None, P(out), 10, ctypes.byref(n_pairs), None) == UNSUPPORTED
    assert "d <= 256" in last(L)


def test_device_entry_dtype(L, pts):
    c = ctypes.c_uint64()
    assert L.hj_self_join_count_device(P(pts), 2, 16, 4, 0.1, None, ctypes.byref(c), None) == INVALID
    assert "dtype_bytes" in last(L)
    assert L.hj_join_count_device(P(pts), 16, P(pts), 16, 16, 4, 0.1, None, ctypes.byref(c), None) == INVALID


def test_message_is_replaced(L, pts):
    assert self_count(L, pts, 16, 0, 0.1) == INVALID
    first = last(L)
    assert self_count(L, pts, 16, 4, -2.0) == INVALID
    second = last(L)
    assert first != second and "eps" in second and "d must be" not in second


def test_reference_signature_shims_check_too(L, pts):
    """The drop-ins with the reference's argument lists report a rejected call
    as *countresult = 0 (and zero times) with the message in hj_last_error()."""
    SZ, D, pD = ctypes.c_size_t, ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    f = L.hj_test_ego_loop3_macro
    f.restype, f.argtypes = None, [SZ, SZ, D, pD, ctypes.POINTER(SZ), ctypes.c_int, pD, pD, pD]
    x = np.ones((16, 4))
    cnt, t1, t2, lp = SZ(99), D(5.0), D(5.0), D(5.0)
    f(16, 4, -0.5, x.ctypes.data_as(pD), ctypes.byref(cnt), 2, ctypes.byref(t1), ctypes.byref(t2), ctypes.byref(lp))
    assert (cnt.value, t1.value, t2.value, lp.value) == (0, 0.0, 0.0, 0.0)
    assert "eps" in last(L)
    g = L.hj_test_ego_loop3_noself
    g.restype, g.argtypes = None, [SZ, SZ, ctypes.c_int, D, pD, pD, ctypes.POINTER(SZ), ctypes.c_int, pD, pD, pD]
    cnt = SZ(99)
    g(16, 16, 0, 0.5, x.ctypes.data_as(pD), x.ctypes.data_as(pD), ctypes.byref(cnt), 2, None, None, None)
    assert cnt.value == 0 and "d must be" in last(L)
