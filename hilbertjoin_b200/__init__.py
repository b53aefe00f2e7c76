"""hilbertjoin_b200 -- a B200-native epsilon-similarity-join engine.

Counts the pairs of points in R^d within Euclidean distance eps, in one set
(self-join, unordered pairs) or between two sets (ordered pairs). The compute
path is the CUDA library ``lib/libhj.so`` (sm_100a kernels behind the C ABI of
``include/hj.h``); this module binds it with ctypes and mirrors the reference's
two library entry points, ``test_ego_loop3_macro`` and
``test_ego_loop3_noself`` (hilbertjoin/egojoin.h:56, :64), with numpy or torch
inputs. There is no CPU fallback: without the library every call raises.

    import hilbertjoin_b200 as hj
    count = hj.self_join_count(points, eps)                  # plain FP64 form
    count, stats = hj.self_join_count(points, eps, form="tf32", return_stats=True)
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libhj.so")

FORMS = {"plain": 0, "fp64": 0, "tf32": 1, "bf16x3": 2, "auto": 3, "fp16": 4}
FORM_NAMES = {0: "plain_fp64", 1: "tc_tf32", 2: "tc_bf16x3", 3: "auto", 4: "tc_fp16"}
# operand centring of the FP16 tensor-core form (hj_centring)
CENTRINGS = {"auto": 0, "global": 1, "block": 2}
CENTRING_NAMES = {0: "none", 1: "global", 2: "block"}

OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "CUDA error", 4: "device wait timed out",
          5: "band queue overflow", 6: "no usable device", 7: "unsupported input for this form",
          8: "rejected by admission", 9: "not found", 10: "output buffer too small"}
ERR_CAPACITY = 10


class HJError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Opts(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int32), ("active_dims", ctypes.c_int32), ("ref_compat", ctypes.c_int32),
                ("device", ctypes.c_int32), ("stream", ctypes.c_void_p), ("shard_index", ctypes.c_int32),
                ("shard_count", ctypes.c_int32), ("reorder_dims", ctypes.c_int32), ("item_chunk", ctypes.c_int32),
                ("tc_centring", ctypes.c_int32), ("reserved_i", ctypes.c_int32), ("reserved", ctypes.c_uint64 * 1)]


class Stats(ctypes.Structure):
    _fields_ = [("h2d_ms", ctypes.c_double), ("sort_ms", ctypes.c_double), ("index_ms", ctypes.c_double),
                ("join_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double),
                ("recheck_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("loadpercent", ctypes.c_double), ("candidate_pairs", ctypes.c_uint64),
                ("tile_pairs", ctypes.c_uint64), ("work_items", ctypes.c_uint64), ("band_pairs", ctypes.c_uint64),
                ("band_fraction", ctypes.c_double), ("band_halfwidth_rel", ctypes.c_double),
                ("max_abs_err_band", ctypes.c_double), ("fp64_items", ctypes.c_uint64),
                ("form_used", ctypes.c_int32), ("stripes", ctypes.c_int32), ("kernel_launches", ctypes.c_int32),
                ("tc_centring", ctypes.c_int32), ("reorder_ms", ctypes.c_double), ("reserved", ctypes.c_uint64 * 3)]

    def to_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_ if not f.startswith("reserved")}
        d["form_used"] = FORM_NAMES.get(d["form_used"], d["form_used"])
        d["tc_centring"] = CENTRING_NAMES.get(d["tc_centring"], d["tc_centring"])
        return d


class ServerOpts(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_uint64), ("max_inflight", ctypes.c_int32),
                ("device", ctypes.c_int32), ("form", ctypes.c_int32), ("batch_max", ctypes.c_int32),
                ("block_centring", ctypes.c_int32), ("reserved_i", ctypes.c_int32), ("reserved", ctypes.c_uint64 * 3)]


class Result(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("status", ctypes.c_int32), ("form_used", ctypes.c_int32),
                ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("candidate_pairs", ctypes.c_uint64), ("band_pairs", ctypes.c_uint64)]


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded engine library. Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"hilbertjoin_b200: {LIB_PATH} not built (run python -m hilbertjoin_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    P, U64, U32, I, D = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_double
    pO, pS, pU64 = ctypes.POINTER(Opts), ctypes.POINTER(Stats), ctypes.POINTER(ctypes.c_uint64)
    sigs = {
        "hj_opts_init": (None, [pO]),
        "hj_status_str": (ctypes.c_char_p, [I]),
        "hj_last_error": (ctypes.c_char_p, []),
        "hj_version": (ctypes.c_char_p, []),
        "hj_self_join_count": (I, [P, U64, U32, D, pO, pU64, pS]),
        "hj_self_join_count_f32": (I, [P, U64, U32, D, pO, pU64, pS]),
        "hj_join_count": (I, [P, U64, P, U64, U32, D, pO, pU64, pS]),
        "hj_join_count_f32": (I, [P, U64, P, U64, U32, D, pO, pU64, pS]),
        "hj_self_join_pairs": (I, [P, U64, U32, D, pO, P, U64, pU64, pS]),
        "hj_self_join_pairs_f32": (I, [P, U64, U32, D, pO, P, U64, pU64, pS]),
        "hj_join_pairs": (I, [P, U64, P, U64, U32, D, pO, P, U64, pU64, pS]),
        "hj_join_pairs_f32": (I, [P, U64, P, U64, U32, D, pO, P, U64, pU64, pS]),
        "hj_dim_order": (I, [P, U64, U32, D, pO, P, P]),
        "hj_self_join_count_device": (I, [P, I, U64, U32, D, pO, pU64, pS]),
        "hj_join_count_device": (I, [P, U64, P, U64, I, U32, D, pO, pU64, pS]),
        "hj_debug_tc_estimates": (I, [P, U64, P, U64, U32, I, P]),
        "hj_debug_tc_estimates_ex": (I, [P, U64, P, U64, U32, I, I, D, P, pS]),
        "hj_ego_sort": (I, [P, U64, U32, D, pO, P, P]),
        "hj_device_sm_count": (I, [I]),
        "hj_test_ego_loop3_macro": (None, [ctypes.c_size_t, ctypes.c_size_t, D, P, ctypes.POINTER(ctypes.c_size_t),
                                           I, ctypes.POINTER(D), ctypes.POINTER(D), ctypes.POINTER(D)]),
        "hj_test_ego_loop3_noself": (None, [ctypes.c_size_t, ctypes.c_size_t, I, D, P, P,
                                            ctypes.POINTER(ctypes.c_size_t), I, ctypes.POINTER(D),
                                            ctypes.POINTER(D), ctypes.POINTER(D)]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def version() -> str:
    return lib().hj_version().decode()


def _check(status: int) -> None:
    if status != OK:
        raise HJError(status, lib().hj_last_error().decode())


def _opts(form, active_dims, ref_compat, device, stream, shard=None, reorder_dims=False, item_chunk=None,
          centring="auto") -> Opts:
    o = Opts()
    lib().hj_opts_init(ctypes.byref(o))
    if isinstance(form, str) and form not in FORMS:
        raise ValueError(f"unknown form {form!r}: one of {sorted(FORMS)}")
    if isinstance(centring, str) and centring not in CENTRINGS:
        raise ValueError(f"unknown centring {centring!r}: one of {sorted(CENTRINGS)}")
    o.form = FORMS[form] if isinstance(form, str) else int(form)
    o.active_dims = -1 if active_dims is None else int(active_dims)
    o.ref_compat = int(bool(ref_compat))
    o.device = -1 if device is None else int(device)
    o.stream = stream
    if shard is not None:
        o.shard_index, o.shard_count = int(shard[0]), int(shard[1])
    o.reorder_dims = int(bool(reorder_dims))
    o.item_chunk = int(item_chunk or 0)
    o.tc_centring = CENTRINGS[centring] if isinstance(centring, str) else int(centring)
    return o


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _host_array(x):
    a = np.asarray(x)
    if a.dtype not in (np.float32, np.float64):
        a = a.astype(np.float64)
    a = np.ascontiguousarray(a)
    if a.ndim != 2:
        raise ValueError("points must be a 2-D array (n, d)")
    return a


def _torch_stream(x, stream):
    if stream is not None:
        return stream
    import torch
    return torch.cuda.current_stream(x.device).cuda_stream


def self_join_count(points, eps: float, form="plain", active_dims=None, ref_compat=False, device=None,
                    stream=None, return_stats=False, shard=None, reorder_dims=False, item_chunk=None, centring="auto"):
    """Number of unordered pairs {a, b}, a != b, of `points` with |a-b| <= eps.

    `points`: (n, d) float32/float64 numpy array (copied to the device inside
    the call) or CUDA torch tensor (used in place, on the tensor's stream)."""
    o = Stats()
    c = ctypes.c_uint64(0)
    if _is_torch_cuda(points):
        if points.dim() != 2 or points.dtype not in (__import__("torch").float32, __import__("torch").float64):
            raise ValueError("points must be a 2-D float32/float64 tensor")
        x = points.contiguous()
        opts = _opts(form, active_dims, ref_compat, x.device.index if device is None else device,
                     _torch_stream(x, stream), shard, reorder_dims, item_chunk, centring)
        _check(lib().hj_self_join_count_device(ctypes.c_void_p(x.data_ptr()), x.element_size(), x.shape[0],
                                               x.shape[1], float(eps), ctypes.byref(opts), ctypes.byref(c),
                                               ctypes.byref(o)))
    else:
        x = _host_array(points)
        opts = _opts(form, active_dims, ref_compat, device, stream, shard, reorder_dims, item_chunk, centring)
        fn = lib().hj_self_join_count if x.dtype == np.float64 else lib().hj_self_join_count_f32
        _check(fn(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], float(eps), ctypes.byref(opts),
                  ctypes.byref(c), ctypes.byref(o)))
    return (int(c.value), o.to_dict()) if return_stats else int(c.value)


def join_count(a, b, eps: float, form="plain", active_dims=None, ref_compat=False, device=None, stream=None,
               return_stats=False, shard=None, reorder_dims=False, item_chunk=None, centring="auto"):
    """Number of ordered pairs (p in a, q in b) with |p-q| <= eps."""
    o = Stats()
    c = ctypes.c_uint64(0)
    if _is_torch_cuda(a) != _is_torch_cuda(b):
        raise ValueError("a and b must both be CUDA tensors or both host arrays")
    if _is_torch_cuda(a):
        import torch
        xa, xb = a.contiguous(), b.contiguous()
        if xa.dim() != 2 or xb.dim() != 2 or xa.dtype not in (torch.float32, torch.float64):
            raise ValueError("a and b must be 2-D float32/float64 tensors")
        if xa.dtype != xb.dtype or xa.shape[1] != xb.shape[1]:
            raise ValueError("a and b must have the same dtype and dimension")
        opts = _opts(form, active_dims, ref_compat, xa.device.index if device is None else device,
                     _torch_stream(xa, stream), shard, reorder_dims, item_chunk, centring)
        _check(lib().hj_join_count_device(ctypes.c_void_p(xa.data_ptr()), xa.shape[0], ctypes.c_void_p(xb.data_ptr()),
                                          xb.shape[0], xa.element_size(), xa.shape[1], float(eps),
                                          ctypes.byref(opts), ctypes.byref(c), ctypes.byref(o)))
    else:
        xa, xb = _host_array(a), _host_array(b)
        if xa.dtype != xb.dtype:
            xb = xb.astype(xa.dtype)
        if xa.shape[1] != xb.shape[1]:
            raise ValueError("a and b must have the same dimension")
        opts = _opts(form, active_dims, ref_compat, device, stream, shard, reorder_dims, item_chunk, centring)
        fn = lib().hj_join_count if xa.dtype == np.float64 else lib().hj_join_count_f32
        _check(fn(xa.ctypes.data_as(ctypes.c_void_p), xa.shape[0], xb.ctypes.data_as(ctypes.c_void_p), xb.shape[0],
                  xa.shape[1], float(eps), ctypes.byref(opts), ctypes.byref(c), ctypes.byref(o)))
    return (int(c.value), o.to_dict()) if return_stats else int(c.value)


def _pairs(call, n_hint: int, capacity, return_stats: bool):
    """Runs a pair entry point, growing the output to the exact total when the
    first buffer is too small (the library writes nothing in that case)."""
    o = Stats()
    cnt = ctypes.c_uint64(0)
    cap = int(capacity) if capacity is not None else max(1 << 16, 4 * n_hint)
    for _ in range(2):
        out = np.empty((max(cap, 1), 2), dtype=np.uint64)
        st = call(out.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(cnt), ctypes.byref(o))
        if st == ERR_CAPACITY and capacity is None:
            cap = int(cnt.value)
            continue
        _check(st)
        res = out[:int(cnt.value)]
        return (res, o.to_dict()) if return_stats else res
    _check(st)


def self_join_pairs(points, eps: float, active_dims=None, ref_compat=False, device=None, capacity=None,
                    return_stats=False, shard=None, reorder_dims=False):
    """The unordered pairs {i, j}, i < j, of `points` (input indices) with
    |p_i - p_j| <= eps, as a (k, 2) uint64 array sorted by (i, j). Exactly the
    pairs self_join_count counts (plain FP64 form). `capacity`: the most pairs
    the caller accepts (HJError with status 10 beyond it); None = as many as
    there are."""
    x = _host_array(points)
    opts = _opts("plain", active_dims, ref_compat, device, None, shard, reorder_dims)
    fn = lib().hj_self_join_pairs if x.dtype == np.float64 else lib().hj_self_join_pairs_f32

    def call(buf, cap, cnt, st):
        return fn(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], float(eps), ctypes.byref(opts), buf,
                  cap, cnt, st)
    return _pairs(call, x.shape[0], capacity, return_stats)


def join_pairs(a, b, eps: float, active_dims=None, ref_compat=False, device=None, capacity=None,
               return_stats=False, shard=None, reorder_dims=False):
    """The ordered pairs (i in a, j in b) with |a_i - b_j| <= eps, (k, 2) uint64
    sorted by (i, j)."""
    xa, xb = _host_array(a), _host_array(b)
    if xa.dtype != xb.dtype:
        xb = xb.astype(xa.dtype)
    if xa.shape[1] != xb.shape[1]:
        raise ValueError("a and b must have the same dimension")
    opts = _opts("plain", active_dims, ref_compat, device, None, shard, reorder_dims)
    fn = lib().hj_join_pairs if xa.dtype == np.float64 else lib().hj_join_pairs_f32

    def call(buf, cap, cnt, st):
        return fn(xa.ctypes.data_as(ctypes.c_void_p), xa.shape[0], xb.ctypes.data_as(ctypes.c_void_p), xb.shape[0],
                  xa.shape[1], float(eps), ctypes.byref(opts), buf, cap, cnt, st)
    return _pairs(call, xa.shape[0], capacity, return_stats)


def dim_order(points, eps: float, device=None, return_costs=False):
    """reorder_dim (int32, d): the key position of every dim when the dims are
    ranked by ascending sampled cost (the reference's outputStatistics
    convention), and optionally the d costs (uint64)."""
    x = np.ascontiguousarray(np.asarray(points, dtype=np.float64))
    rd = np.zeros(x.shape[1], dtype=np.int32)
    costs = np.zeros(x.shape[1], dtype=np.uint64)
    opts = _opts("plain", None, False, device, None)
    _check(lib().hj_dim_order(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], float(eps),
                              ctypes.byref(opts), rd.ctypes.data_as(ctypes.c_void_p),
                              costs.ctypes.data_as(ctypes.c_void_p)))
    return (rd, costs) if return_costs else rd


def ego_sort(points, eps: float, device=None):
    """(perm, sorted_rows): the device epsilon-grid order of `points` (stable)."""
    x = np.ascontiguousarray(np.asarray(points, dtype=np.float64))
    perm = np.zeros(x.shape[0], dtype=np.uint64)
    srt = np.zeros_like(x)
    opts = _opts("plain", None, False, device, None)
    _check(lib().hj_ego_sort(x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1], float(eps),
                             ctypes.byref(opts), perm.ctypes.data_as(ctypes.c_void_p),
                             srt.ctypes.data_as(ctypes.c_void_p)))
    return perm, srt


def tc_estimates(a, b, form="tf32", centring=None, eps=None, return_stats=False):
    """Testing hook: the tensor-core dist^2 estimate of every pair (FP32 inputs).

    Without `centring` and `eps`: one global centre and an eps that puts every
    point in one cell (every pair estimated). With them: that operand centring
    ("global" / "block") and that eps; pairs outside the work list are NaN."""
    xa = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    xb = np.ascontiguousarray(np.asarray(b, dtype=np.float32))
    out = np.zeros((xa.shape[0], xb.shape[0]), dtype=np.float32)
    if centring is None and eps is None and not return_stats:
        _check(lib().hj_debug_tc_estimates(xa.ctypes.data_as(ctypes.c_void_p), xa.shape[0],
                                           xb.ctypes.data_as(ctypes.c_void_p), xb.shape[0], xa.shape[1],
                                           FORMS[form], out.ctypes.data_as(ctypes.c_void_p)))
        return out
    st = Stats()
    c = CENTRINGS[centring or "global"]
    _check(lib().hj_debug_tc_estimates_ex(xa.ctypes.data_as(ctypes.c_void_p), xa.shape[0],
                                          xb.ctypes.data_as(ctypes.c_void_p), xb.shape[0], xa.shape[1],
                                          FORMS[form], c, float(eps or 0.0), out.ctypes.data_as(ctypes.c_void_p),
                                          ctypes.byref(st)))
    return (out, st.to_dict()) if return_stats else out


def test_ego_loop3_macro(array, eps: float, stripes: int = 14):
    """Mirror of the reference's test_ego_loop3_macro (hilbertjoin/egojoin.cpp:777):
    returns (count, sortTime, indexTime, loadpercent). Unlike the reference the
    input is not modified."""
    x = np.ascontiguousarray(np.asarray(array, dtype=np.float64))
    cnt = ctypes.c_size_t(0)
    st, it, lp = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    lib().hj_test_ego_loop3_macro(x.shape[0], x.shape[1], float(eps), x.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.byref(cnt), int(stripes), ctypes.byref(st), ctypes.byref(it),
                                  ctypes.byref(lp))
    err = lib().hj_last_error().decode()
    if err:
        raise HJError(1, err)
    return int(cnt.value), st.value, it.value, lp.value


def test_ego_loop3_noself(a, b, eps: float, activedims: int = 2):
    """Mirror of the reference's test_ego_loop3_noself (hilbertjoin/egojoin.cpp:840)."""
    xa = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    xb = np.ascontiguousarray(np.asarray(b, dtype=np.float64))
    cnt = ctypes.c_size_t(0)
    st, it, lp = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    lib().hj_test_ego_loop3_noself(xa.shape[0], xb.shape[0], xa.shape[1], float(eps), xa.ctypes.data_as(ctypes.c_void_p),
                                   xb.ctypes.data_as(ctypes.c_void_p), ctypes.byref(cnt), int(activedims),
                                   ctypes.byref(st), ctypes.byref(it), ctypes.byref(lp))
    err = lib().hj_last_error().decode()
    if err:
        raise HJError(1, err)
    return int(cnt.value), st.value, it.value, lp.value


test_ego_loop3_macro.__test__ = False  # not pytest tests
test_ego_loop3_noself.__test__ = False
