"""Many joins in one persistent tensor-core launch (csrc/hj_batch.cu, bound
here with ctypes).

    jobs = [(a0, None, eps0), (a1, b1, eps1), ...]     # CUDA tensors, one dtype
    counts = batch_count(jobs, form="fp16")           # one count per job

    with Batch(jobs) as b:                            # plan once ...
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        with torch.cuda.graph(g, stream=s):
            b.run(stream=s)                            # ... capture a run ...
        g.replay()
        counts = b.counts()                            # ... and read its counts

Jobs may differ in n, d (<= 256) and eps; a job's count equals its own
self_join_count / join_count. The input tensors are read only while the batch
is planned.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple

from . import Stats, _check, _opts, lib


class BatchJob(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("na", ctypes.c_uint64), ("nb", ctypes.c_uint64),
                ("d", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("eps", ctypes.c_double)]


def _bind():
    L = lib()
    if getattr(L, "_hj_batch_bound", False):
        return L
    P, U32, I = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
    sigs = {
        "hj_batch_create": (I, [ctypes.POINTER(BatchJob), U32, I, P, ctypes.POINTER(P)]),
        "hj_batch_run": (I, [P, P]),
        "hj_batch_counts": (I, [P, P, ctypes.POINTER(Stats)]),
        "hj_batch_destroy": (I, [P]),
        "hj_batch_count_device": (I, [ctypes.POINTER(BatchJob), U32, I, P, P, ctypes.POINTER(Stats)]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    L._hj_batch_bound = True
    return L


def _jobs(jobs: Sequence[Tuple]) -> Tuple[ctypes.Array, int, list]:
    import torch
    keep = []
    arr = (BatchJob * len(jobs))()
    dtype = None
    for i, job in enumerate(jobs):
        a, b, eps = job
        if not (torch.is_tensor(a) and a.is_cuda and a.dim() == 2):
            raise ValueError("batch inputs are 2-D CUDA tensors")
        a = a.contiguous()
        keep.append(a)
        dtype = dtype or a.dtype
        if a.dtype != dtype or a.dtype not in (torch.float32, torch.float64):
            raise ValueError("all batch inputs share one dtype, float32 or float64")
        arr[i].a = a.data_ptr()
        arr[i].na = a.shape[0]
        arr[i].d = a.shape[1]
        arr[i].eps = float(eps)
        if b is not None:
            b = b.contiguous()
            if b.dtype != dtype or b.shape[1] != a.shape[1]:
                raise ValueError("a and b of a job share dtype and dimension")
            keep.append(b)
            arr[i].b = b.data_ptr()
            arr[i].nb = b.shape[0]
    return arr, (8 if dtype == torch.float64 else 4), keep


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return None
    return stream if isinstance(stream, int) else stream.cuda_stream


def _plan_stream(stream) -> int:
    """Planning runs on the given stream, else on torch's current stream, so
    that it is ordered after whatever produced the input tensors."""
    if stream is not None:
        return _stream_handle(stream)
    import torch
    return torch.cuda.current_stream().cuda_stream


class Batch:
    """A planned batch: one persistent tensor-core launch per run."""

    def __init__(self, jobs: Sequence[Tuple], form="fp16", active_dims=None, ref_compat=False, device=None,
                 stream=None):
        L = _bind()
        arr, dtype_bytes, keep = _jobs(jobs)
        self.n_jobs = len(jobs)
        o = _opts(form, active_dims, ref_compat, device, _plan_stream(stream))
        h = ctypes.c_void_p()
        _check(L.hj_batch_create(arr, self.n_jobs, dtype_bytes, ctypes.byref(o), ctypes.byref(h)))
        self._h, self._L = h, L
        del keep  # the batch holds its own copies

    def run(self, stream=None) -> None:
        """Enqueues one run (no host synchronisation; capturable)."""
        _check(self._L.hj_batch_run(self._h, _stream_handle(stream)))

    def counts(self, return_stats=False):
        import numpy as np
        out = np.zeros(self.n_jobs, dtype=np.uint64)
        st = Stats()
        _check(self._L.hj_batch_counts(self._h, out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st)))
        res = [int(c) for c in out]
        return (res, st.to_dict()) if return_stats else res

    def close(self) -> None:
        if self._h:
            self._L.hj_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_count(jobs: Sequence[Tuple], form="fp16", active_dims=None, ref_compat=False, device=None,
                return_stats=False):
    """One count per job of `jobs` = [(a, b_or_None, eps), ...] (CUDA tensors),
    all in one persistent tensor-core launch."""
    L = _bind()
    arr, dtype_bytes, keep = _jobs(jobs)
    import numpy as np
    out = np.zeros(len(jobs), dtype=np.uint64)
    st = Stats()
    o = _opts(form, active_dims, ref_compat, device, _plan_stream(None))
    _check(L.hj_batch_count_device(arr, len(jobs), dtype_bytes, ctypes.byref(o), out.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.byref(st)))
    res = [int(c) for c in out]
    return (res, st.to_dict()) if return_stats else res
