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
                 stream=None, item_chunk=None, tuned=False):
        """tuned=True: form, item chunk and active dims from the autotuner's
        table for the batch's largest d (explicit arguments other than the
        defaults are then ignored)."""
        L = _bind()
        arr, dtype_bytes, keep = _jobs(jobs)
        if tuned:
            form, item_chunk, active_dims = _tuned(arr)
        self.n_jobs = len(jobs)
        o = _opts(form, active_dims, ref_compat, device, _plan_stream(stream), item_chunk=item_chunk)
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


def _tuned(arr):
    from .autotune import config_for
    cfg = config_for(max(j.d for j in arr))
    return cfg["form"], cfg["item_chunk"], cfg["active_dims"]


def batch_count(jobs: Sequence[Tuple], form="fp16", active_dims=None, ref_compat=False, device=None,
                return_stats=False, item_chunk=None, tuned=False):
    """One count per job of `jobs` = [(a, b_or_None, eps), ...] (CUDA tensors),
    all in one persistent tensor-core launch."""
    L = _bind()
    arr, dtype_bytes, keep = _jobs(jobs)
    if tuned:
        form, item_chunk, active_dims = _tuned(arr)
    import numpy as np
    out = np.zeros(len(jobs), dtype=np.uint64)
    st = Stats()
    o = _opts(form, active_dims, ref_compat, device, _plan_stream(None), item_chunk=item_chunk)
    _check(L.hj_batch_count_device(arr, len(jobs), dtype_bytes, ctypes.byref(o), out.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.byref(st)))
    res = [int(c) for c in out]
    return (res, st.to_dict()) if return_stats else res


# ------------------------------------------------------------------ benchmark

DIMS = (8, 16, 32, 64, 128)


def make_jobs(n_jobs: int = 96, seed: int = 11, n_lo: int = 2000, n_hi: int = 100_000, self_frac: float = 0.7,
              dims=DIMS):
    """A batch of joins on resident device sets: n log-uniform in [n_lo, n_hi],
    d from `dims`, uniform or 16-component Gaussian mixture (FP32), two-set
    joins for 1 - self_frac of the jobs, eps for 8 to 64 neighbours."""
    import numpy as np
    import torch
    from . import workloads as W
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n_jobs):
        d = int(dims[i % len(dims)])
        na = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        gen = (lambda n, s: W.uniform(n, d, s, dtype=np.float32)) if rng.random() < 0.5 else \
            (lambda n, s: W.gmm(n, d, s, components=16, dtype=np.float32))
        a = gen(na, 5000 + i)
        nbr = float(np.exp(rng.uniform(np.log(8), np.log(64))))
        if rng.random() < self_frac:
            eps = W.calibrate_eps(a, na, nbr, sample=1500)
            jobs.append((torch.from_numpy(a).cuda(), None, eps))
        else:
            nb = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
            b = gen(nb, 9000 + i)
            eps = W.calibrate_eps_join(a, b, nb, nbr, sample=1500)
            jobs.append((torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), eps))
    return jobs


def run_benchmark(n_jobs: int = 96, form: str = "fp16", replays: int = 5, seed: int = 11) -> dict:
    """Jobs/s of the same joins run one call at a time, as one planned batch
    (planning + one launch), and as replays of a captured batch run."""
    import time
    import torch
    import hilbertjoin_b200 as hj
    jobs = make_jobs(n_jobs, seed=seed)
    torch.cuda.synchronize()

    def alone(j):
        a, b, eps = j
        return hj.self_join_count(a, eps, form=form) if b is None else hj.join_count(a, b, eps, form=form)

    for j in jobs[:4]:  # warm-up
        alone(j)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seq = [alone(j) for j in jobs]
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0

    batch_count(jobs[:4], form=form)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    got, st = batch_count(jobs, form=form, return_stats=True)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    if got != seq:
        raise RuntimeError("batched and single-call counts differ")

    with Batch(jobs, form=form) as b:
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            b.run(stream=s)
        g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(replays):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        t_rep = e0.elapsed_time(e1) / 1e3 / replays
        if b.counts() != seq:
            raise RuntimeError("replayed batch counts differ")
        del g
    cand = st["candidate_pairs"]
    return {"jobs": n_jobs, "form": form,
            "workload": f"{n_jobs} joins on resident sets, 70% self / 30% A x B, n log-U[2e3, 1e5], d in {DIMS}, "
                        "uniform or 16-GMM FP32, eps for 8-64 neighbours",
            "sequential_calls": {"s": t_seq, "jobs_per_s": n_jobs / t_seq},
            "batch_plan_and_run": {"s": t_batch, "jobs_per_s": n_jobs / t_batch},
            "batch_replay": {"s": t_rep, "jobs_per_s": n_jobs / t_rep, "candidate_pairs_per_s": cand / t_rep},
            "candidate_pairs": cand, "work_items": st["work_items"], "band_pairs": st["band_pairs"],
            "fp64_items": st["fp64_items"], "speedup_batch_vs_calls": t_seq / t_batch,
            "speedup_replay_vs_calls": t_seq / t_rep}
