"""CPU oracle for the epsilon-join count path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s ``cpu_baseline``
leg may import this package. It is the checker the GPU engine is compared
against, never the thing measured or shipped: the engine package
``hilbertjoin_b200`` does not import it and has no CPU fallback.

Two oracles live here:

* ``libhjoracle.so`` (``hj_oracle.c``): a plain-C restatement of the
  reference's count path (EGO order, stripes, the FP64 pair test), plus a
  brute-force count. Parity is pinned against the reference itself through the
  fixtures in ``tests/golden/``.
* ``_ref/hj_ref_k*_t*``: the hilbertJoin reference built from its own sources by
  ``build_ref.sh`` (present when the reference sources were available at build
  time), driven through its library entry points ``test_ego_loop3_macro`` and
  ``test_ego_loop3_noself``.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhjoracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build() -> None:
    """Compile the C oracle, and the reference into _ref/ (build_ref.sh skips
    that step when the reference sources are not on this machine)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    subprocess.run([os.path.join(HERE, "build_ref.sh")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        D, U64, U32, I = ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int
        P = ctypes.c_void_p
        L.hjo_dist2.restype = D
        L.hjo_dist2.argtypes = [P, P, U32]
        L.hjo_eps_wide.restype = D
        L.hjo_eps_wide.argtypes = [D, D]
        L.hjo_self_count_brute.restype = U64
        L.hjo_self_count_brute.argtypes = [P, U64, U32, D, I]
        L.hjo_join_count_brute.restype = U64
        L.hjo_join_count_brute.argtypes = [P, U64, P, U64, U32, D, I]
        L.hjo_self_row_counts.restype = None
        L.hjo_self_row_counts.argtypes = [P, U64, U32, D, P, U64, P, I]
        L.hjo_self_pairs_brute.restype = U64
        L.hjo_self_pairs_brute.argtypes = [P, U64, U32, D, P, U64, I]
        L.hjo_join_pairs_brute.restype = U64
        L.hjo_join_pairs_brute.argtypes = [P, U64, P, U64, U32, D, P, U64, I]
        L.hjo_dim_costs.restype = None
        L.hjo_dim_costs.argtypes = [P, U64, U32, D, P]
        L.hjo_cells.restype = None
        L.hjo_cells.argtypes = [P, U64, U32, D, P]
        L.hjo_ego_order.restype = None
        L.hjo_ego_order.argtypes = [P, U64, U32, D, P]
        L.hjo_self_count_ego.restype = U64
        L.hjo_self_count_ego.argtypes = [P, U64, U32, D, I, I, I, P]
        L.hjo_join_count_ego.restype = U64
        L.hjo_join_count_ego.argtypes = [P, U64, P, U64, U32, D, I, I, I, P]
        _lib = L
    return _lib


def _f64(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def dist2(a, b) -> float:
    a, b = _f64(a), _f64(b)
    return lib().hjo_dist2(_ptr(a), _ptr(b), a.shape[-1])


def self_count_brute(x, eps: float, threads: int = 0) -> int:
    x = _f64(x)
    return int(lib().hjo_self_count_brute(_ptr(x), x.shape[0], x.shape[1], eps, threads))


def join_count_brute(a, b, eps: float, threads: int = 0) -> int:
    a, b = _f64(a), _f64(b)
    return int(lib().hjo_join_count_brute(_ptr(a), a.shape[0], _ptr(b), b.shape[0], a.shape[1], eps, threads))


def self_row_counts(x, eps: float, rows, threads: int = 0) -> np.ndarray:
    x = _f64(x)
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.uint64))
    out = np.zeros(rows.shape[0], dtype=np.uint64)
    lib().hjo_self_row_counts(_ptr(x), x.shape[0], x.shape[1], eps, _ptr(rows), rows.shape[0], _ptr(out), threads)
    return out


def _pairs(call, cap_hint: int) -> np.ndarray:
    cap = max(int(cap_hint), 1)
    for _ in range(2):
        out = np.empty((cap, 2), dtype=np.uint64)
        total = int(call(out, cap))
        if total <= cap:
            return out[:total]
        cap = total
    raise RuntimeError("pair list changed size between passes")


def self_pairs_brute(x, eps: float, threads: int = 0, cap_hint: int = 1 << 16) -> np.ndarray:
    """(k, 2) uint64 pairs (i, j), i < j, with dist2 <= eps^2, sorted by (i, j)."""
    x = _f64(x)
    return _pairs(lambda out, cap: lib().hjo_self_pairs_brute(_ptr(x), x.shape[0], x.shape[1], eps, _ptr(out), cap,
                                                              threads), cap_hint)


def join_pairs_brute(a, b, eps: float, threads: int = 0, cap_hint: int = 1 << 16) -> np.ndarray:
    """(k, 2) uint64 ordered pairs (i in a, j in b), sorted by (i, j)."""
    a, b = _f64(a), _f64(b)
    return _pairs(lambda out, cap: lib().hjo_join_pairs_brute(_ptr(a), a.shape[0], _ptr(b), b.shape[0], a.shape[1],
                                                              eps, _ptr(out), cap, threads), cap_hint)


def dim_costs(x, eps: float) -> np.ndarray:
    """Per-dim Super-EGO cost on the deterministic sample (uint64, d)."""
    x = _f64(x)
    out = np.zeros(x.shape[1], dtype=np.uint64)
    lib().hjo_dim_costs(_ptr(x), x.shape[0], x.shape[1], eps, _ptr(out))
    return out


def dim_order(x, eps: float) -> np.ndarray:
    """reorder_dim: new key position of every dim, ascending cost, ties by index
    (the reference's convention, hilbertjoin/egojoin.cpp:587-589)."""
    c = dim_costs(x, eps)
    ranked = sorted(range(len(c)), key=lambda t: (int(c[t]), t))
    rd = np.zeros(len(c), dtype=np.int32)
    for pos, t in enumerate(ranked):
        rd[t] = pos
    return rd


def cells(x, eps: float) -> np.ndarray:
    x = _f64(x)
    out = np.empty_like(x)
    lib().hjo_cells(_ptr(x), x.shape[0], x.shape[1], eps, _ptr(out))
    return out


def ego_order(x, eps: float) -> np.ndarray:
    x = _f64(x)
    perm = np.empty(x.shape[0], dtype=np.uint64)
    lib().hjo_ego_order(_ptr(x), x.shape[0], x.shape[1], eps, _ptr(perm))
    return perm


def self_count_ego(x, eps: float, active_dims: int = 3, tail_drop: bool = False, threads: int = 0):
    """Returns (count, candidate pairs tested)."""
    x = _f64(x)
    cand = ctypes.c_uint64(0)
    c = lib().hjo_self_count_ego(_ptr(x), x.shape[0], x.shape[1], eps, active_dims, int(tail_drop), threads,
                                 ctypes.byref(cand))
    return int(c), int(cand.value)


def join_count_ego(a, b, eps: float, active_dims: int = 2, tail_drop: bool = False, threads: int = 0):
    a, b = _f64(a), _f64(b)
    cand = ctypes.c_uint64(0)
    c = lib().hjo_join_count_ego(_ptr(a), a.shape[0], _ptr(b), b.shape[0], a.shape[1], eps, active_dims,
                                 int(tail_drop), threads, ctypes.byref(cand))
    return int(c), int(cand.value)


# ----------------------------------------------------------- reference binary

def ref_binaries() -> dict:
    """{(kblock, num_threads): path} of the reference builds present."""
    out = {}
    if not os.path.isdir(REF_DIR):
        return out
    for name in os.listdir(REF_DIR):
        if name.startswith("hj_ref_k") and os.access(os.path.join(REF_DIR, name), os.X_OK):
            kb, nt = name[len("hj_ref_k"):].split("_t")
            out[(int(kb), int(nt))] = os.path.join(REF_DIR, name)
    return out


def host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return " avx512f" in f.read()
    except OSError:
        return False


def pick_ref_binary(kblock: int = 4, threads: int | None = None):
    """The reference build whose NUM_THREADS is the largest not above `threads`
    (default: this host's core count), or None when none exists or the host
    cannot run AVX-512 code."""
    if not host_has_avx512():
        return None
    bins = {nt: p for (kb, nt), p in ref_binaries().items() if kb == kblock}
    if not bins:
        return None
    want = threads or os.cpu_count() or 1
    ok = [nt for nt in bins if nt <= want]
    nt = max(ok) if ok else min(bins)
    return bins[nt]


def _write_bin(path: str, x: np.ndarray) -> None:
    _f64(x).tofile(path)


def ref_self_count(x, eps: float, stripes: int = 14, kblock: int = 4, threads: int | None = None) -> dict:
    """Runs the reference's test_ego_loop3_macro on x (copied, FP64)."""
    exe = pick_ref_binary(kblock, threads)
    if exe is None:
        raise RuntimeError("reference binary unavailable on this host")
    x = _f64(x)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.bin")
        _write_bin(p, x)
        r = subprocess.run([exe, "self", p, str(x.shape[0]), str(x.shape[1]), repr(float(eps)), str(stripes)],
                           check=True, capture_output=True, text=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def ref_join_count(a, b, eps: float, kblock: int = 4, threads: int | None = None) -> dict:
    """Runs the reference's test_ego_loop3_noself on (a, b) (copied, FP64)."""
    exe = pick_ref_binary(kblock, threads)
    if exe is None:
        raise RuntimeError("reference binary unavailable on this host")
    a, b = _f64(a), _f64(b)
    with tempfile.TemporaryDirectory() as td:
        pa, pb = os.path.join(td, "a.bin"), os.path.join(td, "b.bin")
        _write_bin(pa, a)
        _write_bin(pb, b)
        r = subprocess.run([exe, "join", pa, pb, str(a.shape[0]), str(b.shape[0]), str(a.shape[1]),
                            repr(float(eps))], check=True, capture_output=True, text=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def ref_ego_sorted(x, eps: float) -> np.ndarray:
    """The reference's epsilonGridOrdering applied to a copy of x."""
    exe = pick_ref_binary(4, None)
    if exe is None:
        raise RuntimeError("reference binary unavailable on this host")
    x = _f64(x)
    with tempfile.TemporaryDirectory() as td:
        p, q = os.path.join(td, "x.bin"), os.path.join(td, "s.bin")
        _write_bin(p, x)
        subprocess.run([exe, "egosort", p, str(x.shape[0]), str(x.shape[1]), repr(float(eps)), q],
                       check=True, capture_output=True, text=True)
        return np.fromfile(q, dtype=np.float64).reshape(x.shape)
