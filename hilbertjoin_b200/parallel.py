"""One epsilon-join sharded over several GPUs (one process per GPU).

Every rank holds the full point set(s), sorts and indexes them (cheap next to
the distance work), and counts only its shard of the block-pair work list: the
contiguous range of the Hilbert-ordered list whose cumulative tile-pair load
lies in [r L / W, (r+1) L / W) -- the reference's equal-load split of i-blocks
over threads (hilbertjoin/egojoin.h:214-222), over GPUs. The only collective
is one all-reduce of the 64-bit partial counts; there is no data-path exchange.

The process group is the caller's (NCCL on GPUs, gloo on CPU). Give it a short
timeout: a rank that fails before the all-reduce then makes the others raise
instead of waiting for ever.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple


def _reduce_sum(part: int, group=None) -> int:
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([int(part)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t.item())


def sharded_self_join_count(points, eps: float, form: str = "fp16", group=None,
                            count_fn: Optional[Callable[[Tuple[int, int]], int]] = None, **kw) -> int:
    """Self-join count of `points` over all ranks of `group`; every rank returns the total.

    `count_fn(shard)` computes one shard's count; by default the engine
    (hilbertjoin_b200.self_join_count with shard=(rank, world))."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if count_fn is None:
        import hilbertjoin_b200 as hj

        def count_fn(shard):
            return hj.self_join_count(points, eps, form=form, shard=shard, **kw)
    part = count_fn((rank, world))
    return _reduce_sum(part, group)


def sharded_join_count(a, b, eps: float, form: str = "fp16", group=None,
                       count_fn: Optional[Callable[[Tuple[int, int]], int]] = None, **kw) -> int:
    """Two-set join count (ordered pairs) over all ranks of `group`."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if count_fn is None:
        import hilbertjoin_b200 as hj

        def count_fn(shard):
            return hj.join_count(a, b, eps, form=form, shard=shard, **kw)
    part = count_fn((rank, world))
    return _reduce_sum(part, group)


def equal_load_cut(loads, shard: Tuple[int, int]) -> Tuple[int, int]:
    """[a, b) of the items that shard (k, K) takes from a work list with the
    given per-item loads: the first item whose exclusive load prefix reaches
    floor(L k / K) up to the first that reaches floor(L (k+1) / K), L the total
    load; the last shard runs to the end. This is the rule the device applies
    to the Hilbert-ordered list (shard_items in csrc/hj_index.cu), stated here
    so that orchestration can be tested without a GPU."""
    import bisect
    k, K = shard
    prefix, run = [], 0
    for w in loads:
        prefix.append(run)
        run += int(w)
    lo, hi = run * k // K, run * (k + 1) // K
    a = bisect.bisect_left(prefix, lo)
    b = len(prefix) if k + 1 == K else bisect.bisect_left(prefix, hi)
    return a, max(a, b)


def row_shard(n: int, shard: Tuple[int, int]) -> Tuple[int, int]:
    """[lo, hi) of an even split of n rows into shard[1] parts (used by tests and
    by callers that shard by rows instead of by work-list load)."""
    k, K = shard
    return n * k // K, n * (k + 1) // K
