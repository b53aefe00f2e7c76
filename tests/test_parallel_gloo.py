"""Multi-rank host logic of a sharded join on CPU: world size 2, gloo.

Each rank takes its shard of a work list by the engine's equal-load rule
(``parallel.equal_load_cut``, the host statement of the device's shard_items)
and counts it on the CPU; the items are the rows of the set in order, with
load n-1-i (the partners j > i of row i). The test exercises the orchestration
(process group, shard assignment, the all-reduce, failure of a rank) without a
GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    import oracle
    from hilbertjoin_b200.parallel import equal_load_cut, sharded_self_join_count
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    x = np.random.default_rng(3).random((1500, 6))
    eps = 0.3

    n = x.shape[0]

    def part(shard):
        lo, hi = equal_load_cut([n - 1 - i for i in range(n)], shard)
        if mode == "fail" and shard[0] == 1:
            raise RuntimeError("injected failure on rank 1")
        rows = np.arange(lo, hi, dtype=np.uint64)
        # pairs (i, j) with i in the shard and j > i
        c = 0
        for i in rows:
            i = int(i)
            if i + 1 < x.shape[0]:
                d2 = ((x[i + 1:] - x[i]) ** 2).sum(1)
                c += int((d2 <= eps * eps).sum())
        return c

    try:
        total = sharded_self_join_count(x, eps, group=None, count_fn=part)
        q.put((rank, "ok", total, oracle.self_count_brute(x, eps)))
    except Exception as e:  # noqa: BLE001
        q.put((rank, "error", repr(e)[:200], None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_sharded_count_sums_to_total():
    out = _run("ok")
    for rank, status, total, want in out:
        assert status == "ok", out
        assert total == want


def test_failed_rank_ends_in_error_not_hang():
    out = _run("fail")
    by = {r: (s, v) for r, s, v, _ in out}
    assert by[1][0] == "error" and "injected" in by[1][1]
    assert by[0][0] == "error"  # its all-reduce gives up instead of waiting for ever


def test_equal_load_cut_partitions_and_balances():
    from hilbertjoin_b200.parallel import equal_load_cut
    rng = np.random.default_rng(0)
    for n in (1, 7, 100, 1000):
        loads = rng.integers(0, 33, size=n)
        for K in (1, 2, 3, 8):
            cuts = [equal_load_cut(loads, (k, K)) for k in range(K)]
            assert cuts[0][0] == 0 and cuts[-1][1] == n
            for (a0, b0), (a1, b1) in zip(cuts, cuts[1:]):
                assert b0 == a1  # contiguous, disjoint, complete
            total = int(loads.sum())
            for a, b in cuts:  # each shard within one item of its equal share
                assert int(loads[a:b].sum()) <= total // K + 33
