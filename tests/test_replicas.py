"""Replica sharding over ranks (world_size 2, gloo on CPU): balanced disjoint assignment and the
max/sum-over-ranks reductions used for multi-GPU timing."""
import os
import socket

import numpy as np
import pytest

from hamiltonfastmarching_b200.replicas import assign


def test_assign_is_a_balanced_partition():
    rng = np.random.default_rng(0)
    work = rng.uniform(1, 100, 57)
    parts = assign(work, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(57))
    loads = [work[p].sum() for p in parts]
    assert max(loads) - min(loads) <= work.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, queue):
    import torch.distributed as dist
    from hamiltonfastmarching_b200.replicas import assign, max_over_ranks, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    work = [float(3 + (7 * i) % 11) for i in range(20)]
    mine = assign(work, world)[rank]
    done = sum(work[i] for i in mine)            # stands for this rank's solve time
    t = max_over_ranks(done)
    total = sum_over_ranks(len(mine))
    dist.barrier()
    dist.destroy_process_group()
    queue.put((rank, mine, t, total))


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, n0), (r1, m1, t1, n1) = res
    assert set(m0).isdisjoint(m1) and sorted(m0 + m1) == list(range(20))
    work = [float(3 + (7 * i) % 11) for i in range(20)]
    assert t0 == t1 == max(sum(work[i] for i in m0), sum(work[i] for i in m1))
    assert n0 == n1 == 20
