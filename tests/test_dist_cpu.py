"""Replica task distribution over ranks with the gloo backend (world size 2,
CPU): every (frequency, source) task is owned by exactly one rank, in the
order of the reference's distribute_tasks (src/em_fwd.cc:1273-1318)."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from emfem_b200.tasks import distribute_tasks


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, fidx, tidx, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = distribute_tasks(fidx, tidx, world, rank)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out.put(gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_tasks_partition_over_two_gloo_ranks():
    fidx = [0, 0, 1, 1, 2, 2, 0, 1, 2, 3, 3]
    tidx = [-3, -3, -3, 0, 0, 1, 1, 1, -3, 0, -3]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, fidx, tidx, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    allt = [t for g in gathered for t in g]
    expect = sorted(set(zip(fidx, tidx)))
    assert sorted(allt) == expect and len(allt) == len(expect)
    # CSEM block first, contiguous per group, larger share to the first group
    cs = [t for t in expect if t[1] >= 0]
    mt = [t for t in expect if t[1] < 0]
    assert gathered[0] == cs[:3] + mt[:2]
    assert gathered[1] == cs[3:] + mt[2:]


def test_single_group_owns_everything():
    fidx, tidx = [1, 0, 2], [-3, -3, 4]
    assert distribute_tasks(fidx, tidx, 1, 0) == [(2, 4), (0, -3), (1, -3)]
    with pytest.raises(ValueError):
        distribute_tasks(fidx, tidx, 2, 2)
