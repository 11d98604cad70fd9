"""Host logic of the multi-process paths, on CPU with world_size 2 (gloo)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from kielflow_b200 import dist as kdist
from kielflow_b200.sweep import sweep_instances


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst = sweep_instances(seed=3)
        parts = kdist.partition([i.n for i in inst], world)
        gathered = [None] * world
        dist.all_gather_object(gathered, parts)
        mx = kdist.max_over_ranks(float(rank + 1) * 1.5)
        q.put((rank, parts, gathered, mx))
    finally:
        dist.destroy_process_group()


def test_partition_is_agreed_disjoint_and_balanced_across_two_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = res[0][1]
    for r in res:
        assert r[1] == parts and r[2] == [parts] * world  # every rank computed the same partition
        assert r[3] == 3.0                                 # max over ranks of (rank+1)*1.5
    allidx = sorted(i for p in parts for i in p)
    assert allidx == list(range(48))
    inst = sweep_instances(seed=3)
    loads = [sum(kdist.instance_cost(inst[i].n) for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.05


def test_sweep_parameters_in_their_ranges():
    inst = sweep_instances(seed=0)
    assert [i.n for i in inst].count(64) == 16 and [i.n for i in inst].count(128) == 16
    for i in inst:
        assert 0.3 <= i.M <= 1.5 and 0.01 <= i.tau <= 0.3 and -50 <= i.Q <= -5
    assert sweep_instances(seed=0)[5] == inst[5]
