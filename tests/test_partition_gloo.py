"""The partitioned-mesh host path on CPU: the element partition and its
shared-node bookkeeping, nodal loads applied once, and the per-step sum of
shared residual rows over two gloo ranks (the reduction a partitioned run
does with NCCL between the element loop and the nodal update)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from alya_sma_b200 import partition as PT
from alya_sma_b200 import problem as P


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_partition_covers_and_shares_the_cut():
    bar = P.bar_40x4x4(nsteps=10)
    for nparts in (1, 2, 3, 5, 8):
        parts = PT.partition_elements(bar, nparts)
        allel = np.concatenate(parts)
        assert np.array_equal(np.sort(allel), np.arange(bar.nelem))          # disjoint cover
        assert max(p.size for p in parts) - min(p.size for p in parts) <= 1
        node_sets, shared, owner, local = PT.layout(bar, parts)
        if 40 % nparts == 0:      # whole 16-element slabs along x: each cut is one 5 x 5 node plane
            assert shared.size == 25 * (nparts - 1)
        else:                     # a cut inside a slab is a staircase of two planes at most
            assert 25 * (nparts - 1) < shared.size <= 2 * 25 * (nparts - 1)
        for k, g in enumerate(node_sets):
            loc, sl = local[k]
            assert np.array_equal(g[loc], shared[sl])
        assert np.all(owner >= 0)


def test_sub_problems_apply_each_nodal_load_once():
    canti = P.cantilever_400x40x40(nsteps=10, div=10)
    assert canti.fext is not None and np.abs(canti.fext).sum() > 0
    parts = PT.partition_elements(canti, 3)
    node_sets, shared, owner, local = PT.layout(canti, parts)
    total = np.zeros_like(canti.fext)
    for k, e in enumerate(parts):
        q, nodes = PT.sub_problem(canti, e, owner == k)
        assert np.array_equal(nodes, node_sets[k])
        assert q.nelem == e.size
        if q.fext is not None:
            total[nodes] += q.fext
    assert np.array_equal(total, canti.fext)


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as tdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world,
                             timeout=datetime.timedelta(seconds=60))
    bar = P.bar_40x4x4(nsteps=10)
    parts = PT.partition_elements(bar, world)
    node_sets, shared, owner, local = PT.layout(bar, parts)
    loc, sl = local[rank]
    gid = node_sets[rank][loc]
    rows = torch.as_tensor(np.stack([(rank + 1) * gid + c for c in range(3)], axis=1), dtype=torch.float64)
    summed = PT.reduce_shared(rows, torch.as_tensor(sl), shared.size).numpy()
    out[rank] = (gid, summed)
    tdist.barrier()
    tdist.destroy_process_group()


def test_shared_rows_summed_over_gloo_ranks():
    world = 3
    port = _free_port()
    with mp.get_context("spawn").Manager() as man:   # no fork of a threaded process
        out = man.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    bar = P.bar_40x4x4(nsteps=10)
    node_sets, _, _, _ = PT.layout(bar, PT.partition_elements(bar, world))
    for r in range(world):
        gid, summed = res[r]
        holders = [k for k in range(world) if np.isin(gid, node_sets[k]).any()]
        assert len(holders) >= 2
        # each shared node: the sum over the ranks holding it of (rank + 1) * id + c
        for i, g in enumerate(gid):
            who = [k for k in range(world) if g in set(node_sets[k].tolist())]
            expect = [sum((k + 1) * g + c for k in who) for c in range(3)]
            assert np.allclose(summed[i], expect)


def test_interface_elements_come_first():
    bar = P.bar_40x4x4(nsteps=10)
    parts = PT.partition_elements(bar, 3)
    _, shared, _, _ = PT.layout(bar, parts)
    mask = np.zeros(bar.npoin, bool)
    mask[shared] = True
    for e in parts:
        order, ni = PT.interface_first(bar, e, mask)
        assert np.array_equal(np.sort(order), e)                            # same elements
        touch = mask[bar.lnods[order]].any(axis=1)
        assert touch[:ni].all() and not touch[ni:].any() and ni > 0


def _mixed_parts(bar, world):
    """A partition with nodes held by up to four parts: the first element
    layer dealt round robin over the ranks, the rest in slabs."""
    first = np.arange(16)
    rest = PT.partition_elements(bar, world)
    parts = []
    for k in range(world):
        mine = np.concatenate([first[first % world == k], np.setdiff1d(rest[k], first)])
        parts.append(np.sort(mine))
    return parts


def _neighbour_worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as tdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world,
                             timeout=datetime.timedelta(seconds=60))
    bar = P.bar_40x4x4(nsteps=10)
    parts = _mixed_parts(bar, world)
    node_sets, shared, owner, local = PT.layout(bar, parts)
    plan = PT.neighbour_plan(node_sets, local)
    loc, sl = local[rank]
    gid = node_sets[rank][loc]
    rows = torch.as_tensor(np.stack([np.sin(gid * (rank + 2.0)) + c for c in range(3)], axis=1),
                           dtype=torch.float64)
    by_neighbours = PT.exchange_neighbours(rows, plan[rank]).numpy()
    by_allreduce = PT.reduce_shared(rows, torch.as_tensor(sl), shared.size).numpy()
    out[rank] = (by_neighbours, by_allreduce, len(plan[rank]))
    tdist.barrier()
    tdist.destroy_process_group()


def test_neighbour_exchange_equals_the_all_reduce():
    """The per-step sum of shared rows by point-to-point exchange with the
    neighbouring parts only (what a partitioned run does, overlapped with
    its interior elements) equals the all-reduce over every shared node,
    with nodes held by up to four parts."""
    world = 4
    port = _free_port()
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.spawn(_neighbour_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    bar = P.bar_40x4x4(nsteps=10)
    node_sets, shared, _, _ = PT.layout(bar, _mixed_parts(bar, world))
    cnt = np.zeros(bar.npoin, int)
    for g in node_sets:
        cnt[g] += 1
    assert cnt.max() >= 3                                   # some nodes held by three or more parts
    for r in range(world):
        nb, ar, nplan = res[r]
        assert nplan >= 1
        assert np.allclose(nb, ar, rtol=0, atol=1e-12)
