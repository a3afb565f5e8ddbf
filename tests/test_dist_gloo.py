"""The N>1 host path on CPU: two gloo ranks shard the ensemble by specimens
(a disjoint, load-balanced cover; each rank builds identical specimens to
the full ensemble's) and reduce timings as the max over ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from alya_sma_b200 import dist
from alya_sma_b200 import problem as P


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as tdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, w, lr = dist.env()
    sizes = P.ensemble_sizes(12, emin=100, emax=400)
    mine = dist.shard_specimens(sizes, r, w)
    part = P.ensemble(nspec=12, nsteps=10, emin=100, emax=400, subset=mine)
    t_max = dist.max_over_ranks(1.0 + r)
    n_all = dist.sum_over_ranks(part.nelem)
    out[r] = (mine, float(part.props[0, 0]), t_max, n_all, w, lr)
    tdist.barrier()
    tdist.destroy_process_group()


def test_two_gloo_ranks_shard_ensemble_and_reduce():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as man:   # no fork of a threaded process
        out = man.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    ids0, ids1 = res[0][0], res[1][0]
    assert sorted(ids0 + ids1) == list(range(12)) and not set(ids0) & set(ids1)
    sizes = P.ensemble_sizes(12, emin=100, emax=400)
    loads = [int(np.sum(sizes[ids])) for ids in (ids0, ids1)]
    assert max(loads) - min(loads) <= int(sizes.max())           # LPT balance
    full = P.ensemble(nspec=12, nsteps=10, emin=100, emax=400)
    assert res[0][1] == full.props[ids0[0], 0]                    # same specimen as in the full ensemble
    assert res[0][2] == res[1][2] == 2.0                          # max over ranks
    assert res[0][3] == res[1][3] == full.nelem                    # every element counted once
    assert res[0][4] == 2 and {res[0][5], res[1][5]} == {0, 1}


def test_shard_is_a_cover_for_any_world():
    sizes = P.ensemble_sizes(256)
    for world in (1, 2, 3, 8):
        got = sorted(s for r in range(world) for s in dist.shard_specimens(sizes, r, world))
        assert got == list(range(256))
