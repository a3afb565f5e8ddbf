"""A mesh split over several contexts: the partitioned explicit step (element
loop on every part, sum of the shared nodes' residual, nodal update) against
the single-context step, through the C ABI on one GPU.  The parts run one
after another from the host; no kernel waits on another."""
import numpy as np
import pytest

import alya_sma_b200 as sma
from alya_sma_b200 import partition as PT
from alya_sma_b200 import problem as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


@pytest.mark.parametrize("mesh,nparts", [("bar", 2), ("bar", 3), ("cantilever", 3)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("fp32", 1e-5)])
def test_partitioned_run_equals_single_context(mesh, nparts, precision, tol):
    """The bar (prescribed end displacement, transformation) and a coarse
    cantilever (tip traction as nodal loads, so each shared node's load
    must be applied once); 2 x 150 steps.  The parts' residual sums differ
    from the single context's only in summation order."""
    prob = P.bar_40x4x4(nsteps=400) if mesh == "bar" else P.cantilever_400x40x40(nsteps=600, div=10)
    one = sma.ExplicitSolid(prob, precision=precision)
    one.step(150)
    one.step(150)
    ps = PT.PartitionedSolid(prob, nparts=nparts, precision=precision)
    assert ps.nshared > 0
    np.testing.assert_allclose(ps.get("vmass"), one.get("vmass"), rtol=1e-13)
    ps.step(150)
    ps.step(150)
    for field in ("displ", "veloc"):
        ref, got = one.get(field), ps.get(field)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), field
    c = ps.counters()
    assert c["nr_active"] > 0 and c["nonfinite"] == 0 and c["neg_det"] == 0
    ps.close()
    one.close()


def test_partitioned_tw_with_rayleigh_damping():
    """Tchamwa-Wielgosz with Rayleigh alpha damping: the damped element
    kernel reads nodal velocities, which every part must hold identically
    at the shared nodes."""
    import dataclasses
    bar = dataclasses.replace(P.bar_40x4x4(nsteps=400), dampi=np.array([[2.0e5, 0.0]]))
    one = sma.ExplicitSolid(bar, precision="fp64", scheme="tw", phitw=1.033)
    one.step(200)
    ps = PT.PartitionedSolid(bar, nparts=3, precision="fp64", scheme="tw", phitw=1.033)
    ps.step(200)
    for field in ("displ", "veloc"):
        ref, got = one.get(field), ps.get(field)
        assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max(), field


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_worker(rank, world, port, out):
    import datetime
    import os

    import torch
    import torch.distributed as tdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world,
                             timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    bar = P.bar_40x4x4(nsteps=400)
    ps = PT.PartitionedSolid(bar, precision="fp64", group=tdist.group.WORLD)
    ps.step(150)
    ps.step(150)
    u, nodes = ps.get("displ")
    out[rank] = (nodes, u, ps.counters()["nonfinite"], ps.nshared)
    ps.close()
    tdist.barrier()
    tdist.destroy_process_group()


def test_partitioned_ranks_equal_single_context():
    """One part per rank (the distributed path: the shared rows summed by an
    all-reduce ordered on each part's stream), two ranks in two processes.
    gloo reduces CUDA tensors through host memory, so the ranks' kernels
    never wait on one another and both can share this one GPU; a run over
    several GPUs does the same with NCCL."""
    import torch.multiprocessing as mp
    world = 2
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.spawn(_rank_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    bar = P.bar_40x4x4(nsteps=400)
    one = sma.ExplicitSolid(bar, precision="fp64")
    one.step(150)
    one.step(150)
    ref = one.get("displ")
    covered = np.zeros(bar.npoin, bool)
    for r in range(world):
        nodes, u, nonfinite, nshared = res[r]
        assert nshared == 25 and nonfinite == 0
        assert np.abs(u - ref[nodes]).max() <= 1e-9 * np.abs(ref).max()
        covered[nodes] = True
    assert covered.all()


def test_single_part_is_the_plain_step():
    """One part: no shared node, the same kernels as sma_explicit_step in the
    same order (graphs aside), so the colour-scatter run is bitwise equal."""
    bar = P.bar_40x4x4(nsteps=400)
    one = sma.ExplicitSolid(bar, precision="fp64", scatter="color")
    one.step(37)
    ps = PT.PartitionedSolid(bar, nparts=1, precision="fp64", scatter="color")
    assert ps.nshared == 0
    ps.step(37)
    assert np.array_equal(ps.get("displ"), one.get("displ"))
    assert np.array_equal(ps.get("accel"), one.get("accel"))
