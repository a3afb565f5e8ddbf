"""The pipelined element-loop boundary: on atomic-scatter meshes of 32k+
elements sma_assemble copies the displacement in, runs the element loop and
copies the residual out slab by slab on separate streams.  Its outputs must
equal the serial path's (the coloured scatter) to the rounding of the
summation order, with the mesh's own numbering and with a shuffled one that
leaves the slab plan no locality to use."""
import dataclasses

import numpy as np
import pytest

import alya_sma_b200 as sma
from alya_sma_b200 import problem as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


@pytest.fixture(scope="module")
def canti():
    return P.cantilever_400x40x40(nsteps=100, div=2)          # 80,000 elements: 4 slabs


def _field(p, seed):
    rng = np.random.default_rng(seed)
    return P.prestrain(p, 0.012) + rng.normal(size=(p.npoin, 3)) * 1e-4


def _shuffled(p, seed=3):
    """The same mesh with elements and nodes numbered in random order."""
    rng = np.random.default_rng(seed)
    pn = rng.permutation(p.npoin)                             # new id -> old id
    inv = np.empty_like(pn)
    inv[pn] = np.arange(p.npoin)
    pe = rng.permutation(p.nelem)
    q = dataclasses.replace(p, coord=p.coord[pn], lnods=inv[p.lnods[pe]].astype(np.int32),
                            fixno=p.fixno[pn], bcfun=p.bcfun[pn],
                            fext=None if p.fext is None else p.fext[pn])
    return q, pn, pe


def _compare(pa, ua, pb, ub, map_nodes=None, map_elems=None):
    a = sma.ExplicitSolid(pa, precision="fp64", scatter="atomic")
    b = sma.ExplicitSolid(pb, precision="fp64", scatter="color")
    for call in range(2):                                     # two loops in a row
        ra = a.assemble(ua[call], fext_scale=0.5)
        rb = b.assemble(ub[call], fext_scale=0.5)
        for k in ("rhsid", "finte", "fexte", "frxid"):
            x = ra[k] if map_nodes is None else ra[k][np.argsort(map_nodes)]
            scale = max(np.abs(rb[k]).max(), 1e-30)
            assert np.abs(x - rb[k]).max() <= 1e-11 * scale, (call, k)
        sa, sb = a.state, b.state
        if map_elems is not None:
            sa = sa[np.argsort(map_elems)]
        assert np.abs(sa - sb).max() <= 1e-12 * np.abs(sb).max(), call
        a.end_step()
        b.end_step()


@pytest.mark.parametrize("scatter", ["atomic", "color"])
def test_large_mesh_assemble_matches_oracle(oracle, canti, scatter):
    """80k elements with a traction load: every output against the oracle.
    (Context set-up stages coordinates and loads through one buffer; an
    upload that is not ordered behind the previous conversion kernel shows
    up here as coordinates read as loads.)"""
    u = _field(canti, 0)
    g = sma.ExplicitSolid(canti, precision="fp64", scatter=scatter)
    got = g.assemble(u, fext_scale=0.5)
    ref = oracle.Problem(canti).assemble(u, fext_scale=0.5)
    for k in ("rhsid", "finte", "fexte", "frxid"):
        scale = max(np.abs(ref[k]).max(), 1e-30)
        assert np.abs(got[k] - ref[k]).max() <= 1e-8 * scale, k


def test_pipelined_assemble_equals_serial(canti):
    u = [_field(canti, 0), _field(canti, 1)]
    _compare(canti, u, canti, u)


def test_pipelined_assemble_with_damping(canti):
    """Rayleigh alpha damping through the pipelined boundary (the one-tile
    damped kernel per slab, the velocity as set) equals the serial path."""
    p = dataclasses.replace(canti, dampi=np.array([[2.0e5, 0.0]]))
    u = _field(p, 0)
    v = np.random.default_rng(5).normal(size=(p.npoin, 3)) * 1e3
    out = []
    for scatter in ("atomic", "color"):
        g = sma.ExplicitSolid(p, precision="fp64", scatter=scatter)
        g.set("veloc", v)
        out.append(g.assemble(u, fext_scale=0.5))
    und = sma.ExplicitSolid(canti, precision="fp64").assemble(u, fext_scale=0.5)
    for k in ("rhsid", "finte", "frxid"):
        scale = max(np.abs(out[1][k]).max(), 1e-30)
        assert np.abs(out[0][k] - out[1][k]).max() <= 1e-11 * scale, k
    assert np.abs(out[0]["finte"] - und["finte"]).max() <= 1e-11 * np.abs(und["finte"]).max()
    assert np.abs(out[0]["rhsid"] - und["rhsid"]).max() > 1e-3 * np.abs(und["rhsid"]).max()


def test_registered_host_arrays(canti):
    """Page-locked caller arrays (sma_host_register) give the same residual as
    pageable ones, and unregister cleanly."""
    u = _field(canti, 0)
    ref = sma.ExplicitSolid(canti, precision="fp64").assemble(u, want_all=False)["rhsid"]
    d = sma.host_register(np.ascontiguousarray(u))
    r = sma.host_register(np.zeros((canti.npoin, 3)))
    g = sma.ExplicitSolid(canti, precision="fp64")
    try:
        got = g.assemble(d, want_all=False, rhsid=r)["rhsid"]
        assert got is r
        assert np.abs(r - ref).max() <= 1e-11 * np.abs(ref).max()
    finally:
        sma.host_unregister(d)
        sma.host_unregister(r)
    with pytest.raises(sma.SmaError):
        sma.host_unregister(d)                                   # not registered any more
    # that failed runtime call leaves no error behind for the next launch check
    g.end_step()
    again = g.assemble(u, want_all=False)["rhsid"]
    assert np.isfinite(again).all()


def test_pipelined_assemble_without_locality(canti):
    q, pn, pe = _shuffled(canti)
    u = [_field(canti, 0), _field(canti, 1)]
    _compare(q, [x[pn] for x in u], canti, u, map_nodes=pn, map_elems=pe)
