"""Step-level rows beyond the central-difference loop: the Tchamwa-Wielgosz
scheme, the energy balance of sld_energy, reaction histories and
checkpoint/resume -- all through the C ABI, checked against the oracle."""
import ctypes as C
import os

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
def bar():
    return P.bar_40x4x4(nsteps=400)


@pytest.fixture(scope="module")
def canti():
    return P.cantilever_400x40x40(nsteps=600, div=10)


def test_tw_scheme_matches_oracle(oracle, bar):
    """Tchamwa-Wielgosz (phi = 1.033, the scheme of every shipped SMA deck)."""
    nsteps = 300
    mid = int(np.argmin(np.sum((bar.coord - [20, 2, 2]) ** 2, axis=1)))
    wit = [3 * mid, 3 * mid + 1]
    o = oracle.Problem(bar)
    h_ref = o.run(bar.dtime, nsteps, wit_dof=wit, scheme="tw", phi=1.033)
    g = sma.ExplicitSolid(bar, precision="fp64", scheme="tw", phitw=1.033)
    g.set_witness(wit, nsteps)
    g.step(nsteps)
    h = g.witness()
    assert np.abs(h - h_ref).max() / np.abs(h_ref).max() < 1e-6
    assert np.abs(g.get("displ") - o.displ).max() / np.abs(o.displ).max() < 1e-6
    v, a = g.get("veloc"), g.get("accel")
    assert np.abs(v - o.veloc).max() / np.abs(o.veloc).max() < 1e-5
    fixed = bar.fixno == 1
    assert np.all(v[fixed] == 0.0) and np.all(a[fixed] == 0.0)   # prescribed dofs at rest
    assert o.sdv[:, 1, :, 0].max() > 0.05


@pytest.mark.parametrize("scheme", ["cd", "tw"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_rayleigh_alpha_damping_matches_oracle(oracle, bar, scheme, precision):
    """RAYLEIGH_DAMPING RAYALPHA (sld_elmmat.f90:159-164): the element loop
    subtracts alpha rho N v(g) dV with the velocity the reference's loop reads
    (v_n in central differences, the predicted velocity in TW)."""
    import dataclasses
    p = dataclasses.replace(bar, dampi=np.array([[2.0e5, 0.0]]))
    nsteps = 300
    mid = int(np.argmin(np.sum((p.coord - [20, 2, 2]) ** 2, axis=1)))
    wit = [3 * mid, 3 * mid + 1]
    o = oracle.Problem(p)
    h_ref = o.run(p.dtime, nsteps, wit_dof=wit, scheme=scheme, phi=1.033)
    g = sma.ExplicitSolid(p, precision=precision, scheme=scheme, phitw=1.033)
    g.set_witness(wit, nsteps)
    g.step(nsteps)
    h = g.witness()
    tol = 1e-6 if precision == "fp64" else 5e-4
    assert np.abs(h - h_ref).max() / np.abs(h_ref).max() < tol
    assert np.abs(g.get("veloc") - o.veloc).max() / np.abs(o.veloc).max() < 10 * tol
    # the damping acts: the undamped run keeps more kinetic energy
    u = oracle.Problem(bar)
    u.run(bar.dtime, nsteps, scheme=scheme, phi=1.033)
    assert np.sum(o.veloc ** 2) < 0.5 * np.sum(u.veloc ** 2)


def test_rayleigh_assemble_keeps_damping_out_of_finte(oracle, bar):
    """sma_assemble with damping: rhsid and frxid carry the Rayleigh force,
    finte and fexte do not (sld_elmmat.f90:170, sld_element_operations)."""
    import dataclasses
    p = dataclasses.replace(bar, dampi=np.array([[3.0e5, 0.0]]))
    rng = np.random.default_rng(7)
    u = rng.normal(size=(p.npoin, 3)) * 1e-3
    v = rng.normal(size=(p.npoin, 3)) * 1e3
    g = sma.ExplicitSolid(p, precision="fp64", scatter="color")
    g.set("veloc", v)
    got = g.assemble(u)
    o = oracle.Problem(p)
    ref = o.assemble(u, veloc=v)
    for k in ("rhsid", "finte", "fexte", "frxid"):
        scale = max(np.abs(ref[k]).max(), 1e-30)
        assert np.abs(got[k] - ref[k]).max() <= 1e-8 * scale + 1e-300, k
    und = oracle.Problem(bar).assemble(u)
    assert np.abs(ref["finte"] - und["finte"]).max() <= 1e-12 * np.abs(und["finte"]).max()
    assert np.abs(ref["rhsid"] - und["rhsid"]).max() > 1e-3 * np.abs(und["rhsid"]).max()


def _funbou(oracle, tab, smooth, t):
    fn = oracle.lib().orc_funbou_f64
    fn.restype = C.c_double
    fn.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_double]
    tb = np.ascontiguousarray(tab, dtype=np.float64)
    return fn(tb.shape[0], tb.ctypes.data_as(C.POINTER(C.c_double)), int(smooth), 0, float(t))


@pytest.mark.parametrize("alpha,scheme", [(0.0, "cd"), (1.0e5, "cd"), (0.0, "tw")])
def test_energy_balance_matches_restatement(oracle, canti, alpha, scheme):
    """ALLIE/ALLWK/ALLKE/ETOTA/EENER of mod_sld_energy.f90:71-193, computed by
    the device after every step, against the same formulas evaluated on
    oracle step snapshots (central difference and Tchamwa-Wielgosz).  With
    Rayleigh damping the internal force of the balance is finte, which leaves
    the damping force out as the reference's does."""
    import dataclasses
    p = dataclasses.replace(canti, dampi=np.array([[alpha, 0.0]])) if alpha else canti
    nsteps = 200
    g = sma.ExplicitSolid(p, precision="fp64", scheme=scheme)
    g.set_energy(True, nsteps)
    g.step(nsteps)
    tot, hist = g.energy()
    assert hist.shape == (nsteps, 5)
    o = oracle.Problem(p)
    vmass = o.assemble(np.zeros_like(o.displ))["vmass"]
    o.sdv[:] = 0.0
    side = oracle.Problem(p)                                   # re-runs a step's element loop
    tab = p.fun_table(p.load_fun)
    allie = allwk = 0.0
    fint_prev = np.zeros_like(o.displ)
    fext_prev = np.zeros_like(o.displ)
    ref = []
    for s in range(nsteps):
        u0 = o.displ.copy()
        v0, sdv0 = o.veloc.copy(), o.sdv.copy()
        o.run(p.dtime, 1, scheme=scheme, phi=1.033)
        fx = p.fext * _funbou(oracle, tab, p.fun_smooth[p.load_fun], o.cutim[0])
        if alpha:
            side.sdv[:] = sdv0
            fi = side.assemble(o.displ, veloc=v0)["finte"]
        else:
            fi = fx - o.rhsid
        dd = o.displ - u0
        ie = np.sum((fi + fint_prev) * dd)
        wk = np.sum((fx + fext_prev) * dd)
        w = 1.0 if s == 0 else 0.5
        allie += w * abs(ie)
        allwk += w * abs(wk)
        allke = 0.5 * np.sum(vmass[:, None] * o.veloc ** 2)
        ref.append((allie, allwk, allke, allie + allke - allwk, abs(np.sum(o.rhsid * dd))))
        fint_prev, fext_prev = fi, fx
    ref = np.array(ref)
    for q in range(3):
        scale = np.abs(ref[:, q]).max()
        assert np.abs(hist[:, q] - ref[:, q]).max() <= 1e-6 * scale + 1e-30, q
    assert abs(tot["allwk"] - ref[-1, 1]) <= 1e-6 * abs(ref[-1, 1])
    assert ref[-1, 1] > 0.0                                   # the traction did work


def test_reaction_witness(oracle, canti):
    """Residual witnesses on the clamped face are the reactions frxid_sld:
    after the element loop they equal the oracle's rhsid there."""
    p = canti
    nsteps = 150
    root = P.face_nodes(p.coord, 0, 0.0)
    wit = [3 * p.npoin + 3 * int(n) for n in root]            # x-residual of every root node
    g = sma.ExplicitSolid(p, precision="fp64")
    g.set_witness(wit, nsteps)
    g.step(nsteps)
    h = g.witness()
    o = oracle.Problem(p)
    o.run(p.dtime, nsteps)
    last_ref = o.rhsid[root, 0]
    assert np.abs(h[-1] - last_ref).max() <= 1e-8 * np.abs(last_ref).max()
    assert abs(h[-1].sum()) > 0.0


def test_checkpoint_resume_is_bitwise(bar, tmp_path):
    a = sma.ExplicitSolid(bar, precision="fp64", scatter="color")
    a.set_energy(True, 0)
    a.step(60)
    path = os.fspath(tmp_path / "ckpt.bin")
    a.save(path)
    a.step(40)
    b = sma.ExplicitSolid(bar, precision="fp64", scatter="color")
    b.load(path)
    b.step(40)
    for f in ("displ", "veloc", "accel"):
        assert np.array_equal(a.get(f), b.get(f)), f
    assert np.array_equal(a.state, b.state)
    assert a.time == b.time
    assert a.energy()[0] == b.energy()[0]


def test_checkpoint_rejects_other_mesh(bar, tmp_path):
    a = sma.ExplicitSolid(bar, precision="fp64")
    path = os.fspath(tmp_path / "c.bin")
    a.save(path)
    other = P.bar_40x4x4(nsteps=10, scale=2)
    b = sma.ExplicitSolid(other, precision="fp64")
    with pytest.raises(sma.SmaError, match="another mesh"):
        b.load(path)
