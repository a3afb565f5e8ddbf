"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (relative to the largest magnitude of the compared quantity):
  FP64 form vs oracle  -- law stress 1e-8, element-loop forces 1e-8,
    trajectories 1e-6.  The FP64 form evaluates log(b) from A = b - I
    (see sma_law.cuh); against an exact evaluation it is accurate to ~3e-15,
    while the reference's own b -> eig -> log route carries up to ~4e-10
    relative error at small strains, so 1e-8 bounds the reference's rounding,
    not ours.
  FP32 form vs oracle  -- law stress 2e-4, forces 1e-3, tip displacement
    1e-4 (the precision targets of the FP32 form).
"""
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


NITI = P.nitinol_props(**P.NITI)


def rotation(rng):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] *= -1
    return q


def random_gauss_points(n, seed=0, rot=0.2):
    """Gauss points with physically consistent histories: a previous state
    (xS0, F0) inside the law's admissible band (austenite below the AS start,
    mixtures between the SA and AS finish lines, martensite above the SA
    start), and a current F = R U whose deviatoric log strain is within +-5 %
    of the previous one (random direction, small volumetric part, rotation up
    to `rot` rad).  Inconsistent states (F0 far above Rf_AS with 0 < xS0 < 1)
    make the return map's denominator vanish and are not reachable by the law."""
    rng = np.random.default_rng(seed)
    F = np.zeros((n, 3, 3))
    sdv = np.zeros((n, 3))
    E, nu, eL = NITI[0], NITI[1], NITI[2]
    G = E / (2 + 2 * nu)
    aux = np.sqrt(2 / 3)
    Rs_AS, Rf_AS, Rs_SA, Rf_SA = NITI[3] * aux, NITI[4] * aux, NITI[9] * aux, NITI[10] * aux
    for g in range(n):
        kind = g % 4
        if kind == 0:
            x0, F0 = 0.0, rng.uniform(0.0, Rs_AS)
        elif kind == 1:
            x0, F0 = rng.uniform(0.0, 1.0), rng.uniform(Rf_SA, Rf_AS)
        elif kind == 2:
            x0, F0 = 1.0, rng.uniform(Rs_SA, 1.5 * Rf_AS)
        else:
            x0, F0 = 0.0, rng.uniform(0.0, 0.05 * Rs_AS)      # small strains
        en_prev = F0 / (2 * G) + eL * x0
        en = max(en_prev * (1 + rng.uniform(-0.05, 0.05)), 1e-7)
        r = rng.normal(size=3)
        d = r - r.mean()
        d /= np.linalg.norm(d)
        lam = np.exp(en * d + rng.uniform(-0.005, 0.005) / 3)
        Q = rotation(rng)
        U = Q @ np.diag(lam) @ Q.T
        w = rng.normal(size=3)
        w *= rng.uniform(0, rot) / np.linalg.norm(w)
        K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
        th = np.linalg.norm(w)
        R = np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K
        F[g] = R @ U
        sdv[g] = (x0, F0, F0)
    return F, sdv


def oracle_batch(oracle, F, sdv, e_mart=0.0, tmp=None):
    Fc = np.ascontiguousarray(F.transpose(0, 2, 1)).reshape(-1, 9)
    pk2, sn, fl = oracle.law160_batch(NITI, Fc, sdv, tmp=tmp, e_mart=e_mart)
    return pk2.reshape(-1, 3, 3).transpose(0, 2, 1), sn, fl


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 2e-4)])
def test_law_batch_matches_oracle(oracle, precision, tol):
    F, sdv = random_gauss_points(4000, seed=1)
    S_ref, s_ref, fl_ref = oracle_batch(oracle, F, sdv)
    S, s, fl = sma.eval_sld_stress_model_160(NITI, F, sdv, precision=precision)
    S, s, fl = S.cpu().numpy(), s.cpu().numpy(), fl.cpu().numpy()
    scale = np.abs(S_ref).reshape(len(F), -1).max(axis=1)
    err = np.abs(S - S_ref).reshape(len(F), -1).max(axis=1) / scale
    assert np.max(err) < tol, (np.max(err), np.argmax(err))
    same = (fl & 3) == (fl_ref & 3)
    assert same.mean() > (0.999 if precision == "fp64" else 0.99)
    assert np.max(np.abs(s[same, 0] - s_ref[same, 0])) < (1e-9 if precision == "fp64" else 1e-4)
    assert (fl_ref & 1).sum() > 300        # the batch exercises the return map


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 5e-4)])
def test_law_frame_indifference(precision, tol):
    """The CUDA law is objective and isotropic, as law 160 is: the second
    Piola stress does not change under a spatial rotation (S(R F) = S(F))
    and turns with a rotation of the reference configuration
    (S(F Q) = Q^T S(F) Q), with the same state update.  A rotation changes
    rounding, so a point sitting on a transformation threshold may switch
    branch; such points (same flags required for 99 %) are left out.  The
    FP32 form's absolute stress error under a rotation is ~E eps32 |F - I|
    whatever the strain, so errors are taken relative to max(|S|, 1e-3 E)."""
    F, sdv = random_gauss_points(3000, seed=9)
    rng = np.random.default_rng(19)
    R = np.stack([rotation(rng) for _ in range(len(F))])
    Q = np.stack([rotation(rng) for _ in range(len(F))])
    S, s, fl = (x.cpu().numpy() for x in sma.eval_sld_stress_model_160(NITI, F, sdv, precision=precision))
    SR, sR, flR = (x.cpu().numpy() for x in sma.eval_sld_stress_model_160(NITI, R @ F, sdv, precision=precision))
    SQ, sQ, flQ = (x.cpu().numpy() for x in sma.eval_sld_stress_model_160(NITI, F @ Q, sdv, precision=precision))
    same = (fl == flR) & (fl == flQ)
    assert same.mean() >= 0.99
    scale = np.maximum(np.abs(S).reshape(len(F), -1).max(axis=1), 1e-3 * NITI[0])[same]
    errR = np.abs(SR - S).reshape(len(F), -1).max(axis=1)[same] / scale
    SQ_back = np.einsum("gki,gkl,glj->gij", Q, S, Q)                # Q^T S Q
    errQ = np.abs(SQ - SQ_back).reshape(len(F), -1).max(axis=1)[same] / scale
    assert errR.max() < tol and errQ.max() < tol, (errR.max(), errQ.max())
    assert np.abs(sR[same, 0] - s[same, 0]).max() < (1e-9 if precision == "fp64" else 1e-4)


def test_law_tangent_matches_oracle(oracle):
    """flagt = 1: the algorithmic tangent (sld_stress_model_160.f90:118-155,
    170-191).  The GPU evaluates the six distinct perturbations and carries
    the tangent on symmetric pairs; the oracle follows the reference's nine
    perturbations and 81-term pull-back literally.  Forward differences with
    eps = 1e-5 magnify the stress difference between the two law forms
    (<= ~4e-10 relative, the reference's eigen route) by |tau| / eps, and a
    perturbation that crosses a transformation threshold in one form but not
    the other changes that point's tangent outright: elastic points are held
    to 1e-6 of the point's largest entry, 99 % of all points to 1e-5."""
    F, sdv = random_gauss_points(4000, seed=5)
    F[0], sdv[0] = np.eye(3), 0.0
    Fc = np.ascontiguousarray(F.transpose(0, 2, 1)).reshape(-1, 9)
    pk2_ref, s_ref, dds_ref, fl_ref = oracle.law160_tangent_batch(NITI, Fc, sdv)
    D_ref = dds_ref.reshape(-1, 3, 3, 3, 3).transpose(0, 4, 3, 2, 1)
    S, s, fl, D = sma.eval_sld_stress_model_160(NITI, F, sdv, flagt=1)
    S, D, fl = S.cpu().numpy(), D.cpu().numpy(), fl.cpu().numpy()
    S_ref = pk2_ref.reshape(-1, 3, 3).transpose(0, 2, 1)
    assert np.abs(S - S_ref).max() <= 1e-8 * np.abs(S_ref).max()
    n = len(F)
    err = np.abs(D - D_ref).reshape(n, -1).max(axis=1) / np.abs(D_ref).reshape(n, -1).max(axis=1)
    elastic = (fl_ref == 0) & (fl == 0)
    assert elastic.sum() > 300 and (fl_ref & 1).sum() > 300
    assert err[elastic].max() < 1e-6, err[elastic].max()
    assert np.mean(err < 1e-5) >= 0.99, np.quantile(err, 0.99)
    # the known answer at F = I: isotropic elasticity of the austenite
    E, nu = NITI[0], NITI[1]
    K, G = E / (3 * (1 - 2 * nu)), E / (2 * (1 + nu))
    d = np.eye(3)
    c = (K - 2 * G / 3) * np.einsum("ij,kl->ijkl", d, d) + G * (
        np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d))
    assert np.abs(D[0] - c).max() <= 1e-5 * np.abs(c).max()
    with pytest.raises(sma.SmaError, match="FP64 only"):
        sma.eval_sld_stress_model_160(NITI, F[:4], sdv[:4], flagt=1, precision="fp32")


def test_law_batch_extension_modulus_and_temperature(oracle):
    F, sdv = random_gauss_points(1000, seed=2)
    tmp = np.random.default_rng(3).uniform(-10, 10, size=len(F))
    props = NITI.copy()
    props[5] = props[11] = 6.5 * np.sqrt(2 / 3)
    Fc = np.ascontiguousarray(F.transpose(0, 2, 1)).reshape(-1, 9)
    pk2, sn, fl = oracle.law160_batch(props, Fc, sdv, tmp=tmp, e_mart=40000.0)
    S_ref = pk2.reshape(-1, 3, 3).transpose(0, 2, 1)
    S, s, f = sma.eval_sld_stress_model_160(props, F, sdv, gptmp=tmp, e_mart=40000.0)
    S = S.cpu().numpy()
    err = np.abs(S - S_ref).max() / np.abs(S_ref).max()
    assert err < 1e-8


@pytest.fixture(scope="module")
def bar():
    return P.bar_40x4x4(nsteps=400)


def deformed(p, seed=0, strain=0.02):
    rng = np.random.default_rng(seed)
    X = p.coord
    u = np.zeros_like(X)
    u[:, 0] = strain * X[:, 0] * (1 + 0.3 * np.sin(X[:, 0] / 7.0))
    u[:, 1] = -0.3 * strain * (X[:, 1] - 2.0) + 0.002 * np.sin(X[:, 0] / 5.0)
    u[:, 2] = -0.3 * strain * (X[:, 2] - 2.0)
    u += rng.normal(size=u.shape) * 1e-4
    return u


@pytest.mark.parametrize("precision,scatter,tol", [("fp64", "atomic", 1e-8), ("fp64", "color", 1e-8),
                                                   ("fp32", "atomic", 1e-3)])
def test_element_loop_matches_oracle(oracle, bar, precision, scatter, tol):
    o = oracle.Problem(bar)
    g = sma.ExplicitSolid(bar, precision=precision, scatter=scatter)
    for it, strain in enumerate((0.006, 0.012, 0.03)):      # elastic, onset, plateau
        u = deformed(bar, seed=it, strain=strain)
        ro = o.assemble(u)
        o.end_step()
        rg = g.assemble(u)
        g.end_step()
        scale = np.abs(ro["finte"]).max()
        for q in ("rhsid", "finte", "frxid"):
            err = np.abs(rg[q] - ro[q]).max() / scale
            assert err < tol, (q, strain, err)
        np.testing.assert_allclose(rg["vmass"], ro["vmass"], rtol=1e-13)
        sg, so = g.state, o.sdv
        assert np.abs(sg[:, 1, :, 0] - so[:, 1, :, 0]).max() < (1e-8 if precision == "fp64" else 2e-3)
    assert so[:, 1, :, 0].max() > 0.05                     # martensite formed
    g.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_compact_records_equal_the_material_table(oracle, precision):
    """Per-element materials that differ only in E_A, E_M, eL and the
    transformation stresses (the cylinder's sampling) run from compact 8-word
    records in registers; SMA_VARIANT_TABLE stages each element's full
    material through shared memory.  Both give the oracle's residual and
    state, and each other's to round-off of the record's precision.  A mesh
    whose materials also differ in nu cannot use the records and runs from
    the table."""
    import dataclasses
    p = P.cylinder_2m(nsteps=600, div=8)
    u = P.prestrain(p, 0.03) + np.random.default_rng(5).normal(size=p.coord.shape) * 1e-4
    u[p.fixno == 1] = 0.0
    o = oracle.Problem(p)
    ro = o.assemble(u)
    o.end_step()
    scale = np.abs(ro["finte"]).max()
    out = {}
    for variant in ("plain", "table"):
        g = sma.ExplicitSolid(p, precision=precision, scatter="color", variant=variant)
        out[variant] = g.assemble(u)["rhsid"]
        g.end_step()
        out[variant + "_xs"] = g.state[:, 1, :, 0]
        g.close()
        tol = 1e-8 if precision == "fp64" else 1e-3
        assert np.abs(out[variant] - ro["rhsid"]).max() / scale < tol, variant
    d = np.abs(out["plain"] - out["table"]).max() / scale
    assert d < (1e-12 if precision == "fp64" else 1e-5), d
    assert np.abs(out["plain_xs"] - out["table_xs"]).max() < (1e-12 if precision == "fp64" else 1e-4)
    # materials that also differ in Poisson's ratio: the table path
    props = p.props.copy()
    props[:, 1] *= np.random.default_rng(6).uniform(0.97, 1.03, size=len(props))
    q = dataclasses.replace(p, props=props)
    oq = oracle.Problem(q)
    rq = oq.assemble(u)
    g = sma.ExplicitSolid(q, precision=precision, scatter="color")
    rg = g.assemble(u)["rhsid"]
    assert np.abs(rg - rq["rhsid"]).max() / np.abs(rq["finte"]).max() < (1e-8 if precision == "fp64" else 1e-3)
    g.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("mesh", ["bar", "cylinder"])
def test_every_block_width_matches_oracle(oracle, bar, mesh, precision):
    """The element kernel is compiled twice: for blocks of at most 128 threads
    (a tighter register cap, more warps per SM) and for up to 256.  Both,
    with one material and with per-element materials, give the oracle's
    residual and state; the two colour-scatter FP64 results agree to
    round-off."""
    if mesh == "bar":
        p, u = bar, deformed(bar, seed=3, strain=0.03)
    else:
        p = P.cylinder_2m(nsteps=600, div=8)
        u = P.prestrain(p, 0.03) + np.random.default_rng(3).normal(size=p.coord.shape) * 1e-4
        u[p.fixno == 1] = 0.0
    o = oracle.Problem(p)
    ro = o.assemble(u)
    o.end_step()
    so = o.sdv[:, 1, :, 0]
    assert so.max() > 0.0                                  # martensite forms
    scale = np.abs(ro["finte"]).max()
    tol, tol_x = (1e-8, 1e-8) if precision == "fp64" else (1e-3, 2e-3)
    rhs = {}
    for block in (32, 64, 128, 192, 256):
        g = sma.ExplicitSolid(p, precision=precision, scatter="color", block=block)
        rg = g.assemble(u)
        g.end_step()
        for q in ("rhsid", "finte"):
            err = np.abs(rg[q] - ro[q]).max() / scale
            assert err < tol, (block, q, err)
        assert np.abs(g.state[:, 1, :, 0] - so).max() < tol_x, block
        rhs[block] = rg["rhsid"]
        g.close()
    if precision == "fp64":
        assert np.abs(rhs[128] - rhs[256]).max() <= 1e-12 * scale


def _first_elements(p, k):
    """The first k elements of p with their nodes renumbered."""
    nodes = np.unique(p.lnods[:k])
    remap = -np.ones(p.npoin, np.int64)
    remap[nodes] = np.arange(nodes.size)
    return P.Problem(coord=p.coord[nodes], lnods=remap[p.lnods[:k]].astype(np.int32), props=p.props,
                     e_mart=p.e_mart, densi=p.densi, fixno=p.fixno[nodes], bcfun=p.bcfun[nodes],
                     fun_npts=p.fun_npts, fun_smooth=p.fun_smooth, fun_tab=p.fun_tab,
                     fext=None if p.fext is None else p.fext[nodes], load_fun=p.load_fun,
                     dtime=p.dtime, nsteps=p.nsteps)


@pytest.mark.parametrize("k", [1, 3, 9])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 1e-3)])
def test_meshes_smaller_than_a_tile(oracle, bar, k, precision, tol):
    """1, 3 and 9 elements: fewer than the 8 elements of one default block,
    and one ragged tile past it (the lanes of missing elements gather a valid
    element's nodes but neither write state nor scatter forces)."""
    q = _first_elements(bar, k)
    assert q.nelem == k
    u = deformed(q, seed=k, strain=0.03)
    u[q.fixno == 1] = 0.0
    o = oracle.Problem(q)
    ro = o.assemble(u)
    o.end_step()
    g = sma.ExplicitSolid(q, precision=precision)
    rg = g.assemble(u)
    g.end_step()
    scale = np.abs(ro["finte"]).max()
    for key in ("rhsid", "finte"):
        assert np.abs(rg[key] - ro[key]).max() <= tol * scale, key
    np.testing.assert_allclose(rg["vmass"], ro["vmass"], rtol=1e-13)
    assert np.abs(g.state[:, 1, :, 0] - o.sdv[:, 1, :, 0]).max() < (1e-8 if precision == "fp64" else 2e-3)
    # free vibration from the deformed state
    o2 = oracle.Problem(q)
    o2.displ[:] = u
    o2.run(q.dtime, 30)
    g2 = sma.ExplicitSolid(q, precision=precision)
    g2.set("displ", u)
    g2.step(30)
    ud, ud_ref = g2.get("displ"), o2.displ
    assert np.abs(ud - ud_ref).max() <= (1e-6 if precision == "fp64" else 1e-3) * np.abs(ud_ref).max()
    assert g2.counters()["nonfinite"] == 0


def test_colour_scatter_is_deterministic(bar):
    runs = []
    for _ in range(2):
        g = sma.ExplicitSolid(bar, precision="fp64", scatter="color")
        g.step(150)
        runs.append((g.get("displ"), g.get("veloc"), g.state))
        g.close()
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)


def test_trajectory_fp64_matches_oracle(oracle, bar):
    nsteps = 400
    mid = int(np.argmin(np.sum((bar.coord - [20, 2, 2]) ** 2, axis=1)))
    q = int(np.argmin(np.sum((bar.coord - [30, 4, 0]) ** 2, axis=1)))
    wit = [3 * mid, 3 * mid + 1, 3 * q, 3 * q + 2]
    o = oracle.Problem(bar)
    h_ref = o.run(bar.dtime, nsteps, wit_dof=wit)
    g = sma.ExplicitSolid(bar, precision="fp64")
    g.set_witness(wit, nsteps)
    g.step(nsteps)
    h = g.witness()
    assert h.shape == h_ref.shape
    err = np.abs(h - h_ref).max() / np.abs(h_ref).max()
    assert err < 1e-6, err
    u_ref, u = o.displ, g.get("displ")
    assert np.abs(u - u_ref).max() / np.abs(u_ref).max() < 1e-6
    assert np.abs(g.get("veloc") - o.veloc).max() / np.abs(o.veloc).max() < 1e-5
    xs, xs_ref = g.state[:, 1, :, 0], o.sdv[:, 1, :, 0]
    assert xs_ref.max() > 0.1
    assert np.abs(xs - xs_ref).max() < 1e-5
    assert abs(g.time - o.cutim[0]) <= 1e-18
    c = g.counters()
    assert c["nr_failed"] == 0 and c["nonfinite"] == 0 and c["neg_det"] == 0
    assert c["gpdet_min"] == 0.0 and c["ielem_min"] == -1      # no det F <= 0 met
    assert c["nr_active"] > 0


def test_step_chunking_is_invisible(bar):
    """one call of 37 steps == calls of 1 + 8 + 20 + 8 steps (graph chunks,
    remainders and the per-call prologue/epilogue)."""
    a = sma.ExplicitSolid(bar, precision="fp64", scatter="color")
    a.step(37)
    b = sma.ExplicitSolid(bar, precision="fp64", scatter="color")
    for n in (1, 8, 20, 8):
        b.step(n)
    assert np.array_equal(a.get("displ"), b.get("displ"))
    assert np.array_equal(a.get("accel"), b.get("accel"))
    assert np.array_equal(a.state, b.state)
    assert a.time == b.time


def test_precision_form_cantilever(oracle):
    """FP32 form vs the FP64 oracle on a traction-loaded cantilever
    (400x40x40 mm at 1/10 resolution): tip displacement and stress."""
    p = P.cantilever_400x40x40(nsteps=1500, div=10)
    tip = int(np.argmin(np.sum((p.coord - [400, 20, 20]) ** 2, axis=1)))
    wit = [3 * tip]
    o = oracle.Problem(p)
    h_ref = o.run(p.dtime, 1500, wit_dof=wit)
    g = sma.ExplicitSolid(p, precision="fp32")
    g.set_witness(wit, 1500)
    g.step(1500)
    h = g.witness()[:, 0]
    h_ref = h_ref[:, 0]
    # peak tip displacement: the precision target 1e-4
    ipk = int(np.argmax(np.abs(h_ref)))
    rel_peak = abs(h[ipk] - h_ref[ipk]) / abs(h_ref[ipk])
    assert rel_peak < 1e-4, rel_peak                         # measured 1.5e-8
    # whole history: the activation test of the law (F > F0 and F > Rs,
    # sld_stress_model_160.f90:351,368) is discontinuous, so a rounding-level
    # difference shifts the step at which a Gauss point starts transforming
    # and the tip history parts by more than the rounding.  The FP64 oracle
    # moved by one FP32 ulp of its coordinates parts from itself by
    # 2.3e-4 over this history; the FP32 form (1.8e-4 measured) is held to
    # the 1e-4 target or, where the law's own spread exceeds it, to twice
    # that spread.
    import dataclasses
    pert = dataclasses.replace(p, coord=p.coord * (1 + 2.0 ** -24))
    h_self = oracle.Problem(pert).run(p.dtime, 1500, wit_dof=wit)[:, 0]
    spread = np.abs(h_self - h_ref).max() / np.abs(h_ref).max()
    rel_hist = np.abs(h - h_ref).max() / np.abs(h_ref).max()
    assert rel_hist <= max(1e-4, 2.0 * spread), (rel_hist, spread)
    # stresses at the final displacement: FP32 element loop vs FP64 oracle
    u = o.displ.copy()
    g2 = sma.ExplicitSolid(p, precision="fp32")
    g2.state = o.sdv
    o2 = oracle.Problem(p)
    o2.sdv[:] = o.sdv
    rg, ro = g2.assemble(u), o2.assemble(u)
    rel_f = np.abs(rg["finte"] - ro["finte"]).max() / np.abs(ro["finte"]).max()
    assert rel_f < 1e-3, rel_f


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_patch_and_rigid_motion(bar, precision):
    """Known answers of the element loop on the jittered bar, through the C
    ABI: constant strain leaves no force on interior nodes; a finite rigid
    rotation plus translation gives no force at all (FP32: the rounding of
    F = R is a strain of ~1e-7)."""
    import dataclasses
    p = dataclasses.replace(bar, e_mart=np.full_like(bar.e_mart, bar.props[0, 0]))
    X = p.coord
    inner = np.all((X > X.min(axis=0) + 1e-9) & (X < X.max(axis=0) - 1e-9), axis=1)
    rng = np.random.default_rng(3)
    G = rng.normal(size=(3, 3)) * 1e-4
    g = sma.ExplicitSolid(p, precision=precision)
    r = g.assemble(X @ G.T, want_all=False)["rhsid"]
    tol = 1e-10 if precision == "fp64" else 1e-4
    assert np.abs(r[inner]).max() <= tol * np.abs(r).max()
    c, s = np.cos(0.7), np.sin(0.7)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    rr = g.assemble(X @ (R - np.eye(3)).T + np.array([3.0, -1.0, 2.0]), want_all=False)["rhsid"]
    ref = g.assemble(X * np.array([1e-4, 0.0, 0.0]), want_all=False)["rhsid"]
    assert np.abs(rr).max() <= (1e-9 if precision == "fp64" else 1e-2) * np.abs(ref).max()


def test_full_load_cycle_within_the_laws_own_sensitivity(oracle):
    """The whole 40x4x4 bar load cycle (4,000 steps: pull to 6 % strain and
    release).  During loading the GPU and the oracle agree to round-off; in
    the reverse transformation the law's strict activation inequalities
    (sld_stress_model_160.f90:351,368) amplify round-off by ~1e9, so over the
    full cycle the GPU is held to the oracle's own sensitivity: the oracle
    against itself with coordinates scaled by (1 + 1e-15)."""
    import dataclasses
    p = P.bar_40x4x4(nsteps=4000)
    mid = int(np.argmin(np.sum((p.coord - [20, 2, 2]) ** 2, axis=1)))
    q = int(np.argmin(np.sum((p.coord - [30, 4, 0]) ** 2, axis=1)))
    wit = [3 * mid, 3 * mid + 1, 3 * q, 3 * q + 2]
    h_ref = oracle.Problem(p).run(p.dtime, 4000, wit_dof=wit)
    pert = dataclasses.replace(p, coord=p.coord * (1 + 1e-15))
    h_self = oracle.Problem(pert).run(p.dtime, 4000, wit_dof=wit)
    scale = np.abs(h_ref).max()
    e_self = np.abs(h_self - h_ref).max(axis=1) / scale
    # the same for a perturbation of one FP32 ulp, the precision form's scale
    pert32 = dataclasses.replace(p, coord=p.coord * (1 + 2.0 ** -24))
    h_self32 = oracle.Problem(pert32).run(p.dtime, 4000, wit_dof=wit)
    e_self32 = np.abs(h_self32 - h_ref).max(axis=1) / scale
    out = {}
    for prec in ("fp64", "fp32"):
        g = sma.ExplicitSolid(p, precision=prec, scatter="color")
        g.set_witness(wit, 4000)
        g.step(4000)
        out[prec] = np.abs(g.witness() - h_ref).max(axis=1) / scale
    assert out["fp64"][:3000].max() < 1e-9                        # loading and plateau: round-off
    assert out["fp64"].max() <= 10 * e_self.max() + 1e-9           # whole cycle: the law's own spread
    assert out["fp32"][:2000].max() < 1e-4                         # precision form, loading half
    # precision form over the whole cycle, reverse transformation included:
    # up to every 500th step within 5x the spread of the oracle moved by one
    # FP32 ulp, and within 2e-5 while that spread is smaller (measured on
    # B200: 7.0e-6 / 1.0e-4 / 1.3e-3 at steps 2,000 / 3,000 / 4,000 against a
    # spread of 5.1e-8 / 4.2e-5 / 1.4e-3)
    for k in range(500, 4001, 500):
        got, lim = out["fp32"][:k].max(), max(2e-5, 5.0 * e_self32[:k].max())
        assert got <= lim, (k, got, e_self32[:k].max())
