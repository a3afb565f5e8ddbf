"""Stress and strain post-processing (sld_calculate_pp_tensors): nodal
Cauchy stress, Green and log strain, von Mises and the Gauss-point Cauchy
stress through the C ABI, against the oracle's literal restatement
(sigma = F P^T / det F, Green from F^T F, log strain from an eigen-
decomposition of F F^T, N dV projection over the volume-lumped mass)."""
import numpy as np
import pytest

import alya_sma_b200 as sma
from alya_sma_b200 import problem as P

pytestmark = pytest.mark.gpu

KEYS = ("caust", "green", "lepsi", "seqvm", "gp_sigma")


@pytest.fixture(scope="module", autouse=True)
def need_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


def _field(p, strain, seed, axis_len):
    """Axial stretch with a wavy profile, lateral contraction and noise."""
    rng = np.random.default_rng(seed)
    X = p.coord - p.coord.mean(axis=0)
    x = p.coord[:, 0]
    u = np.stack([strain * x * (1 + 0.2 * np.sin(6.0 * x / axis_len)),
                  -0.3 * strain * X[:, 1], -0.3 * strain * X[:, 2]], axis=1)
    return u + rng.normal(size=u.shape) * 1e-4


def _two_loops(g, o, p, strains, axis_len):
    """Two element loops in a row (the first one ended), the same on both."""
    for call, strain in enumerate(strains):
        u = _field(p, strain, call, axis_len)
        g.assemble(u)
        o.assemble(u)
        if call + 1 < len(strains):
            g.end_step()
            o.end_step()
    return u


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_postprocess_matches_oracle_bar(oracle, precision):
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    g = sma.ExplicitSolid(p, precision=precision)
    o = oracle.Problem(p)
    u = _two_loops(g, o, p, (0.012, 0.03), 40.0)
    st0 = g.state
    got = g.postprocess(gp_sigma=True)
    ref = o.postprocess(u, slot=1, gp_sigma=True)
    assert np.array_equal(g.state, st0)                         # the state is not changed
    assert o.sdv[:, 0, :, 0].max() > 0.05                       # martensite formed
    tol = {"fp64": dict(caust=1e-8, green=1e-12, lepsi=1e-8, seqvm=1e-8, gp_sigma=1e-8),
           "fp32": dict(caust=1e-3, green=1e-5, lepsi=1e-5, seqvm=2e-3, gp_sigma=1e-3)}[precision]
    for k in KEYS:
        assert _rel(got[k], ref[k]) < tol[k], (k, _rel(got[k], ref[k]))


def test_postprocess_per_element_materials_and_colour_order(oracle):
    """Cylinder (per-element materials, temperature field) with the coloured
    scatter, whose internal element order differs from the caller's: the
    Gauss-point output comes back in the caller's order."""
    p = P.cylinder_2m(nsteps=10, div=8)
    g = sma.ExplicitSolid(p, precision="fp64", scatter="color")
    o = oracle.Problem(p)
    u = _two_loops(g, o, p, (0.008, 0.02), 50.0)
    got = g.postprocess(gp_sigma=True)
    ref = o.postprocess(u, slot=1, gp_sigma=True)
    for k in KEYS:
        assert _rel(got[k], ref[k]) < 1e-8, (k, _rel(got[k], ref[k]))


def test_postprocess_after_steps_is_repeatable():
    """After a run of steps it reads the last loop's start state; calling it
    twice gives the same result (to the rounding of the FP64 atomic nodal
    sums, whose order varies) and leaves the run bit-for-bit unchanged."""
    p = P.bar_40x4x4(nsteps=200)
    a = sma.ExplicitSolid(p, precision="fp64", scatter="color")
    b = sma.ExplicitSolid(p, precision="fp64", scatter="color")
    a.step(120)
    b.step(120)
    r1 = a.postprocess()
    r2 = a.postprocess()
    for k in ("caust", "green", "lepsi", "seqvm"):
        assert _rel(r2[k], r1[k]) < 1e-12, (k, _rel(r2[k], r1[k]))
    assert r1["seqvm"].max() > 0.0
    a.step(30)
    b.step(30)
    assert np.array_equal(a.get("displ"), b.get("displ"))
    assert np.array_equal(a.state, b.state)
    # zero displacement and a fresh state: every field vanishes
    z = sma.ExplicitSolid(p, precision="fp64")
    r0 = z.postprocess()
    assert all(np.abs(r0[k]).max() == 0.0 for k in ("caust", "green", "lepsi", "seqvm"))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gauss_fields_match_oracle(oracle, precision):
    """gpgdi, gppio, det F per Gauss point and volum_sld(1:2), from the same
    evaluation as the stresses (the state the last element loop read)."""
    p = P.cylinder_2m(nsteps=10, div=8)                         # per-element materials
    g = sma.ExplicitSolid(p, precision=precision, scatter="color")
    o = oracle.Problem(p)
    u = _two_loops(g, o, p, (0.008, 0.02), 50.0)
    got = g.gauss_fields()
    ref = o.postprocess(u, slot=1, gauss=True)
    tol = {"fp64": dict(gpgdi=1e-13, gppio=1e-8, gpdet=1e-13, volum=1e-12),
           "fp32": dict(gpgdi=1e-6, gppio=1e-3, gpdet=1e-6, volum=1e-6)}[precision]
    for k in ("gpgdi", "gppio", "gpdet", "volum"):
        assert _rel(got[k], ref[k]) < tol[k], (k, _rel(got[k], ref[k]))
    assert ref["volum"][1] > ref["volum"][0]                      # stretched: volume grew


def test_negative_jacobian_report(oracle):
    """An element turned inside out: the element loop counts the Gauss points
    with det F <= 0 and reports the smallest det F and its element, as the
    reference's gpdet_min / ielem_min (sld_elmpre.f90:229-238)."""
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    u = np.zeros((p.npoin, 3))
    q = int(np.argmin(np.sum((p.coord - [20.0, 2.0, 2.0]) ** 2, axis=1)))
    u[q, 0] = 3.0                                                 # node pushed 3 element sizes along x
    g = sma.ExplicitSolid(p, precision="fp64", scatter="color")
    g.counters(reset=True)
    g.assemble(u)
    c = g.counters()
    ref = oracle.Problem(p).assemble(u)
    assert c["neg_det"] > 0
    assert ref["gpdet_min"] < 0.0
    assert abs(c["gpdet_min"] - ref["gpdet_min"]) <= 1e-6 * abs(ref["gpdet_min"])
    assert q in p.lnods[c["ielem_min"]]                           # an element of the moved node
    det = g.gauss_fields()["gpdet"]
    assert abs(det[c["ielem_min"]].min() - det.min()) <= 1e-6 * abs(det.min())
    g.counters(reset=True)
    c = g.counters()
    assert c["neg_det"] == 0 and c["ielem_min"] == -1
