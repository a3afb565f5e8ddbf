"""Known answers for the oracle's stress/strain post-processing
(sld_calculate_pp_tensors): homogeneous deformations of the 40x4x4 bar give
the same tensors at every node, whatever the N dV weighting."""
import numpy as np

from alya_sma_b200 import problem as P


def _homogeneous(p, Fm):
    """Displacement of the homogeneous deformation x = F X about the centre."""
    X = p.coord - p.coord.mean(axis=0)
    return X @ (np.asarray(Fm) - np.eye(3)).T


def test_uniform_stretch_strains_and_elastic_stress(oracle):
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    o = oracle.Problem(p)
    lam = 1.0 + 2e-4                                              # elastic (no transformation)
    u = _homogeneous(p, np.diag([lam, 1.0, 1.0]))
    r = o.postprocess(u, gp_sigma=True)
    eps = np.log(lam)
    green = np.zeros(6)
    green[0] = 0.5 * (lam * lam - 1.0)
    lepsi = np.zeros(6)
    lepsi[0] = eps
    assert np.abs(r["green"] - green).max() < 1e-15
    assert np.abs(r["lepsi"] - lepsi).max() < 1e-15
    # tau = K eps I + 2 G dev(diag(eps, 0, 0)), sigma = tau / J
    E, nu = p.props[0, 0], p.props[0, 1]
    K, G = E / (3 * (1 - 2 * nu)), E / (2 * (1 + nu))
    sig = np.zeros(6)
    sig[0] = (K * eps + 2 * G * (2.0 / 3.0) * eps) / lam
    sig[1] = sig[2] = (K * eps - 2 * G * eps / 3.0) / lam
    assert np.abs(r["caust"] - sig).max() < 1e-9 * abs(sig[0])
    assert np.abs(r["gp_sigma"] - sig).max() < 1e-9 * abs(sig[0])
    vm = abs(sig[0] - sig[1])
    assert np.abs(r["seqvm"] - vm).max() < 1e-9 * vm


def test_rigid_rotation_has_no_strain_or_stress(oracle):
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    o = oracle.Problem(p)
    c, s = np.cos(0.3), np.sin(0.3)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    r = o.postprocess(_homogeneous(p, R))
    assert np.abs(r["green"]).max() < 1e-14
    assert np.abs(r["lepsi"]).max() < 1e-14
    assert np.abs(r["caust"]).max() < 1e-8                        # MPa, against E = 6e4
    assert np.abs(r["seqvm"]).max() < 1e-8


def test_shear_green_and_log_strain_components(oracle):
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    o = oracle.Problem(p)
    g = 1e-3
    Fm = np.eye(3)
    Fm[0, 1] = g                                                  # simple shear x += g y
    r = o.postprocess(_homogeneous(p, Fm))
    # Green strain of simple shear: E_xy = g/2, E_yy = g^2/2 (Voigt xx yy zz yz xz xy)
    assert abs(r["green"][:, 5].mean() - 0.5 * g) < 1e-15
    assert abs(r["green"][:, 1].mean() - 0.5 * g * g) < 1e-15
    # log strain: (ln V)_xy = g/2 + O(g^3), nothing out of plane
    assert abs(r["lepsi"][:, 5].mean() - 0.5 * g) < 1e-9
    assert np.abs(r["lepsi"][:, 2]).max() < 1e-15
