"""The oracle's algorithmic tangent (flagt = 1, sld_stress_model_160.f90:
118-155, 170-191) against known answers: at F = I it is the isotropic
elasticity tensor of the austenite, up to the O(eps) truncation of its
eps = 1e-5 forward differences; it has both minor symmetries exactly and, in
the elastic (hyperelastic) range, the major symmetry to that truncation."""
import numpy as np

from alya_sma_b200 import problem as P

NITI = P.nitinol_props(**P.NITI)


def _tangent(oracle, F, sdv):
    Fc = np.ascontiguousarray(np.asarray(F).transpose(0, 2, 1)).reshape(-1, 9)
    pk2, sn, dds, fl = oracle.law160_tangent_batch(NITI, Fc, sdv)
    return dds.reshape(-1, 3, 3, 3, 3).transpose(0, 4, 3, 2, 1), fl


def test_tangent_at_identity_is_isotropic_elasticity(oracle):
    E, nu = NITI[0], NITI[1]
    K, G = E / (3 * (1 - 2 * nu)), E / (2 * (1 + nu))
    d = np.eye(3)
    c = (K - 2 * G / 3) * np.einsum("ij,kl->ijkl", d, d) + G * (
        np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d))
    D, fl = _tangent(oracle, np.eye(3)[None], np.zeros((1, 3)))
    assert fl[0] == 0
    assert np.abs(D[0] - c).max() <= 1e-5 * np.abs(c).max()


def test_tangent_symmetries(oracle):
    rng = np.random.default_rng(4)
    F = np.eye(3)[None] + 0.001 * rng.normal(size=(20, 3, 3))   # below the AS start
    D, fl = _tangent(oracle, F, np.zeros((20, 3)))
    assert np.all(fl == 0)
    scale = np.abs(D).max()
    assert np.abs(D - D.transpose(0, 2, 1, 3, 4)).max() <= 1e-12 * scale
    assert np.abs(D - D.transpose(0, 1, 2, 4, 3)).max() <= 1e-12 * scale
    assert np.abs(D - D.transpose(0, 3, 4, 1, 2)).max() <= 1e-4 * scale
