"""The CPU oracle against the reference's own known answers.

* tests/golden/data1_transitions.npz: every martensite-transformation row of
  the reference's law-160 Gauss-point trace (tests/sma_explicit/data1.dat),
  replayed through the oracle's full 3-D law (made by
  tests/golden/make_golden.py).
* analytic answers of the law (elastic response, transformation onset, the
  linear flow rule's plateau) and of the eigen solver.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rot(a, b, c):
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    Rz = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rx = np.array([[1, 0, 0], [0, cc, -sc], [0, sc, cc]])
    return Rz @ Ry @ Rx


def colmajor(M):
    return np.asarray(M, dtype=np.float64).T.reshape(9).copy()


def F_from_enorm(en, theta=0.0, R=np.eye(3), Q=np.eye(3)):
    """Isochoric uniaxial stretch with deviatoric log-strain norm en (plus a
    volumetric log strain theta), rotated: F = Q R diag(l) R^T."""
    a = en / np.sqrt(1.5)
    lam = np.exp(np.array([a, -0.5 * a, -0.5 * a]) + theta / 3.0)
    return Q @ R @ np.diag(lam) @ R.T


def test_data1_transitions_reproduced(oracle):
    z = np.load(os.path.join(GOLD, "data1_transitions.npz"))
    props = z["props"]
    assert len(z["row"]) == 2300
    R = rot(0.3, -0.7, 1.1)
    Q = rot(-0.2, 0.4, 0.9)
    worst_F, worst_x, n_active = 0.0, 0.0, 0
    for k in range(len(z["row"])):
        F = F_from_enorm(z["en_new"][k], theta=0.01 * (k % 5), R=R if k % 2 else np.eye(3),
                         Q=Q if k % 3 == 0 else np.eye(3))
        sdv = [z["xS0"][k], z["F0"][k], z["F0"][k]]
        tau, s, fl = oracle.law160_kirchhoff(props, colmajor(F), sdv)
        worst_F = max(worst_F, abs(s[1] - z["F_new"][k]))
        worst_x = max(worst_x, abs(s[0] - z["xS_new"][k]))
        assert not (fl & oracle.NR_FAILED)
        n_active += bool(fl & oracle.NR_CONVERGED)
    # most rows are return-map updates; the rest are elastic steps of a Gauss
    # point whose predecessor lies further back than the 16-row filter
    assert n_active > 1500, n_active
    # data1.dat prints 17 significant digits; F is O(100)
    assert worst_F < 1e-9, worst_F
    assert worst_x < 1e-11, worst_x


def test_data1_envelope(oracle):
    with open(os.path.join(GOLD, "data1_envelope.json")) as fh:
        env = json.load(fh)
    assert env["F_max"] <= env["Rf_AS"]
    assert -1e-12 <= env["xS_min"] and env["xS_max"] <= 1.0
    assert env["transitions_within_1e9"] == env["transitions"]


def test_eigen_solver_matches_lapack(oracle):
    rng = np.random.default_rng(1)
    for _ in range(200):
        A = rng.normal(size=(3, 3))
        A = A @ A.T + np.eye(3) * rng.uniform(0, 2)
        w, Q, fail = oracle.dsyevq3(colmajor(A))
        assert fail == 0
        Qm = Q.T  # back to row-major
        np.testing.assert_allclose(np.sort(w), np.linalg.eigvalsh(A), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(Qm @ np.diag(w) @ Qm.T, A, atol=1e-12)
        d, V = oracle.eigsrt(w, Q.reshape(9))
        assert d[0] >= d[1] >= d[2]


def test_eigen_degenerate(oracle):
    for A in (np.eye(3), np.diag([2.0, 1.0, 1.0]), np.diag([1.0 + 1e-14, 1.0, 1.0])):
        w, Q, fail = oracle.dsyevq3(colmajor(A))
        assert fail == 0
        np.testing.assert_allclose(np.sort(w), np.linalg.eigvalsh(A), atol=1e-14)


NITI = np.array([60000.0, 0.33, 0.05 * np.sqrt(1.5), 400, 500, 0, 0, 0, 0, 250, 150, 0, 0, 0, 0, 0, 0, 0])


def test_elastic_response(oracle):
    """Below the AS start stress: tau = K theta I + 2G dev(ln V)."""
    E, nu = NITI[0], NITI[1]
    K, G = E / (3 - 6 * nu), E / (2 + 2 * nu)
    R = rot(0.5, 0.2, -0.4)
    U = R @ np.diag([1.003, 0.999, 0.9985]) @ R.T
    Qr = rot(0.1, 0.9, 0.3)
    F = Qr @ U
    tau, s, fl = oracle.law160_kirchhoff(NITI, colmajor(F), [0, 0, 0])
    lnV = Qr @ R @ np.diag(np.log([1.003, 0.999, 0.9985])) @ R.T @ Qr.T
    th = np.trace(lnV)
    expect = K * th * np.eye(3) + 2 * G * (lnV - th / 3 * np.eye(3))
    np.testing.assert_allclose(tau.reshape(3, 3).T, expect, atol=1e-9 * np.abs(expect).max())
    assert fl == oracle.NR_NONE and s[0] == 0


def test_transformation_onset_and_plateau(oracle):
    """AS starts when 2G|e| exceeds Rs_AS; along a monotone path the linear
    flow rule keeps xS = (F - F_first)/(Rf - F_first) step by step, i.e. the
    discrete update is exact: xS - xS0 = (F - F0)(1 - xS)/(Rf - F)."""
    E, nu, eL = NITI[0], NITI[1], NITI[2]
    G = E / (2 + 2 * nu)
    aux = np.sqrt(2 / 3)
    Rs, Rf = 400 * aux, 500 * aux
    en_onset = Rs / (2 * G)
    _, s, fl = oracle.law160_kirchhoff(NITI, colmajor(F_from_enorm(en_onset * (1 - 1e-9))), [0, 0, 0])
    assert fl == oracle.NR_NONE
    sdv = np.array([0.0, 2 * G * en_onset * (1 - 1e-9), 2 * G * en_onset * (1 - 1e-9)])
    first = True
    for en in np.linspace(en_onset * (1 + 1e-6), en_onset + 0.9 * eL, 400):
        x0, F0 = sdv[0], sdv[1]
        _, sdv, fl = oracle.law160_kirchhoff(NITI, colmajor(F_from_enorm(en)), sdv)
        assert fl & oracle.NR_CONVERGED
        F = sdv[1]
        assert F < Rf
        if not first:
            # exact discrete flow rule (converged to the NR tolerance)
            lhs = sdv[0] - x0
            rhs = (F - F0) * (1 - sdv[0]) / (Rf - F)
            assert abs(lhs - rhs) < 1e-8
        first = False
    # plateau: F stays between Rs and Rf, xS in (0,1)
    assert Rs < sdv[1] < Rf and 0 < sdv[0] < 1


def test_reverse_transformation_and_full_strain(oracle):
    E, nu, eL = NITI[0], NITI[1], NITI[2]
    G = E / (2 + 2 * nu)
    aux = np.sqrt(2 / 3)
    # fully transformed state loaded above Rf_AS, then unloaded elastically
    en = eL + 550 * aux / (2 * G)
    sdv = np.array([1.0, 2 * G * (en - eL), 2 * G * (en - eL)])
    _, s1, fl = oracle.law160_kirchhoff(NITI, colmajor(F_from_enorm(en * 0.999)), sdv)
    assert fl == oracle.NR_NONE and s1[0] == 1.0        # elastic unloading of martensite
    np.testing.assert_allclose(s1[1], 2 * G * (0.999 * en - eL), rtol=1e-12)
    # below Rs_SA the reverse transformation starts and xS decreases
    en2 = eL + 240 * aux / (2 * G)
    _, s2, fl = oracle.law160_kirchhoff(NITI, colmajor(F_from_enorm(en2)), s1)
    assert fl & oracle.NR_CONVERGED and s2[0] < 1.0
    Rf_SA = 150 * aux
    assert s2[1] > Rf_SA


def test_float_instance_elastic_close(oracle):
    """All-FP32 restatement: fine in the elastic range."""
    F = F_from_enorm(0.005, 0.002, rot(0.2, 0.3, 0.4))
    t64, s64, f64 = oracle.law160_kirchhoff(NITI, colmajor(F), [0, 0, 0])
    t32, s32, f32 = oracle.law160_kirchhoff(NITI, colmajor(F), [0, 0, 0], dtype=np.float32)
    assert f64 == f32 == oracle.NR_NONE
    assert np.max(np.abs(t32 - t64)) < 1e-4 * np.max(np.abs(t64))


def test_float_instance_return_map_cannot_converge(oracle):
    """The reference's absolute NR tolerance (1e-8, sld_stress_model_160.f90:253)
    is below FP32 resolution of a residual of size |F| * dxS, so an all-FP32
    law resets every transforming point (WARNING 2).  This is why the FP32
    GPU form runs the scalar return map in FP64."""
    F = F_from_enorm(0.01, 0.002, rot(0.2, 0.3, 0.4))
    _, s64, f64 = oracle.law160_kirchhoff(NITI, colmajor(F), [0, 0, 0])
    _, s32, f32 = oracle.law160_kirchhoff(NITI, colmajor(F), [0, 0, 0], dtype=np.float32)
    assert f64 & oracle.NR_CONVERGED and s64[0] > 0.1
    assert f32 & oracle.NR_FAILED and s32[0] == 0.0


def test_return_map_single_newton_step(oracle):
    """With the linear flow rule the residual is linear in xS (the xS^2 terms
    cancel), so the return map lands on the closed-form root
    xS = ((A-Rf) xS0 - (A-F0)) / ((F0-Rf) - G1 (1-xS0)) for AS loading."""
    E, nu, eL = NITI[0], NITI[1], NITI[2]
    G = E / (2 + 2 * nu)
    aux = np.sqrt(2 / 3)
    Rf = 500 * aux
    G1 = 2 * G * eL
    Rs = 400 * aux
    for x0, delta in ((0.0, 0.0003), (0.05, 0.0004), (0.3, 0.0006), (0.6, 0.001)):
        en = eL * x0 + Rs / (2 * G) + delta
        A = 2 * G * en
        F0 = 2 * G * (en - 0.0004 - eL * x0)
        _, s, fl = oracle.law160_kirchhoff(NITI, colmajor(F_from_enorm(en)), [x0, F0, F0])
        assert fl & oracle.NR_CONVERGED
        x = ((A - Rf) * x0 - (A - F0)) / ((F0 - Rf) - G1 * (1 - x0))
        assert abs(s[0] - min(max(x, 0.0), 1.0)) < 1e-12
