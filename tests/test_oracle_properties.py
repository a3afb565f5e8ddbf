"""Physical properties law 160 has by construction, checked on the oracle
(sld_stress_model_160.f90's algorithm restated): the Kirchhoff stress is
symmetric, zero in the undeformed austenite, frame indifferent
(tau(R F) = R tau(F) R^T with the same state update), and isotropic in the
reference configuration (tau(F R) = tau(F))."""
import numpy as np
import pytest

from alya_sma_b200 import problem as P

NITI = P.nitinol_props(**P.NITI)


def _rotation(rng):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] *= -1
    return q


def _tau(oracle, F, sdv):
    t, s, fl = oracle.law160_kirchhoff(NITI, np.ascontiguousarray(F.T).reshape(9), sdv)
    return t.reshape(3, 3).T, s, fl


def _states(rng, n):
    """Deformations with their previous states, elastic and transforming."""
    out = []
    for k in range(n):
        e = [0.002, 0.03, 0.06][k % 3] * rng.uniform(0.7, 1.0)
        U = _rotation(rng) @ np.diag([1 + e, 1 - 0.3 * e, 1 - 0.3 * e]) @ _rotation(rng).T
        U = 0.5 * (U + U.T)
        x0 = [0.0, 0.0, 0.4][k % 3]
        out.append((U, [x0, 0.0, 0.0]))
    return out


def test_zero_stress_in_the_undeformed_austenite(oracle):
    t, s, fl = _tau(oracle, np.eye(3), [0.0, 0.0, 0.0])
    assert np.abs(t).max() == 0.0 and fl == 0 and s[0] == 0.0


@pytest.mark.parametrize("seed", [0, 1])
def test_symmetric_and_frame_indifferent(oracle, seed):
    rng = np.random.default_rng(seed)
    for U, sdv in _states(rng, 30):
        t, s, fl = _tau(oracle, U, list(sdv))
        scale = max(np.abs(t).max(), 1.0)
        assert np.abs(t - t.T).max() <= 1e-12 * scale
        R = _rotation(rng)
        tr, sr, flr = _tau(oracle, R @ U, list(sdv))               # spatial rotation
        assert flr == fl
        assert np.abs(tr - R @ t @ R.T).max() <= 1e-8 * scale
        assert abs(sr[0] - s[0]) <= 1e-9


@pytest.mark.parametrize("seed", [2, 3])
def test_isotropic_in_the_reference_configuration(oracle, seed):
    """tau depends on F only through b = F F^T, so a rotation of the
    reference configuration (F R) changes nothing."""
    rng = np.random.default_rng(seed)
    for U, sdv in _states(rng, 30):
        t, s, fl = _tau(oracle, U, list(sdv))
        scale = max(np.abs(t).max(), 1.0)
        tq, sq, flq = _tau(oracle, U @ _rotation(rng), list(sdv))
        assert flq == fl
        assert np.abs(tq - t).max() <= 1e-8 * scale
        assert abs(sq[0] - s[0]) <= 1e-9
