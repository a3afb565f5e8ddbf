"""Known answers for the oracle's element loop and time-step estimate, which
have no reference-computed golden output: the constant-strain patch test on a
jittered mesh, zero force under a finite rigid motion, lumped mass equal to
rho V, and the critical time step h / c of a regular mesh."""
import numpy as np

from alya_sma_b200 import problem as P


def _interior(p, tol=1e-9):
    X = p.coord
    lo, hi = X.min(axis=0), X.max(axis=0)
    return np.all((X > lo + tol) & (X < hi - tol), axis=1)


def test_patch_test_constant_strain_on_jittered_mesh(oracle):
    """u = G X with G constant: every Gauss point has the same F and stress, so
    the internal force of every interior node vanishes (sum over its elements
    of the integral of grad N_a), however the mesh is distorted."""
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)              # interior nodes jittered 5 %
    rng = np.random.default_rng(3)
    G = rng.normal(size=(3, 3)) * 1e-4                            # elastic, general (non-symmetric)
    u = p.coord @ G.T
    r = oracle.Problem(p).assemble(u)["rhsid"]
    inner = _interior(p)
    assert inner.sum() == 39 * 3 * 3
    scale = np.abs(r).max()
    assert scale > 0.0
    assert np.abs(r[inner]).max() <= 1e-10 * scale


def test_rigid_motion_gives_no_force(oracle):
    """A finite rigid rotation (40 degrees) plus a translation: F = R, b = I,
    no strain, no stress, no force -- the law and the element loop are
    objective."""
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    c, s = np.cos(0.7), np.sin(0.7)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    u = p.coord @ (R - np.eye(3)).T + np.array([3.0, -1.0, 2.0])
    r = oracle.Problem(p).assemble(u)["rhsid"]
    # force scale of a 1e-4 stretch on the same mesh, for comparison
    ref = oracle.Problem(p).assemble(p.coord * np.array([1e-4, 0.0, 0.0]))["rhsid"]
    assert np.abs(r).max() <= 1e-9 * np.abs(ref).max()


def test_lumped_mass_is_rho_times_volume(oracle):
    """Row-sum lumping of rho N_a N_b dV: the masses add up to rho V, and the
    jitter moves only interior nodes, so V is the box volume 40 x 4 x 4."""
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    vmass = oracle.Problem(p).assemble(np.zeros((p.npoin, 3)))["vmass"]
    rho = float(p.densi[0])
    assert abs(vmass.sum() - rho * 640.0) <= 1e-12 * rho * 640.0
    assert (vmass > 0).all()


def test_critical_time_step_is_h_over_c(oracle):
    """On a regular mesh of unit cubes the element length is 1 and
    dt_crit = h / sqrt((lambda + 2 mu) / rho) (mod_sld_minle_time_step.f90:
    262-268, sld_velsnd.f90:117-124)."""
    coord, lnods = P.structured_box(10, 3, 2, 10.0, 3.0, 2.0)
    props, _, densi = P.nitinol_props(**P.NITI), None, np.array([P.NITI_DENSITY])
    E, nu, rho = props[0], props[1], densi[0]
    lam, mu = nu * E / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    dt = oracle.critical_dt(lnods, coord, props.reshape(1, 18), densi)
    assert abs(dt - 1.0 / np.sqrt((lam + 2 * mu) / rho)) <= 1e-14 * dt
