"""Problem description for the explicit SMA step: mesh, materials, boundary
conditions and time functions, in the reference's own terms.

The fields mirror what Alya's solidz reads from its input decks:

* ``props`` rows are the NITINOL parameter vector ``parco_sld(1:18)`` in the
  order the law reads it (``sld_stress_model_160.f90:263-279``):
  ``[E, nu, eL, Ss_AS, Sf_AS, C_AS, Tf_AS, Ts_AS, Sn_AS, Ss_SA, Sf_SA, C_SA,
  Tf_SA, Ts_SA, alpha, B_AS, B_SA, (unused)]``; a deck line
  ``CONSTITUTIVE_MODEL: NITINOL ...`` pastes into a row directly
  (``sld_reaphy.f90:477-489``).
* ``densi`` is the density after ``MASS_SCALING`` (``sld_reanut.f90:361-362``).
* ``fixno`` holds the per-dof fixity codes ``kfl_fixno_sld`` (1 = prescribed).
* time functions are ``DISCRETE`` tables ``tload_sld(ifunc)%a(ndime+1, n)``
  stored row-wise as ``(time, v_x, v_y, v_z)`` with the ``SMOOTH`` flag
  (``sld_reabcs.f90:606-640``, evaluated as ``sld_funbou.f90:99-140``).

Extensions with no reference counterpart (the reference law has one Young's
modulus and hard-wires the temperature to zero, ``sld_stress_model_160.f90:105``):
``e_mart`` (martensite modulus, Reuss-mixed at the start-of-step martensite
fraction) and ``tempe`` (per-element temperature fed to the loading function).
``e_mart == props[:,0]`` and ``tempe is None`` give the reference law.

Meshes are structured HEX08 boxes (node numbering of ``mod_lagrange.f90:935-977``)
and HEX08 O-grid cylinders, with seeded interior-node jitter.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SQRT_2_3 = np.sqrt(2.0 / 3.0)
SQRT_3_2 = np.sqrt(1.5)


def nitinol_props(E, nu, eps_L, Ss_AS, Sf_AS, Ss_SA, Sf_SA, C_AS=0.0, C_SA=0.0,
                  T_ref=0.0, alpha=0.0, B_AS=0.0, B_SA=0.0):
    """18-entry NITINOL parameter vector from uniaxial engineering data.

    ``eps_L`` is the uniaxial maximum transformation strain; the law's ``eL`` is
    the norm of the deviatoric transformation strain, ``eL = eps_L*sqrt(3/2)``.
    Transformation stresses are uniaxial: the law multiplies them by
    ``sqrt(2/3)`` (``sld_stress_model_160.f90:284-288``) to compare with the
    deviatoric Kirchhoff norm.  ``C_*`` are per-kelvin slopes in the law's
    deviatoric units; the thresholds shift by ``C*(T - T_ref)`` when the start
    and finish temperatures are set to ``-T_ref``.
    """
    p = np.zeros(18)
    p[0], p[1], p[2] = E, nu, eps_L * SQRT_3_2
    p[3], p[4], p[5], p[6], p[7] = Ss_AS, Sf_AS, C_AS, -T_ref, -T_ref
    p[9], p[10], p[11], p[12], p[13] = Ss_SA, Sf_SA, C_SA, -T_ref, -T_ref
    p[14], p[15], p[16] = alpha, B_AS, B_SA
    return p


# Material of the 40x4x4 bar and the 400x40x40 cantilever: NiTi with
# E_A = 60 GPa, E_M = 40 GPa, nu = 0.33, eps_L = 0.05, AS 400/500 MPa,
# SA 250/150 MPa, rho = 6450 kg/m^3 (units mm, MPa, tonne/mm^3, s).
NITI = dict(E=60000.0, nu=0.33, eps_L=0.05, Ss_AS=400.0, Sf_AS=500.0,
            Ss_SA=250.0, Sf_SA=150.0)
NITI_E_MART = 40000.0
NITI_DENSITY = 6.45e-9


@dataclass
class Problem:
    coord: np.ndarray                 # (npoin, 3) float64
    lnods: np.ndarray                 # (nelem, 8) int32, 0-based
    props: np.ndarray                 # (nmate, 18)
    e_mart: np.ndarray                # (nmate,)
    densi: np.ndarray                 # (nmate,)
    fixno: np.ndarray                 # (npoin, 3) int32
    bcfun: np.ndarray                 # (npoin,) int32, -1 = value 0
    fun_npts: np.ndarray              # (nfun,) int32
    fun_smooth: np.ndarray            # (nfun,) int32
    fun_tab: np.ndarray               # (sum npts, 4) rows (t, vx, vy, vz)
    lmate: np.ndarray | None = None   # (nelem,) int32 material id
    tempe: np.ndarray | None = None   # (nelem,) temperature (extension)
    fext: np.ndarray | None = None    # (npoin, 3) nodal load at load factor 1
    dampi: np.ndarray | None = None   # (nmate, 2) Rayleigh (alpha, beta) per material
    load_fun: int = -1                # table scaling fext (column v_x)
    dtime: float = 0.0                # time step (0: not chosen yet)
    nsteps: int = 0
    name: str = ""
    info: dict = field(default_factory=dict)

    @property
    def nelem(self):
        return self.lnods.shape[0]

    @property
    def npoin(self):
        return self.coord.shape[0]

    def fun_table(self, ifun):
        off = int(np.sum(self.fun_npts[:ifun]))
        return self.fun_tab[off: off + int(self.fun_npts[ifun])]


# --------------------------------------------------------------------------
# meshes
# --------------------------------------------------------------------------

def structured_box(nx, ny, nz, lx, ly, lz, jitter=0.0, seed=0):
    """HEX08 box [0,lx]x[0,ly]x[0,lz]; node id = i + (nx+1)*(j + (ny+1)*k).

    Interior nodes move by U(-jitter, jitter)*h per direction (h = spacing in
    that direction), drawn from ``numpy.random.default_rng(seed)``."""
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    i = np.arange(nx + 1)
    j = np.arange(ny + 1)
    k = np.arange(nz + 1)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    coord = np.stack([I * hx, J * hy, K * hz], axis=-1).reshape(-1, 3).astype(np.float64)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        interior = ((I > 0) & (I < nx) & (J > 0) & (J < ny) & (K > 0) & (K < nz)).reshape(-1)
        d = rng.uniform(-jitter, jitter, size=(coord.shape[0], 3)) * np.array([hx, hy, hz])
        coord[interior] += d[interior]
    ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ei, ej, ek = (a.transpose(2, 1, 0).reshape(-1) for a in (ei, ej, ek))
    def nid(a, b, c):
        return a + (nx + 1) * (b + (ny + 1) * c)
    lnods = np.stack([nid(ei, ej, ek), nid(ei + 1, ej, ek), nid(ei + 1, ej + 1, ek),
                      nid(ei, ej + 1, ek), nid(ei, ej, ek + 1), nid(ei + 1, ej, ek + 1),
                      nid(ei + 1, ej + 1, ek + 1), nid(ei, ej + 1, ek + 1)], axis=1)
    return coord, lnods.astype(np.int32)


def ogrid_cylinder(radius, length, n_core, n_ring, n_axial, jitter=0.0, seed=0):
    """HEX08 O-grid cylinder along x: a square core block of n_core x n_core
    cells (half-width radius/2) wrapped by four ring blocks of n_core x n_ring
    cells that blend from the core square to the circle.  Interior nodes
    (not on the lateral surface or the end faces) are jittered by
    U(-jitter, jitter) times the local spacing."""
    nc, nr = n_core, n_ring
    a = 0.5 * radius  # half-width of the square core block
    # 2-D cross-section nodes and quads --------------------------------------
    pts = {}
    quads = []
    def key_core(i, j):
        return ("c", i, j)
    # core lattice (nc+1)^2
    for j in range(nc + 1):
        for i in range(nc + 1):
            pts[key_core(i, j)] = (-a + 2 * a * i / nc, -a + 2 * a * j / nc)
    # boundary of the core square, counter-clockwise, 4*nc points
    ring_keys = []
    for i in range(nc):
        ring_keys.append(key_core(i, 0))
    for j in range(nc):
        ring_keys.append(key_core(nc, j))
    for i in range(nc, 0, -1):
        ring_keys.append(key_core(i, nc))
    for j in range(nc, 0, -1):
        ring_keys.append(key_core(0, j))
    nb = len(ring_keys)
    for m, kk in enumerate(ring_keys):
        x0, y0 = pts[kk]
        ang = np.arctan2(y0, x0)
        xc, yc = radius * np.cos(ang), radius * np.sin(ang)
        for r in range(1, nr + 1):
            t = r / nr
            pts[("r", m, r)] = ((1 - t) * x0 + t * xc, (1 - t) * y0 + t * yc)
    for j in range(nc):
        for i in range(nc):
            quads.append((key_core(i, j), key_core(i + 1, j), key_core(i + 1, j + 1), key_core(i, j + 1)))
    for m in range(nb):
        m1 = (m + 1) % nb
        for r in range(nr):
            k00 = ring_keys[m] if r == 0 else ("r", m, r)
            k10 = ring_keys[m1] if r == 0 else ("r", m1, r)
            # counter-clockwise in (y, z): outward first, then along the ring
            quads.append((k00, ("r", m, r + 1), ("r", m1, r + 1), k10))
    keys = list(pts.keys())
    index = {kk: n for n, kk in enumerate(keys)}
    xy = np.array([pts[kk] for kk in keys], dtype=np.float64)
    q = np.array([[index[kk] for kk in qu] for qu in quads], dtype=np.int64)
    outer = np.array([kk[0] == "r" and kk[2] == nr for kk in keys])
    n2 = xy.shape[0]
    # local spacing per 2-D node: shortest incident quad edge
    h2 = np.full(n2, np.inf)
    for e in range(4):
        p0, p1 = q[:, e], q[:, (e + 1) % 4]
        d = np.linalg.norm(xy[p0] - xy[p1], axis=1)
        np.minimum.at(h2, p0, d)
        np.minimum.at(h2, p1, d)
    # extrude along x ---------------------------------------------------------
    hx = length / n_axial
    xs = np.arange(n_axial + 1) * hx
    coord = np.zeros(((n_axial + 1) * n2, 3))
    coord[:, 0] = np.repeat(xs, n2)
    coord[:, 1] = np.tile(xy[:, 0], n_axial + 1)
    coord[:, 2] = np.tile(xy[:, 1], n_axial + 1)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        lay = np.repeat(np.arange(n_axial + 1), n2)
        interior = (~np.tile(outer, n_axial + 1)) & (lay > 0) & (lay < n_axial)
        hloc = np.tile(h2, n_axial + 1)
        d = rng.uniform(-jitter, jitter, size=coord.shape)
        d[:, 0] *= hx
        d[:, 1] *= hloc
        d[:, 2] *= hloc
        coord[interior] += d[interior]
    nq = q.shape[0]
    lay = np.repeat(np.arange(n_axial), nq)
    qq = np.tile(q, (n_axial, 1))
    # quad (p0..p3) counter-clockwise in (y,z); the brick's local s runs along
    # x, so order nodes so that det J > 0: bottom face at x_k, top at x_{k+1}
    b0 = qq + (lay * n2)[:, None]
    b1 = qq + ((lay + 1) * n2)[:, None]
    # local axes: s = x (layer), t = quad edge p0->p1, z = edge p0->p3
    lnods = np.stack([b0[:, 0], b1[:, 0], b1[:, 1], b0[:, 1],
                      b0[:, 3], b1[:, 3], b1[:, 2], b0[:, 2]], axis=1).astype(np.int32)
    return coord, lnods


# --------------------------------------------------------------------------
# boundary helpers
# --------------------------------------------------------------------------

def face_nodes(coord, axis, value, tol=1e-9):
    return np.nonzero(np.abs(coord[:, axis] - value) <= tol * max(1.0, abs(value)))[0]


def face_load(coord, lnods, axis, value, traction):
    """Consistent nodal forces of a uniform traction vector on the mesh faces
    lying in the plane coord[axis] == value (2x2 Gauss on each bilinear quad)."""
    on = np.zeros(coord.shape[0], bool)
    on[face_nodes(coord, axis, value)] = True
    faces = [(0, 3, 2, 1), (1, 2, 6, 5), (4, 5, 6, 7), (3, 0, 4, 7), (0, 1, 5, 4), (2, 3, 7, 6)]
    f = np.zeros_like(coord)
    g = np.array([-1.0, 1.0]) / np.sqrt(3.0)
    for fc in faces:
        nodes = lnods[:, fc]
        sel = on[nodes].all(axis=1)
        if not sel.any():
            continue
        X = coord[nodes[sel]]                     # (nf, 4, 3)
        for s in g:
            for t in g:
                N = 0.25 * np.array([(1 - s) * (1 - t), (1 + s) * (1 - t), (1 + s) * (1 + t), (1 - s) * (1 + t)])
                dNs = 0.25 * np.array([-(1 - t), (1 - t), (1 + t), -(1 + t)])
                dNt = 0.25 * np.array([-(1 - s), -(1 + s), (1 + s), (1 - s)])
                xs = np.einsum("a,fai->fi", dNs, X)
                xt = np.einsum("a,fai->fi", dNt, X)
                dA = np.linalg.norm(np.cross(xs, xt), axis=1)
                contrib = (N[None, :, None] * dA[:, None, None]) * np.asarray(traction)[None, None, :]
                np.add.at(f, nodes[sel], contrib)
    return f


def smooth_cycle_table(t_total, peak, t_peak=None):
    """Table 0 -> peak (at t_peak, default half) -> 0 with SMOOTH steps;
    the value goes into column v_x (and is reused by every direction)."""
    tp = 0.5 * t_total if t_peak is None else t_peak
    return np.array([[0.0, 0.0, 0.0, 0.0], [tp, peak, peak, peak], [t_total, 0.0, 0.0, 0.0]])


def critical_dt(coord, lnods, props, densi, lmate=None):
    """Stable time step dt_crit = min_e h_min(e) / c (c for law 160 from
    lambda + 2 mu), with h_min the smallest element length at the centre
    (elmlen.f90 with natural length 2).  Vectorised host version."""
    X = coord[lnods]                                       # (ne, 8, 3)
    sgn = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
    dercg = 0.125 * sgn                                    # dN/dxi at the centre
    J = np.einsum("eai,aj->eij", X, dercg)                 # xjacm(i,j)
    Jinv = np.linalg.inv(J)
    enor = np.sum(Jinv ** 2, axis=2)                       # rows of tragl
    hmin = np.min(2.0 / np.sqrt(enor), axis=1)
    props = np.atleast_2d(props)
    im = np.zeros(lnods.shape[0], np.int64) if lmate is None else lmate
    E, nu = props[im, 0], props[im, 1]
    lame1 = nu * E / ((1 + nu) * (1 - 2 * nu))
    lame2 = E / (2 * (1 + nu))
    c = np.sqrt((lame1 + 2 * lame2) / np.atleast_1d(densi)[im])
    return float(np.min(hmin / c))


def prestrain(prob, eps, nu_eff=0.45):
    """Axial prestrain along x with lateral contraction nu_eff about the
    cross-section centre, compatible with the prescribed dofs (their tables
    start at 0): a uniform strain eps when the x = max end is free, and
    u_x = eps L s (1 - s), s = (x - x_min) / L, when that end is held too
    (strain from +eps to -eps, zero displacement at both ends; a uniform
    field there would crush the last element layer).  Used to start a timed
    run on the transformation plateau, where Gauss points run the return map."""
    X = prob.coord
    x0, L = X[:, 0].min(), X[:, 0].max() - X[:, 0].min()
    s = (X[:, 0] - x0) / L
    yc = 0.5 * (X[:, 1].min() + X[:, 1].max())
    zc = 0.5 * (X[:, 2].min() + X[:, 2].max())
    far = np.isclose(s, 1.0)
    held = bool(np.any(prob.fixno[far, 0] == 1))
    if held:
        ux, ex = eps * L * s * (1.0 - s), eps * (1.0 - 2.0 * s)
    else:
        ux, ex = eps * L * s, np.full_like(s, eps)
    u = np.stack([ux, -nu_eff * ex * (X[:, 1] - yc), -nu_eff * ex * (X[:, 2] - zc)], axis=1)
    u[prob.fixno == 1] = 0.0
    return u


def _niti_material(ref_equivalent=False):
    props = nitinol_props(**NITI)[None, :]
    e_mart = props[:, 0].copy() if ref_equivalent else np.array([NITI_E_MART])
    return props, e_mart, np.array([NITI_DENSITY])


# --------------------------------------------------------------------------
# named workloads
# --------------------------------------------------------------------------

def bar_40x4x4(nsteps=4000, seed=0, ref_equivalent=False, scale=1):
    """Uniaxial NiTi bar 40x4x4 mm, HEX08 (40x4x4)*scale elements, interior
    jitter U(-0.05,0.05)h.  x=0 clamped; the x=40 face is displaced along x by
    a smooth ramp to 6 % strain (2.4 mm) and back over nsteps steps of
    dt = 0.5 * dt_crit (central difference)."""
    coord, lnods = structured_box(40 * scale, 4 * scale, 4 * scale, 40.0, 4.0, 4.0, 0.05, seed)
    props, e_mart, densi = _niti_material(ref_equivalent)
    npoin = coord.shape[0]
    fixno = np.zeros((npoin, 3), np.int32)
    bcfun = np.full(npoin, -1, np.int32)
    x0 = face_nodes(coord, 0, 0.0)
    xl = face_nodes(coord, 0, 40.0)
    fixno[x0] = 1
    fixno[xl, 0] = 1
    bcfun[xl] = 0
    dt = 0.5 * critical_dt(coord, lnods, props, densi)
    tab = smooth_cycle_table(nsteps * dt, 0.06 * 40.0)
    return Problem(coord=coord, lnods=lnods, props=props, e_mart=e_mart, densi=densi,
                   fixno=fixno, bcfun=bcfun, fun_npts=np.array([3], np.int32),
                   fun_smooth=np.array([1], np.int32), fun_tab=tab, dtime=dt, nsteps=nsteps,
                   name="bar_40x4x4" + ("" if scale == 1 else f"_x{scale}"),
                   info=dict(mesh=f"{40*scale}x{4*scale}x{4*scale}", ref_equivalent=ref_equivalent))


def cylinder_2m(nsteps=10000, seed=0, div=1, spread=0.10, t_range=(300.0, 320.0), layers=None):
    """NiTi cylinder r = 5 mm, L = 50 mm, HEX08 O-grid: a 32x32 core block and
    four 32x24 ring blocks per cross-section (4,096 cells), 488 layers
    (1,998,848 elements at div=1; every count divided by div).  Interior nodes
    jittered U(-0.1,0.1)h.  Every element gets its own material: E_A, E_M,
    eps_L and the four transformation stresses scaled by U(1-spread, 1+spread)
    from numpy.random.default_rng(seed).  Temperature rises linearly from
    t_range[0] at x = 0 to t_range[1] at x = L; the transformation stresses
    shift by 6.5 MPa/K above 300 K (extension: the reference law has no
    temperature).  x = 0 clamped; the x = L face is pushed to -3 % axial strain
    and released with smooth steps over nsteps steps of dt = 0.5 dt_crit.
    layers: that many axial element layers instead, the length shortened so
    the elements keep their size (a smaller case of the same mesh)."""
    nc, nr, nx = max(2, 32 // div), max(1, 24 // div), max(2, 488 // div)
    length = 50.0
    if layers:
        length, nx = 50.0 * layers / nx, int(layers)
    coord, lnods = ogrid_cylinder(5.0, length, nc, nr, nx, jitter=0.1, seed=seed)
    ne, npo = lnods.shape[0], coord.shape[0]
    rng = np.random.default_rng(seed + 1)
    base = nitinol_props(**NITI, C_AS=6.5 * SQRT_2_3, C_SA=6.5 * SQRT_2_3, T_ref=300.0)
    props = np.tile(base, (ne, 1))
    f = rng.uniform(1.0 - spread, 1.0 + spread, size=(ne, 7))
    props[:, 0] *= f[:, 0]
    props[:, 2] *= f[:, 1]
    props[:, 3] *= f[:, 2]
    props[:, 4] *= f[:, 3]
    props[:, 9] *= f[:, 4]
    props[:, 10] *= f[:, 5]
    e_mart = NITI_E_MART * f[:, 6]
    densi = np.full(ne, NITI_DENSITY)
    xc = coord[lnods].mean(axis=1)[:, 0]
    tempe = t_range[0] + (t_range[1] - t_range[0]) * xc / length
    fixno = np.zeros((npo, 3), np.int32)
    bcfun = np.full(npo, -1, np.int32)
    x0 = face_nodes(coord, 0, 0.0)
    xl = face_nodes(coord, 0, length)
    fixno[x0] = 1
    fixno[xl, 0] = 1
    bcfun[xl] = 0
    lmate = np.arange(ne, dtype=np.int32)
    # E_M (at most 44 GPa here) stays below E_A (at least 54 GPa): E_A sets c
    dt = 0.5 * critical_dt(coord, lnods, props, densi, lmate)
    tab = smooth_cycle_table(nsteps * dt, -0.03 * length)
    return Problem(coord=coord, lnods=lnods, props=props, e_mart=e_mart, densi=densi,
                   fixno=fixno, bcfun=bcfun, fun_npts=np.array([3], np.int32),
                   fun_smooth=np.array([1], np.int32), fun_tab=tab, lmate=lmate, tempe=tempe,
                   dtime=dt, nsteps=nsteps, name=f"cylinder_ogrid_{ne}",
                   info=dict(mesh=f"O-grid core {nc}x{nc}, ring {nr}, {nx} layers", elements=ne))


def ensemble_sizes(nspec=256, seed=0, emin=1000, emax=50000):
    """Element counts of the ensemble's specimens (10 k^3 for k = round((n/10)^(1/3)),
    n drawn log-uniform in [emin, emax])."""
    rng = np.random.default_rng(seed)
    n_target = np.exp(rng.uniform(np.log(emin), np.log(emax), size=nspec))
    k = np.maximum(2, np.round((n_target / 10.0) ** (1.0 / 3.0)).astype(int))
    return 10 * k ** 3


def ensemble(nspec=256, nsteps=5000, seed=0, emin=1000, emax=50000, spread=0.15, subset=None,
             by_size=False):
    """Batched ensemble: nspec independent NiTi specimens (10:1:1 bars, 1 mm
    elements) with element counts drawn log-uniform in [emin, emax] and every
    specimen's E_A, E_M, eps_L and transformation stresses scaled by
    U(1-spread, 1+spread).  Specimens are concatenated into one mesh (disjoint
    node ranges), so one element launch and one step graph cover all of them.
    Each is clamped at its x = 0 face and pulled by an axial tip traction of
    its own amplitude (0.8 to 1.5 times its forward-finish stress) through a
    shared smooth load cycle; one dt (0.5 dt_crit of the stiffest specimen).
    `subset` (specimen ids) builds only those specimens -- each specimen's
    random numbers come from its own stream, so a subset is identical to the
    same specimens of the full ensemble (used to shard across GPUs).
    by_size concatenates the specimens in increasing size (stable), so each
    size bucket is one contiguous element range (`size_buckets`)."""
    sizes = ensemble_sizes(nspec, seed, emin, emax)
    ids = list(range(nspec)) if subset is None else [int(v) for v in subset]
    if by_size:
        ids = sorted(ids, key=lambda s: (sizes[s], s))
    coords, lnods_l, props_l, em_l, fixno_l, fext_l, spec_of = [], [], [], [], [], [], []
    off = 0
    base = nitinol_props(**NITI)
    for local, s in enumerate(ids):
        rng = np.random.default_rng((seed, s))
        k = int(round((sizes[s] / 10) ** (1.0 / 3.0)))
        nx, ny = 10 * k, k
        c, l = structured_box(nx, ny, ny, float(nx), float(ny), float(ny), 0.05, seed + 100 + s)
        f = rng.uniform(1.0 - spread, 1.0 + spread, size=7)
        pr = base.copy()
        pr[0] *= f[0]; pr[2] *= f[1]; pr[3] *= f[2]; pr[4] *= f[3]; pr[9] *= f[4]; pr[10] *= f[5]
        props_l.append(pr)
        em_l.append(NITI_E_MART * f[6])
        fx = np.zeros((c.shape[0], 3), np.int32)
        fx[face_nodes(c, 0, 0.0)] = 1
        amp = rng.uniform(0.8, 1.5) * pr[4]
        fe = face_load(c, l, 0, float(nx), (amp, 0.0, 0.0))
        coords.append(c)
        lnods_l.append(l + off)
        fixno_l.append(fx)
        fext_l.append(fe)
        spec_of.append(np.full(l.shape[0], local, np.int32))
        off += c.shape[0]
    coord = np.concatenate(coords)
    lnods = np.concatenate(lnods_l).astype(np.int32)
    lmate = np.concatenate(spec_of)
    props = np.array(props_l)
    e_mart = np.array(em_l)
    densi = np.full(len(ids), NITI_DENSITY)
    fixno = np.concatenate(fixno_l)
    fext = np.concatenate(fext_l)
    dt = 0.5 * critical_dt(coord, lnods, props, densi, lmate)
    tab = smooth_cycle_table(nsteps * dt, 1.0)
    return Problem(coord=coord, lnods=lnods, props=props, e_mart=e_mart, densi=densi,
                   fixno=fixno, bcfun=np.full(coord.shape[0], -1, np.int32),
                   fun_npts=np.array([3], np.int32), fun_smooth=np.array([1], np.int32),
                   fun_tab=tab, lmate=lmate, fext=fext, load_fun=0, dtime=dt, nsteps=nsteps,
                   name=f"ensemble_{nspec}", info=dict(specimens=len(ids), ids=ids,
                                                       elements=int(lnods.shape[0]),
                                                       sizes=[int(v) for v in np.bincount(lmate)]))


def size_buckets(prob):
    """Contiguous element ranges of an ensemble built with by_size=True, one
    per specimen-size bucket (the element count rounded down to a power of
    two): [(elements per specimen of the bucket's smallest, end element)]."""
    sizes = prob.info["sizes"]                               # elements of each local specimen, in order
    out, end = [], 0
    cur = None
    for n in sizes:
        b = 1 << int(np.floor(np.log2(n)))
        if cur is not None and b != cur:
            out.append((cur, end))
        cur = b
        end += n
    out.append((cur, end))
    return out


def cantilever_400x40x40(nsteps=20000, seed=0, ref_equivalent=False, div=1):
    """NiTi cantilever 400x40x40 mm, HEX08 (400x40x40)/div elements, jitter
    U(-0.05,0.05)h, clamped at x=0, uniform axial tip traction on x=L cycled
    0 -> 1.5*Sf_AS (750 MPa) -> 0 with smooth steps over nsteps steps of
    dt = 0.5 * dt_crit."""
    nx, ny, nz = 400 // div, 40 // div, 40 // div
    coord, lnods = structured_box(nx, ny, nz, 400.0, 40.0, 40.0, 0.05, seed)
    props, e_mart, densi = _niti_material(ref_equivalent)
    npoin = coord.shape[0]
    fixno = np.zeros((npoin, 3), np.int32)
    fixno[face_nodes(coord, 0, 0.0)] = 1
    bcfun = np.full(npoin, -1, np.int32)
    fext = face_load(coord, lnods, 0, 400.0, (1.0, 0.0, 0.0))
    dt = 0.5 * critical_dt(coord, lnods, props, densi)
    tab = smooth_cycle_table(nsteps * dt, 1.5 * NITI["Sf_AS"])
    return Problem(coord=coord, lnods=lnods, props=props, e_mart=e_mart, densi=densi,
                   fixno=fixno, bcfun=bcfun, fun_npts=np.array([3], np.int32),
                   fun_smooth=np.array([1], np.int32), fun_tab=tab, fext=fext, load_fun=0,
                   dtime=dt, nsteps=nsteps, name=f"cantilever_{nx}x{ny}x{nz}",
                   info=dict(mesh=f"{nx}x{ny}x{nz}", ref_equivalent=ref_equivalent))
