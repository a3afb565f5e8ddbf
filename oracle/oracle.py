"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``; the product package never imports
it.  The C sources restate the reference CPU path of Alya's solidz module with
law 160 (see sma_oracle_impl.h for the file:line of every routine).

Array conventions follow the reference (Fortran column-major):
  * nodal arrays     shape (npoin, 3) C-order  == Fortran (3, npoin)
  * lnods            shape (nelem, 8) int32, 0-based node ids
  * state (svegm)    shape (nelem, 2, 8, 3)     == Fortran (3, 8, 2, nelem);
                     slot 0 = ITER_K (new), slot 1 = TIME_N (old)
  * 3x3 tensors      shape (..., 3, 3) holding Fortran T(i,j) at [..., j, i]
                     (i.e. the flat 9-vector is column-major)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

NR_NONE, NR_CONVERGED, NR_FAILED, NR_BOTH = 0, 1, 2, 4
CNT_NR_ACTIVE, CNT_NR_FAILED, CNT_NR_BOTH, CNT_NEG_DET, CNT_EIG_FAIL, CNT_NONFINITE = range(6)
NCOUNTERS = 8

_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (needs gcc + libgomp)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


NATIVE_PATH = os.path.join(HERE, "liboracle_native.so")
_native_lib = None


def native_lib():
    """The same oracle compiled with -march=native for the machine it runs on
    (the timed CPU baseline): built there by `make native`, since a library
    tuned for one host's instruction set may not run on another's.  Falls
    back to the portable liboracle.so when the build fails; returns
    (library, True if native)."""
    global _native_lib
    if _native_lib is None:
        try:
            subprocess.run(["make", "-s", "-B", "-C", HERE, "native"], check=True,
                           capture_output=True, timeout=300)
            _native_lib = (C.CDLL(NATIVE_PATH), True)
        except (OSError, subprocess.SubprocessError):
            _native_lib = (lib(), False)
    return _native_lib


COUNT_PATH = os.path.join(HERE, "liboracle_count.so")
OPS = ("add", "mul", "div", "cmp", "sqrt", "log", "pow")
_count_lib = None


def count_lib():
    """The oracle on a counting number type (liboracle_count.so)."""
    global _count_lib
    if _count_lib is None:
        if not os.path.exists(COUNT_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(COUNT_PATH)
        L.orc_count_law160.restype = C.c_int
        L.orc_count_law160.argtypes = [C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double), C.c_double,
                                       C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
        L.orc_count_element.restype = C.c_int
        L.orc_count_element.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.c_double, C.c_double, C.POINTER(C.c_double),
                                        C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
        _count_lib = L
    return _count_lib


def count_law160(props, F, sdv, tmp=0.0, e_mart=0.0):
    """Operations of one compute_kirchoff_stress call (F column-major, 9):
    ({op: count}, sdv_new, nr_flag)."""
    p = np.ascontiguousarray(props, dtype=np.float64).reshape(18)
    f = np.ascontiguousarray(F, dtype=np.float64).reshape(9)
    sv = np.array(sdv, dtype=np.float64)
    ops = np.zeros(len(OPS), np.uint64)
    fl = count_lib().orc_count_law160(_ptr(p, C.c_double), float(e_mart), _ptr(f, C.c_double), float(tmp),
                                      _ptr(sv, C.c_double), _ptr(ops, C.c_uint64))
    return dict(zip(OPS, (int(x) for x in ops))), sv, fl


def count_element(elcod, eldis, props, densi, sdv_old, e_mart=0.0):
    """Operations of one HEX08 element of the explicit element loop
    (elcod, eldis (3, 8) column-major as 24; sdv_old (8, 3)):
    ({op: count}, Gauss points that ran the return map)."""
    c = np.ascontiguousarray(elcod, dtype=np.float64).reshape(24)
    u = np.ascontiguousarray(eldis, dtype=np.float64).reshape(24)
    p = np.ascontiguousarray(props, dtype=np.float64).reshape(18)
    so = np.ascontiguousarray(sdv_old, dtype=np.float64).reshape(24)
    ops = np.zeros(len(OPS), np.uint64)
    nr = C.c_int(0)
    count_lib().orc_count_element(_ptr(c, C.c_double), _ptr(u, C.c_double), _ptr(p, C.c_double), float(e_mart),
                                  float(densi), _ptr(so, C.c_double), _ptr(ops, C.c_uint64), C.byref(nr))
    return dict(zip(OPS, (int(x) for x in ops))), nr.value


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _f(dtype):
    return (np.float64, C.c_double, "_f64") if np.dtype(dtype) == np.float64 else (np.float32, C.c_float, "_f32")


def dsyevq3(A, dtype=np.float64):
    npt, ct, sfx = _f(dtype)
    A = np.ascontiguousarray(A, dtype=npt).reshape(9)
    Q = np.zeros(9, npt)
    w = np.zeros(3, npt)
    fail = C.c_int(0)
    getattr(lib(), "orc_dsyevq3" + sfx)(_ptr(A, ct), _ptr(Q, ct), _ptr(w, ct), C.byref(fail))
    return w, Q.reshape(3, 3), fail.value


def eigsrt(d, V, dtype=np.float64):
    npt, ct, sfx = _f(dtype)
    d = np.array(d, dtype=npt)
    V = np.array(V, dtype=npt).reshape(9)
    getattr(lib(), "orc_eigsrt" + sfx)(_ptr(d, ct), _ptr(V, ct))
    return d, V.reshape(3, 3)


def law160_kirchhoff(props, F, sdv, tmp=0.0, e_mart=0.0, dtype=np.float64):
    """compute_kirchoff_stress for one Gauss point.

    F is the flat column-major 3x3 deformation gradient.  Returns
    (tau[9] column-major, sdv_new[3], nr_flag)."""
    npt, ct, sfx = _f(dtype)
    props = np.ascontiguousarray(props, dtype=npt)
    F = np.ascontiguousarray(F, dtype=npt).reshape(9)
    s = np.array(sdv, dtype=npt)
    tau = np.zeros(9, npt)
    fn = getattr(lib(), "orc_law160_kirchhoff" + sfx)
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(ct), ct, C.POINTER(ct), ct, C.POINTER(ct), C.POINTER(ct)]
    fl = fn(_ptr(props, ct), ct(e_mart), _ptr(F, ct), ct(tmp), _ptr(s, ct), _ptr(tau, ct))
    return tau, s, fl


def law160_batch(props, F, sdv_old, tmp=None, e_mart=0.0, dtype=np.float64):
    """Batched eval of law 160: F (n,9) column-major, sdv_old (n,3).

    Returns (pk2 (n,9) column-major second Piola stress, sdv_new (n,3), flags)."""
    npt, ct, sfx = _f(dtype)
    props = np.ascontiguousarray(props, dtype=npt)
    F = np.ascontiguousarray(F, dtype=npt).reshape(-1, 9)
    n = F.shape[0]
    so = np.ascontiguousarray(sdv_old, dtype=npt).reshape(n, 3)
    sn = np.zeros((n, 3), npt)
    pk2 = np.zeros((n, 9), npt)
    fl = np.zeros(n, np.int32)
    t = None if tmp is None else np.ascontiguousarray(tmp, dtype=npt)
    fn = getattr(lib(), "orc_law160_batch" + sfx)
    fn.argtypes = [C.c_int64, C.POINTER(ct), ct, C.POINTER(ct), C.POINTER(ct), C.POINTER(ct),
                   C.POINTER(ct), C.POINTER(ct), C.POINTER(C.c_int32)]
    fn(n, _ptr(props, ct), ct(e_mart), _ptr(F, ct), _ptr(t, ct), _ptr(so, ct), _ptr(sn, ct),
       _ptr(pk2, ct), _ptr(fl, C.c_int32))
    return pk2, sn, fl


def law160_tangent_batch(props, F, sdv_old, tmp=None, e_mart=0.0, dtype=np.float64):
    """Batched law with the algorithmic tangent (flagt = 1): F (n,9) column-major.

    Returns (pk2 (n,9), sdv_new (n,3), dds (n,81) with dds[g, i+3j+9k+27l] =
    gpdds(i,j,k,l), flags)."""
    npt, ct, sfx = _f(dtype)
    props = np.ascontiguousarray(props, dtype=npt)
    F = np.ascontiguousarray(F, dtype=npt).reshape(-1, 9)
    n = F.shape[0]
    so = np.ascontiguousarray(sdv_old, dtype=npt).reshape(n, 3)
    sn = np.zeros((n, 3), npt)
    pk2 = np.zeros((n, 9), npt)
    dds = np.zeros((n, 81), npt)
    fl = np.zeros(n, np.int32)
    t = None if tmp is None else np.ascontiguousarray(tmp, dtype=npt)
    fn = getattr(lib(), "orc_law160_tangent_batch" + sfx)
    fn.argtypes = [C.c_int64, C.POINTER(ct), ct, C.POINTER(ct), C.POINTER(ct), C.POINTER(ct),
                   C.POINTER(ct), C.POINTER(ct), C.POINTER(ct), C.POINTER(C.c_int32)]
    fn(n, _ptr(props, ct), ct(e_mart), _ptr(F, ct), _ptr(t, ct), _ptr(so, ct), _ptr(sn, ct),
       _ptr(pk2, ct), _ptr(dds, ct), _ptr(fl, C.c_int32))
    return pk2, sn, dds, fl


def color_elements(lnods, npoin):
    lnods = np.ascontiguousarray(lnods, dtype=np.int32)
    nelem = lnods.shape[0]
    color_of = np.zeros(nelem, np.int32)
    color_ptr = np.zeros(65, np.int32)
    color_elem = np.zeros(nelem, np.int32)
    nc = lib().orc_color_elements(nelem, npoin, _ptr(lnods, C.c_int32), _ptr(color_of, C.c_int32),
                                  _ptr(color_ptr, C.c_int32), _ptr(color_elem, C.c_int32))
    return nc, color_ptr[: nc + 1].copy(), color_elem, color_of


def critical_dt(lnods, coord, props, densi, lmate=None, dtype=np.float64):
    npt, ct, sfx = _f(dtype)
    lnods = np.ascontiguousarray(lnods, dtype=np.int32)
    coord = np.ascontiguousarray(coord, dtype=npt)
    props = np.ascontiguousarray(props, dtype=npt).reshape(-1)
    densi = np.ascontiguousarray(np.atleast_1d(densi), dtype=npt)
    lm = None if lmate is None else np.ascontiguousarray(lmate, dtype=np.int32)
    fn = getattr(lib(), "orc_critical_dt" + sfx)
    fn.restype = ct
    return float(fn(lnods.shape[0], _ptr(lnods, C.c_int32), _ptr(coord, ct), _ptr(lm, C.c_int32),
                    _ptr(props, ct), _ptr(densi, ct)))


class Problem:
    """A mesh + material + boundary-condition set held as oracle-ready arrays.

    Built from the package's mesh/problem description (duck-typed: any object
    with the attributes read below works)."""

    def __init__(self, p, dtype=np.float64, nthreads=None, native=False):
        npt, ct, sfx = _f(dtype)
        self._lib, self.native = native_lib() if native else (lib(), False)
        self.dtype, self.ct, self.sfx = npt, ct, sfx
        self.nthreads = nthreads or os.cpu_count() or 1
        self.lnods = np.ascontiguousarray(p.lnods, dtype=np.int32)
        self.coord = np.ascontiguousarray(p.coord, dtype=npt)
        self.nelem, self.npoin = self.lnods.shape[0], self.coord.shape[0]
        self.lmate = None if p.lmate is None else np.ascontiguousarray(p.lmate, dtype=np.int32)
        self.props = np.ascontiguousarray(p.props, dtype=npt).reshape(-1, 18)
        self.e_mart = np.ascontiguousarray(p.e_mart, dtype=npt).reshape(-1)
        self.densi = np.ascontiguousarray(p.densi, dtype=npt).reshape(-1)
        self.tempe = None if p.tempe is None else np.ascontiguousarray(p.tempe, dtype=npt)
        self.fixno = np.ascontiguousarray(p.fixno, dtype=np.int32)
        self.bcfun = np.ascontiguousarray(p.bcfun, dtype=np.int32)
        self.fun_npts = np.ascontiguousarray(p.fun_npts, dtype=np.int32)
        self.fun_smooth = np.ascontiguousarray(p.fun_smooth, dtype=np.int32)
        self.fun_tab = np.ascontiguousarray(p.fun_tab, dtype=npt)
        self.fext = None if p.fext is None else np.ascontiguousarray(p.fext, dtype=npt)
        self.load_fun = int(p.load_fun)
        dampi = getattr(p, "dampi", None)
        self.dampi = None if dampi is None else np.ascontiguousarray(dampi, dtype=npt).reshape(-1, 2)
        nc, cp, ce, _ = color_elements(self.lnods, self.npoin)
        self.ncolor, self.color_ptr, self.color_elem = nc, cp, ce
        self.reset()

    def reset(self):
        npt = self.dtype
        self.cutim = np.zeros(1, npt)
        self.displ = np.zeros((self.npoin, 3), npt)
        self.veloc = np.zeros((self.npoin, 3), npt)
        self.accel = np.zeros((self.npoin, 3), npt)
        self.sdv = np.zeros((self.nelem, 2, 8, 3), npt)
        self.rhsid = np.zeros((self.npoin, 3), npt)
        self.counters = np.zeros(NCOUNTERS, np.int32)

    def assemble(self, displ=None, want_all=False, fext_scale=0.0, veloc=None):
        """One element loop (sld_matrix explicit) at the given displacement
        (and, with Rayleigh damping, nodal velocity).

        Reads state slot TIME_N, writes slot ITER_K.  Returns a dict."""
        ct = self.ct
        d = self.displ if displ is None else np.ascontiguousarray(displ, dtype=self.dtype)
        v = None if veloc is None else np.ascontiguousarray(veloc, dtype=self.dtype)
        n3 = (self.npoin, 3)
        out = {k: np.zeros(n3, self.dtype) for k in ("rhsid", "finte", "fexte", "frxid")}
        out["vmass"] = np.zeros(self.npoin, self.dtype)
        dmin = np.zeros(1, self.dtype)
        fn = getattr(self._lib, "orc_assemble" + self.sfx)
        fn(self.nelem, self.npoin, _ptr(self.lnods, C.c_int32), _ptr(self.coord, ct), _ptr(d, ct),
           _ptr(self.lmate, C.c_int32), _ptr(self.props, ct), _ptr(self.e_mart, ct),
           _ptr(self.densi, ct), _ptr(self.tempe, ct), None, _ptr(self.fext, ct),
           ct(fext_scale), _ptr(self.fixno, C.c_int32), _ptr(self.sdv, ct), self.ncolor,
           _ptr(self.color_ptr, C.c_int32), _ptr(self.color_elem, C.c_int32), self.nthreads,
           _ptr(out["rhsid"], ct), _ptr(out["finte"], ct), _ptr(out["fexte"], ct),
           _ptr(out["frxid"], ct), _ptr(out["vmass"], ct), _ptr(dmin, ct),
           _ptr(self.counters, C.c_int32), _ptr(v, ct), _ptr(self.dampi, ct))
        out["gpdet_min"] = float(dmin[0])
        return out

    def postprocess(self, displ=None, slot=1, gp_sigma=False, gauss=False):
        """Nodal Cauchy stress, Green and log strain (npoin, 6) in Voigt order
        xx yy zz yz xz xy, von Mises (npoin,), and optionally the Gauss-point
        Cauchy stress (nelem, 8, 6), with the law evaluated on state `slot`
        (1 = TIME_N, what the last assemble() started from).  gauss=True adds
        the element-loop fields gpgdi / gppio (nelem, 8, 3, 3) holding
        Fortran T(i,j) at [..., j, i], gpdet (nelem, 8) and volum (2,)."""
        ct = self.ct
        d = self.displ if displ is None else np.ascontiguousarray(displ, dtype=self.dtype)
        out = {k: np.zeros((self.npoin, 6), self.dtype) for k in ("caust", "green", "lepsi")}
        out["seqvm"] = np.zeros(self.npoin, self.dtype)
        gp = np.zeros((self.nelem, 8, 6), self.dtype) if gp_sigma else None
        gf = {k: np.zeros((self.nelem, 8, 3, 3), self.dtype) for k in ("gpgdi", "gppio")} if gauss else {}
        gdet = np.zeros((self.nelem, 8), self.dtype) if gauss else None
        vol = np.zeros(2, self.dtype) if gauss else None
        fn = getattr(self._lib, "orc_postprocess" + self.sfx)
        fn.argtypes = None
        rc = fn(self.nelem, self.npoin, _ptr(self.lnods, C.c_int32), _ptr(self.coord, ct),
                _ptr(d, ct), _ptr(self.lmate, C.c_int32), _ptr(self.props, ct),
                _ptr(self.e_mart, ct), _ptr(self.tempe, ct), _ptr(self.sdv, ct), int(slot),
                _ptr(out["caust"], ct), _ptr(out["green"], ct), _ptr(out["lepsi"], ct),
                _ptr(out["seqvm"], ct), _ptr(gp, ct), _ptr(gf.get("gpgdi"), ct),
                _ptr(gf.get("gppio"), ct), _ptr(gdet, ct), _ptr(vol, ct))
        if rc:
            raise MemoryError("orc_postprocess")
        if gp_sigma:
            out["gp_sigma"] = gp
        if gauss:
            out.update(gf, gpdet=gdet, volum=vol)
        return out

    def end_step(self):
        """sld_updunk(ITASK_ENDSTE) for the state: TIME_N <- ITER_K."""
        self.sdv[:, 1] = self.sdv[:, 0]

    def critical_dt(self):
        return critical_dt(self.lnods, self.coord, self.props, self.densi, self.lmate, self.dtype)

    def run(self, dtime, nsteps, wit_dof=None, scheme="cd", phi=1.033):
        """Explicit time loop (scheme "cd" central difference or "tw"
        Tchamwa-Wielgosz); returns the witness history (nsteps, nwit) of displ
        at flat dof ids 3*ipoin+idime."""
        ct = self.ct
        wit = np.zeros(0, np.int32) if wit_dof is None else np.ascontiguousarray(wit_dof, np.int32)
        if wit.size and (wit.min() < 0 or wit.max() >= 3 * self.npoin):
            raise ValueError("oracle witnesses are displacement dofs in [0, 3*npoin)")
        hist = np.zeros((nsteps, max(1, wit.size)), self.dtype)
        fn = getattr(self._lib, "orc_run_cd" + self.sfx)
        fn.argtypes = None
        fn(self.nelem, self.npoin, _ptr(self.lnods, C.c_int32), _ptr(self.coord, ct),
           _ptr(self.lmate, C.c_int32), _ptr(self.props, ct), _ptr(self.e_mart, ct),
           _ptr(self.densi, ct), _ptr(self.tempe, ct), _ptr(self.fixno, C.c_int32),
           _ptr(self.bcfun, C.c_int32), int(self.fun_npts.size), _ptr(self.fun_npts, C.c_int32),
           _ptr(self.fun_smooth, C.c_int32), _ptr(self.fun_tab, ct), _ptr(self.fext, ct),
           self.load_fun, self.ncolor, _ptr(self.color_ptr, C.c_int32),
           _ptr(self.color_elem, C.c_int32), self.nthreads, ct(dtime), int(nsteps),
           _ptr(self.cutim, ct), _ptr(self.displ, ct), _ptr(self.veloc, ct), _ptr(self.accel, ct),
           _ptr(self.sdv, ct), _ptr(self.rhsid, ct), int(wit.size), _ptr(wit, C.c_int32),
           _ptr(hist, ct), _ptr(self.counters, C.c_int32), 1 if scheme == "tw" else 0, ct(phi),
           _ptr(self.dampi, ct))
        return hist[:, : wit.size]


# -- learned surrogate's network (FP64 restatement, sma_mlp.c) --------------
MLP_NIN, MLP_NOUT = 14, 13


def mlp_nparam():
    return int(lib().orc_mlp_nparam())


def mlp_forward(params, stats, x):
    """Raw outputs (n, 13) of the network on raw inputs x (n, 14)."""
    p = np.ascontiguousarray(params, np.float64)
    s = np.ascontiguousarray(stats, np.float64)
    xx = np.ascontiguousarray(x, np.float64).reshape(-1, MLP_NIN)
    y = np.zeros((xx.shape[0], MLP_NOUT))
    lib().orc_mlp_forward(_ptr(p, C.c_double), _ptr(s, C.c_double), C.c_int64(xx.shape[0]),
                          _ptr(xx, C.c_double), _ptr(y, C.c_double))
    return y


def mlp_loss_grad(params, stats, x, y, grad=True):
    """(loss, gradient) of the normalised mean squared error of the batch."""
    p = np.ascontiguousarray(params, np.float64)
    s = np.ascontiguousarray(stats, np.float64)
    xx = np.ascontiguousarray(x, np.float64).reshape(-1, MLP_NIN)
    yy = np.ascontiguousarray(y, np.float64).reshape(-1, MLP_NOUT)
    g = np.zeros(p.size) if grad else None
    fn = lib().orc_mlp_loss_grad
    fn.restype = C.c_double
    loss = fn(_ptr(p, C.c_double), _ptr(s, C.c_double), C.c_int64(xx.shape[0]), _ptr(xx, C.c_double),
              _ptr(yy, C.c_double), _ptr(g, C.c_double) if grad else None)
    return float(loss), g
