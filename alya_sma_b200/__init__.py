"""alya_sma_b200 -- B200 (sm_100a) explicit solid-mechanics step for
superelastic shape-memory alloys: Alya solidz with constitutive law 160.

Host-side mirror of the reference's interfaces over the C ABI of
``libalya_sma_b200.so`` (declared in include/alya_sma.h):

* ``eval_sld_stress_model_160`` -- the material plugin
  (sld_stress_model_160.f90:36-195, flagt = 0) on a batch of Gauss points;
* ``ExplicitSolid.assemble``    -- the explicit element loop
  sld_matrix(SLD_EXPLICIT_SCHEME) (sld_matrix.f90:29-327) with host arrays;
* ``ExplicitSolid.step``        -- the central-difference step sld_explicit
  (mod_sld_solution_methods.f90:101-223) with BC update and state swap,
  device resident and replayed as CUDA graphs.

There is no CPU fallback: every call runs the CUDA library and raises
``SmaError`` when it cannot (library missing, no sm_100 device, bad input).
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

from . import problem  # noqa: F401  (re-export)

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libalya_sma_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "alya_sma.h")

PREC = {"fp64": 0, "fp32": 1}
SCATTER = {"auto": 0, "atomic": 1, "color": 2}
FIELD = {"displ": 0, "veloc": 1, "accel": 2, "rhsid": 3, "vmass": 4}
COUNTERS = ["nr_active", "nr_failed", "nr_both", "neg_det", "nonfinite"]


class SmaError(RuntimeError):
    pass


class _Mesh(C.Structure):
    _fields_ = [("nelem", C.c_int32), ("npoin", C.c_int32), ("lnods", C.c_void_p),
                ("coord", C.c_void_p), ("lmate", C.c_void_p)]


class _Mat(C.Structure):
    _fields_ = [("nmate", C.c_int32), ("props", C.c_void_p), ("e_mart", C.c_void_p),
                ("densi", C.c_void_p), ("tempe", C.c_void_p), ("dampi", C.c_void_p)]


class _Run(C.Structure):
    _fields_ = [("precision", C.c_int32), ("scatter", C.c_int32), ("device", C.c_int32),
                ("nfun", C.c_int32), ("dtime", C.c_double), ("fixno", C.c_void_p),
                ("bcfun", C.c_void_p), ("fun_npts", C.c_void_p), ("fun_smooth", C.c_void_p),
                ("fun_tab", C.c_void_p), ("fext", C.c_void_p), ("load_fun", C.c_int32),
                ("block", C.c_int32), ("scheme", C.c_int32), ("phitw", C.c_double),
                ("variant", C.c_int32)]


SCHEME = {"cd": 0, "tw": 1}
VARIANT = {"auto": 0, "pipe": 1, "plain": 2, "table": 3}


class _Counters(C.Structure):
    _fields_ = [("c", C.c_int64 * 8), ("gpdet_min", C.c_double), ("ielem_min", C.c_int64)]


_lib = None


def header_functions() -> list[str]:
    """Names of every entry point declared in include/alya_sma.h."""
    with open(HEADER) as fh:
        txt = fh.read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\*\s]+?\b(sma_\w+)\s*\(", txt, re.M)))


def lib():
    """Load the CUDA library (raises SmaError when it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SmaError(f"{LIB_PATH} is missing: run `python -m alya_sma_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.sma_last_error.restype = C.c_char_p
        L.sma_version.restype = C.c_char_p
        L.sma_stream.restype = C.c_void_p
        L.sma_stream.argtypes = [C.c_void_p]
        L.sma_kernel_launches.restype = C.c_int64
        L.sma_kernel_launches.argtypes = [C.c_void_p]
        L.sma_ctx_create.argtypes = [C.POINTER(_Mesh), C.POINTER(_Mat), C.POINTER(_Run), C.POINTER(C.c_void_p)]
        L.sma_ctx_destroy.argtypes = [C.c_void_p]
        L.sma_explicit_step.argtypes = [C.c_void_p, C.c_int32]
        L.sma_assemble.argtypes = [C.c_void_p, C.c_void_p, C.c_double] + [C.c_void_p] * 5
        L.sma_assemble_device.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        L.sma_end_step.argtypes = [C.c_void_p]
        L.sma_postprocess.argtypes = [C.c_void_p] * 6
        L.sma_host_register.argtypes = [C.c_void_p, C.c_size_t]
        L.sma_host_unregister.argtypes = [C.c_void_p]
        L.sma_gauss_fields.argtypes = [C.c_void_p] * 5
        L.sma_eval_law160.argtypes = [C.c_int64, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                      C.c_void_p]
        L.sma_eval_law160_tangent.argtypes = [C.c_int64, C.c_void_p, C.c_double, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p]
        L.sma_set_nodal.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.sma_step_prologue.argtypes = [C.c_void_p]
        L.sma_step_elements.argtypes = [C.c_void_p]
        L.sma_step_elements_range.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        L.sma_step_nodes.argtypes = [C.c_void_p, C.c_int32]
        L.sma_gather_residual.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.sma_scatter_residual.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.sma_get_nodal.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.sma_set_state.argtypes = [C.c_void_p, C.c_void_p]
        L.sma_get_state.argtypes = [C.c_void_p, C.c_void_p]
        L.sma_get_time.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.sma_set_time.argtypes = [C.c_void_p, C.c_double]
        L.sma_get_counters.argtypes = [C.c_void_p, C.POINTER(_Counters)]
        L.sma_reset_counters.argtypes = [C.c_void_p]
        L.sma_set_witness.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
        L.sma_get_witness.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]
        L.sma_critical_dt.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.sma_set_timing.argtypes = [C.c_void_p, C.c_int32]
        L.sma_get_timers.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.sma_set_energy.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        L.sma_get_energy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]
        L.sma_checkpoint_save.argtypes = [C.c_void_p, C.c_char_p]
        L.sma_checkpoint_load.argtypes = [C.c_void_p, C.c_char_p]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise SmaError(f"alya_sma error {rc}: {lib().sma_last_error().decode()}")


def _p(a):
    return None if a is None else a.ctypes.data


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


class ExplicitSolid:
    """One explicit SMA solid on one GPU (a ``sma_ctx``).

    ``prob`` is an ``alya_sma_b200.problem.Problem``.  precision "fp64" is the
    reference's arithmetic; "fp32" runs element kinematics and the
    constitutive update in FP32 (return map, force accumulation and time
    integration stay FP64)."""

    def __init__(self, prob, precision="fp64", scatter="atomic", device=0, dtime=None, block=0,
                 scheme="cd", phitw=0.0, variant="auto"):
        L = lib()
        self.prob = prob
        self.precision = precision
        self.npoin, self.nelem = prob.npoin, prob.nelem
        self._keep = dict(
            lnods=_c(prob.lnods, np.int32), coord=_c(prob.coord, np.float64),
            lmate=_c(prob.lmate, np.int32), props=_c(prob.props, np.float64),
            e_mart=_c(prob.e_mart, np.float64), densi=_c(prob.densi, np.float64),
            tempe=_c(prob.tempe, np.float64), fixno=_c(prob.fixno, np.int32),
            bcfun=_c(prob.bcfun, np.int32), fun_npts=_c(prob.fun_npts, np.int32),
            fun_smooth=_c(prob.fun_smooth, np.int32), fun_tab=_c(prob.fun_tab, np.float64),
            fext=_c(prob.fext, np.float64), dampi=_c(getattr(prob, "dampi", None), np.float64))
        k = self._keep
        mesh = _Mesh(self.nelem, self.npoin, _p(k["lnods"]), _p(k["coord"]), _p(k["lmate"]))
        mat = _Mat(k["props"].reshape(-1, 18).shape[0], _p(k["props"]), _p(k["e_mart"]),
                   _p(k["densi"]), _p(k["tempe"]), _p(k["dampi"]))
        run = _Run(PREC[precision], SCATTER[scatter], device, int(k["fun_npts"].size),
                   float(prob.dtime if dtime is None else dtime), _p(k["fixno"]), _p(k["bcfun"]),
                   _p(k["fun_npts"]), _p(k["fun_smooth"]), _p(k["fun_tab"]), _p(k["fext"]),
                   int(prob.load_fun), int(block), SCHEME[scheme], float(phitw), VARIANT[variant])
        self._ctx = C.c_void_p()
        _check(L.sma_ctx_create(C.byref(mesh), C.byref(mat), C.byref(run), C.byref(self._ctx)))

    def close(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            lib().sma_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- step boundary ------------------------------------------------------
    def step(self, nsteps=1):
        _check(lib().sma_explicit_step(self._ctx, int(nsteps)))

    # -- element-loop boundary ----------------------------------------------
    def assemble(self, displ, fext_scale=0.0, want_all=True, rhsid=None):
        """sld_matrix explicit: returns dict of (npoin,3) rhsid, finte, fexte,
        frxid and (npoin,) vmass.  Reads state TIME_N, writes ITER_K.  rhsid:
        an optional caller-owned (npoin, 3) float64 output array (e.g. one
        page-locked with host_register, like displ)."""
        d = np.ascontiguousarray(displ, dtype=np.float64).reshape(self.npoin, 3)
        out = {q: np.zeros((self.npoin, 3)) for q in ("rhsid", "finte", "fexte", "frxid")}
        if rhsid is not None:
            if rhsid.dtype != np.float64 or rhsid.shape != (self.npoin, 3) or not rhsid.flags["C_CONTIGUOUS"]:
                raise ValueError("rhsid must be a C-contiguous float64 (npoin, 3) array")
            out["rhsid"] = rhsid
        out["vmass"] = np.zeros(self.npoin)
        if not want_all:
            for q in ("finte", "fexte", "frxid", "vmass"):
                out[q] = None
        _check(lib().sma_assemble(self._ctx, _p(d), float(fext_scale), _p(out["rhsid"]),
                                  _p(out["finte"]), _p(out["fexte"]), _p(out["frxid"]),
                                  _p(out["vmass"])))
        return out

    def end_step(self):
        _check(lib().sma_end_step(self._ctx))

    def postprocess(self, gp_sigma=False):
        """sld_calculate_pp_tensors: nodal Cauchy stress 'caust', Green strain
        'green' and log strain 'lepsi' as (npoin, 6) in Voigt order xx yy zz
        yz xz xy, von Mises 'seqvm' (npoin,), and with gp_sigma the Cauchy
        stress per Gauss point (nelem, 8, 6).  Evaluated at the current
        displacement from the state the last element loop started from."""
        out = {k: np.zeros((self.npoin, 6)) for k in ("caust", "green", "lepsi")}
        out["seqvm"] = np.zeros(self.npoin)
        gp = np.zeros((self.nelem, 8, 6)) if gp_sigma else None
        _check(lib().sma_postprocess(self._ctx, _p(out["caust"]), _p(out["green"]), _p(out["lepsi"]),
                                     _p(out["seqvm"]), _p(gp)))
        if gp_sigma:
            out["gp_sigma"] = gp
        return out

    # -- data ----------------------------------------------------------------
    def get(self, field):
        n = (self.npoin,) if field == "vmass" else (self.npoin, 3)
        out = np.zeros(n)
        _check(lib().sma_get_nodal(self._ctx, FIELD[field], _p(out)))
        return out

    def set(self, field, arr):
        n = (self.npoin,) if field == "vmass" else (self.npoin, 3)
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(n)
        _check(lib().sma_set_nodal(self._ctx, FIELD[field], _p(a)))

    @property
    def state(self):
        """svegm in the reference layout: (nelem, 2, 8, 3), slot 0 = ITER_K,
        slot 1 = TIME_N."""
        out = np.zeros((self.nelem, 2, 8, 3))
        _check(lib().sma_get_state(self._ctx, _p(out)))
        return out

    @state.setter
    def state(self, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.nelem, 2, 8, 3)
        _check(lib().sma_set_state(self._ctx, _p(a)))

    @property
    def time(self):
        t = C.c_double()
        _check(lib().sma_get_time(self._ctx, C.byref(t)))
        return t.value

    @time.setter
    def time(self, t):
        _check(lib().sma_set_time(self._ctx, float(t)))

    def counters(self, reset=False):
        c = _Counters()
        _check(lib().sma_get_counters(self._ctx, C.byref(c)))
        if reset:
            _check(lib().sma_reset_counters(self._ctx))
        out = {name: int(c.c[i]) for i, name in enumerate(COUNTERS)}
        out["sur_fallback"] = int(c.c[5])                     # surrogate points the plain law handled
        out["sur_ood"] = int(c.c[7])                          # network evaluations its gates refused
        out["gpdet_min"] = float(c.gpdet_min)                 # smallest det F <= 0, 0.0 if none
        out["ielem_min"] = int(c.ielem_min)                   # its element, -1 if none
        return out

    def gauss_fields(self):
        """Element-loop fields per Gauss point from the same evaluation as
        postprocess(): 'gpgdi' (F) and 'gppio' (P = F S) as (nelem, 8, 3, 3)
        holding Fortran T(i,j) at [..., j, i], 'gpdet' (nelem, 8) and
        'volum' = (reference volume, deformed volume)."""
        out = {k: np.zeros((self.nelem, 8, 3, 3)) for k in ("gpgdi", "gppio")}
        out["gpdet"] = np.zeros((self.nelem, 8))
        out["volum"] = np.zeros(2)
        _check(lib().sma_gauss_fields(self._ctx, _p(out["gpgdi"]), _p(out["gppio"]), _p(out["gpdet"]),
                                      _p(out["volum"])))
        return out

    def set_witness(self, dofs, max_steps):
        d = np.ascontiguousarray(dofs, dtype=np.int32)
        _check(lib().sma_set_witness(self._ctx, int(d.size), _p(d), int(max_steps)))
        self._nwit = int(d.size)
        self._wmax = int(max_steps)

    def witness(self):
        out = np.zeros((self._wmax, self._nwit))
        n = C.c_int32()
        _check(lib().sma_get_witness(self._ctx, _p(out), C.byref(n)))
        return out[: n.value]

    def set_surrogate(self, net, gate=3.0, xs_tol=1e-3, f_margin=10.0, period=64, enable=True):
        """The learned surrogate (alya_sma_b200.surrogate.Surrogate) in the
        element loop of this FP32 context (sma_set_surrogate), or back to the
        plain law with enable=False."""
        L = lib()
        L.sma_set_surrogate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                        C.c_int32, C.c_int32]
        if not enable:
            _check(L.sma_set_surrogate(self._ctx, None, None, 1.0, 0.0, 0.0, 1, 0))
            return
        w = np.ascontiguousarray(net.params(), dtype=np.float32)
        st = net.stats_host
        _check(L.sma_set_surrogate(self._ctx, w.ctypes.data, C.addressof(st), float(gate), float(xs_tol),
                                   float(f_margin), int(period), 1))
        self._sur_keep = (w, st)

    def surrogate_status(self):
        s = C.c_int32()
        L = lib()
        L.sma_surrogate_status.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        _check(L.sma_surrogate_status(self._ctx, C.byref(s)))
        return int(s.value)

    def set_launch_plan(self, ends, blocks):
        """Element ranges [ends[r-1], ends[r]) launched with blocks[r] threads
        per block (sma_set_launch_plan); empty lists return to one launch."""
        L = lib()
        L.sma_set_launch_plan.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        e = np.ascontiguousarray(ends, dtype=np.int32)
        b = np.ascontiguousarray(blocks, dtype=np.int32)
        _check(L.sma_set_launch_plan(self._ctx, int(e.size), _p(e) if e.size else None,
                                     _p(b) if b.size else None))

    def critical_dt(self):
        d = C.c_double()
        _check(lib().sma_critical_dt(self._ctx, C.byref(d)))
        return d.value

    def set_energy(self, on=True, max_steps=0):
        """Energy balance of sld_energy after every step (history rows of
        ALLIE, ALLWK, ALLKE, ETOTA, EENER up to max_steps)."""
        _check(lib().sma_set_energy(self._ctx, int(bool(on)), int(max_steps)))
        self._emax = int(max_steps)

    def energy(self):
        """(totals dict, history array (nrows, 5))."""
        tot = np.zeros(5)
        hist = np.zeros((max(1, getattr(self, "_emax", 0)), 5))
        n = C.c_int32()
        _check(lib().sma_get_energy(self._ctx, _p(tot), _p(hist), C.byref(n)))
        names = ("allie", "allwk", "allke", "etota", "eener")
        return {k: float(tot[i]) for i, k in enumerate(names)}, hist[: n.value]

    def save(self, path):
        """Checkpoint of the step-boundary state (restart)."""
        _check(lib().sma_checkpoint_save(self._ctx, os.fsencode(path)))

    def load(self, path):
        _check(lib().sma_checkpoint_load(self._ctx, os.fsencode(path)))

    def set_timing(self, on=True):
        _check(lib().sma_set_timing(self._ctx, int(bool(on))))

    def timers(self):
        """{'element': (ms, launches), 'nodal': (...), 'step': (...)} since
        set_timing(True)."""
        ms = np.zeros(3)
        cnt = np.zeros(3, np.int64)
        _check(lib().sma_get_timers(self._ctx, _p(ms), _p(cnt)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(("element", "nodal", "step"))}

    @property
    def stream(self):
        return lib().sma_stream(self._ctx)

    @property
    def kernel_launches(self):
        return int(lib().sma_kernel_launches(self._ctx))

    def launch_info(self):
        """The element kernel's launch shape this context chose
        (sma_launch_info): threads per block, variant, compact records."""
        b, v, k = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().sma_launch_info(self._ctx, C.byref(b), C.byref(v), C.byref(k)))
        names = {val: name for name, val in VARIANT.items()}
        return {"block": int(b.value), "variant": names.get(int(v.value), int(v.value)),
                "compact_records": bool(k.value)}


def host_register(arr):
    """Page-lock a C-contiguous numpy array in place (sma_host_register), so
    ExplicitSolid.assemble's copies of it overlap the element loop."""
    if not arr.flags["C_CONTIGUOUS"]:
        raise ValueError("host_register needs a C-contiguous array")
    _check(lib().sma_host_register(arr.ctypes.data, arr.nbytes))
    return arr


def host_unregister(arr):
    _check(lib().sma_host_unregister(arr.ctypes.data))


def eval_sld_stress_model_160(props, gpgdi, gpsdv, gptmp=None, flagt=0, e_mart=0.0,
                              precision="fp64"):
    """Material plugin of law 160 on the GPU, batched.

    Mirrors eval_sld_stress_model_160(pgaus, props, gpgdi, gptmp, gpsdv,
    gpstr, gpdds, flagt) (sld_stress_model_160.f90:36-48) for any number of
    Gauss points: ``gpgdi`` (n, 3, 3) deformation gradients with
    gpgdi[g, i, j] = F(i, j); ``gpsdv`` (n, 3) state of slot TIME_N.  Returns
    (gpstr (n, 3, 3) second Piola stress, new state (n, 3) for slot ITER_K,
    NR flags (n,)); with flagt = 1 (FP64 only) also gpdds (n, 3, 3, 3, 3),
    gpdds[g, i, j, k, l] = gpdds(i, j, k, l, igaus), the algorithmic tangent
    (sld_stress_model_160.f90:118-155, 170-191).

    Arrays may be numpy (copied through the device) or torch CUDA tensors
    (used in place)."""
    if flagt not in (0, 1):
        raise SmaError("flagt is 0 (stress) or 1 (stress and algorithmic tangent)")
    if flagt == 1 and precision != "fp64":
        raise SmaError("the algorithmic tangent is FP64 only: its eps = 1e-5 forward differences "
                       "are below FP32 resolution")
    import torch
    if not torch.cuda.is_available():
        raise SmaError("eval_sld_stress_model_160 needs a CUDA device")
    dev = torch.device("cuda")
    F = torch.as_tensor(np.asarray(gpgdi) if not torch.is_tensor(gpgdi) else gpgdi,
                        dtype=torch.float64, device=dev)
    n = F.shape[0]
    Fc = F.reshape(n, 3, 3).transpose(1, 2).contiguous()          # column-major per point
    S0 = torch.as_tensor(np.asarray(gpsdv) if not torch.is_tensor(gpsdv) else gpsdv,
                         dtype=torch.float64, device=dev).reshape(n, 3).contiguous()
    T = None
    if gptmp is not None:
        T = torch.as_tensor(np.asarray(gptmp) if not torch.is_tensor(gptmp) else gptmp,
                            dtype=torch.float64, device=dev).reshape(n).contiguous()
    S1 = torch.empty_like(S0)
    P = torch.empty((n, 9), dtype=torch.float64, device=dev)
    fl = torch.empty(n, dtype=torch.int32, device=dev)
    pr = np.ascontiguousarray(props, dtype=np.float64).reshape(18)
    if flagt == 1:
        D = torch.empty((n, 81), dtype=torch.float64, device=dev)
        _check(lib().sma_eval_law160_tangent(n, _p(pr), float(e_mart), Fc.data_ptr(),
                                             None if T is None else T.data_ptr(), S0.data_ptr(),
                                             S1.data_ptr(), P.data_ptr(), D.data_ptr(),
                                             fl.data_ptr(), torch.cuda.current_stream().cuda_stream))
        torch.cuda.current_stream().synchronize()
        gpdds = D.reshape(n, 3, 3, 3, 3).permute(0, 4, 3, 2, 1)     # column-major (i,j,k,l)
        return P.reshape(n, 3, 3).transpose(1, 2), S1, fl, gpdds
    _check(lib().sma_eval_law160(n, _p(pr), float(e_mart), Fc.data_ptr(),
                                 None if T is None else T.data_ptr(), S0.data_ptr(),
                                 S1.data_ptr(), P.data_ptr(), fl.data_ptr(), PREC[precision],
                                 torch.cuda.current_stream().cuda_stream))
    torch.cuda.current_stream().synchronize()
    gpstr = P.reshape(n, 3, 3).transpose(1, 2)
    return gpstr, S1, fl
