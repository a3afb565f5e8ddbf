"""sma_assemble_noalloc: the element loop for callers that cannot allocate
device memory (their device arrays belong to an OpenACC region or a pool of
their own, or a cudaMalloc would synchronise the device).  Checked through
the C ABI against the context entry point sma_assemble on two calls in a
row, with the FP64 tolerance of the other element-loop tests; a call after
the first allocates no device memory, leaves the caller's TIME_N state slot
untouched, and reports its return-map and det F <= 0 counters.

The file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes as C

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


def _noalloc(L):
    fn = L.sma_assemble_noalloc
    fn.restype = C.c_int32
    fn.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_double, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    return fn


class _Counters(C.Structure):
    _fields_ = [("c", C.c_int64 * 8), ("gpdet_min", C.c_double), ("ielem_min", C.c_int64)]


def _counters(L, stream):
    fn = L.sma_noalloc_counters
    fn.restype = C.c_int32
    fn.argtypes = [C.POINTER(_Counters), C.c_void_p]
    c = _Counters()
    assert fn(C.byref(c), stream) == 0, L.sma_last_error().decode()
    return c


def _field(p, strain, seed):
    rng = np.random.default_rng(seed)
    X = p.coord
    u = np.stack([strain * X[:, 0] * (1 + 0.2 * np.sin(X[:, 0] / 6.0)),
                  -0.3 * strain * (X[:, 1] - 2.0), -0.3 * strain * (X[:, 2] - 2.0)], axis=1)
    return u + rng.normal(size=u.shape) * 1e-4


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_context_entry_point(precision):
    import torch
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    L = sma.lib()
    fn = _noalloc(L)
    ref = sma.ExplicitSolid(p, precision=precision)
    dev = torch.device("cuda")
    lnods = torch.as_tensor(p.lnods, dtype=torch.int32, device=dev).contiguous()
    coord = torch.as_tensor(p.coord, dtype=torch.float64, device=dev).contiguous()
    sdv = torch.zeros((p.nelem, 2, 8, 3), dtype=torch.float64, device=dev)
    rhs = torch.empty((p.npoin, 3), dtype=torch.float64, device=dev)
    props = np.ascontiguousarray(p.props[0], dtype=np.float64)
    stream = torch.cuda.current_stream()
    tol = 1e-8 if precision == "fp64" else 1e-3
    for call, strain in enumerate((0.012, 0.03)):           # two calls in a row
        u = _field(p, strain, call)
        r = ref.assemble(u)
        ref.end_step()
        displ = torch.as_tensor(u, dtype=torch.float64, device=dev).contiguous()
        timen = sdv[:, 1].clone()
        stream.synchronize()
        held, free0 = torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0]
        rc = fn(p.nelem, p.npoin, lnods.data_ptr(), coord.data_ptr(), displ.data_ptr(),
                props.ctypes.data, 0.0, sdv.data_ptr(), rhs.data_ptr(),
                sma.PREC[precision], stream.cuda_stream)
        assert rc == 0, L.sma_last_error().decode()
        stream.synchronize()
        if call > 0:                                        # the first call may load the module
            assert torch.cuda.memory_allocated() == held
            assert torch.cuda.mem_get_info()[0] == free0, "a call allocated device memory"
        assert torch.equal(sdv[:, 1], timen), "slot TIME_N changed"
        cnt = _counters(L, stream.cuda_stream)
        assert cnt.c[0] > 0 and cnt.c[1] == 0 and cnt.c[3] == 0 and cnt.ielem_min == -1
        got = rhs.cpu().numpy()
        err = np.abs(got - r["rhsid"]).max() / np.abs(r["finte"]).max()
        assert err < tol, (call, err)
        st = sdv.cpu().numpy()
        st_ref = ref.state                                  # after end_step: slot 1 = TIME_N
        # relative to the largest state value (the F_AS/F_SA entries are ~1e2)
        srel = np.abs(st[:, 0] - st_ref[:, 1]).max() / np.abs(st_ref[:, 1]).max()
        assert srel < (1e-11 if precision == "fp64" else 1e-5), (call, srel)
        sdv[:, 1] = sdv[:, 0]                               # end of step: TIME_N <- ITER_K
    assert st[:, 0, :, 0].max() > 0.05                      # martensite formed
    ref.close()


def test_noalloc_rejects_oversized_mesh_and_bad_ids():
    import torch
    L = sma.lib()
    fn = _noalloc(L)
    props = np.ascontiguousarray(P.nitinol_props(**P.NITI), dtype=np.float64)
    rc = fn(16385, 8, None, None, None, props.ctypes.data, 0.0, None, None, 0, None)
    assert rc == -1 and b"exceeds" in L.sma_last_error()
    p = P.bar_40x4x4(nsteps=10)
    dev = torch.device("cuda")
    ln = p.lnods.copy()
    ln[5, 3] = p.npoin + 7
    lnods = torch.as_tensor(ln, dtype=torch.int32, device=dev)
    coord = torch.as_tensor(p.coord, dtype=torch.float64, device=dev)
    sdv = torch.zeros((p.nelem, 2, 8, 3), dtype=torch.float64, device=dev)
    rhs = torch.empty((p.npoin, 3), dtype=torch.float64, device=dev)
    rc = fn(p.nelem, p.npoin, lnods.data_ptr(), coord.data_ptr(), coord.data_ptr(),
            props.ctypes.data, 0.0, sdv.data_ptr(), rhs.data_ptr(), 0, None)
    assert rc == -1 and b"lnods" in L.sma_last_error()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_reports_inverted_gauss_points(precision):
    """A node pushed through the opposite corner of its elements inverts
    Gauss points; the counters of the call report them, with the smallest
    det F and an element around that node, as the context path does."""
    import torch
    p = P.bar_40x4x4(nsteps=10, ref_equivalent=True)
    L = sma.lib()
    fn = _noalloc(L)
    dev = torch.device("cuda")
    X = p.coord
    node = int(np.argmin(np.linalg.norm(X - np.array([20.0, 2.0, 2.0]), axis=1)))   # interior
    u = np.zeros_like(X)
    u[node] = (-1.6, -1.6, -1.6)
    lnods = torch.as_tensor(p.lnods, dtype=torch.int32, device=dev).contiguous()
    coord = torch.as_tensor(X, dtype=torch.float64, device=dev).contiguous()
    displ = torch.as_tensor(u, dtype=torch.float64, device=dev).contiguous()
    sdv = torch.zeros((p.nelem, 2, 8, 3), dtype=torch.float64, device=dev)
    rhs = torch.empty((p.npoin, 3), dtype=torch.float64, device=dev)
    props = np.ascontiguousarray(p.props[0], dtype=np.float64)
    stream = torch.cuda.current_stream()
    rc = fn(p.nelem, p.npoin, lnods.data_ptr(), coord.data_ptr(), displ.data_ptr(), props.ctypes.data,
            0.0, sdv.data_ptr(), rhs.data_ptr(), sma.PREC[precision], stream.cuda_stream)
    assert rc == 0, L.sma_last_error().decode()
    cnt = _counters(L, stream.cuda_stream)
    around = set(np.nonzero((p.lnods == node).any(axis=1))[0].tolist())
    assert cnt.c[3] > 0, "no det F <= 0 reported"
    assert cnt.gpdet_min <= 0.0
    assert cnt.ielem_min in around
