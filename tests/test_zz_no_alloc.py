"""sma_assemble_noalloc: the element loop for callers that cannot allocate
device memory (their device arrays belong to an OpenACC region or a pool of
their own, or a cudaMalloc would synchronise the device).  Checked through
the C ABI against the context entry point sma_assemble on two calls in a
row, with the FP64 tolerance of the other element-loop tests.

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
        rc = fn(p.nelem, p.npoin, lnods.data_ptr(), coord.data_ptr(), displ.data_ptr(),
                props.ctypes.data, 0.0, sdv.data_ptr(), rhs.data_ptr(),
                sma.PREC[precision], stream.cuda_stream)
        assert rc == 0, L.sma_last_error().decode()
        stream.synchronize()
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
