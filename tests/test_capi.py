"""C-ABI checks that need no GPU: the library loads, exports every entry
point include/alya_sma.h declares, and rejects bad input before touching a
device (so a GPU-less host gets an error code, never a fallback)."""
import ctypes as C

import numpy as np
import pytest

import alya_sma_b200 as sma
from alya_sma_b200 import problem as P


def test_header_symbols_exported():
    names = sma.header_functions()
    assert len(names) >= 20
    L = sma.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in sma.lib().sma_version()


def _prob():
    return P.bar_40x4x4(nsteps=10)


def test_rejects_bad_connectivity():
    p = _prob()
    p.lnods = p.lnods.copy()
    p.lnods[3, 2] = p.npoin + 5
    with pytest.raises(sma.SmaError, match="lnods entry out of range"):
        sma.ExplicitSolid(p)


def test_rejects_bad_material():
    p = _prob()
    p.props = p.props.copy()
    p.props[0, 1] = 0.5
    with pytest.raises(sma.SmaError, match="nu"):
        sma.ExplicitSolid(p)


def test_rejects_rayleigh_beta_and_negative_alpha():
    """Stiffness-proportional (beta) damping is refused at the boundary rather
    than ignored; alpha must be >= 0."""
    import dataclasses
    p = dataclasses.replace(_prob(), dampi=np.array([[0.0, 1e-6]]))
    with pytest.raises(sma.SmaError, match="beta"):
        sma.ExplicitSolid(p)
    p = dataclasses.replace(_prob(), dampi=np.array([[-1.0, 0.0]]))
    with pytest.raises(sma.SmaError, match="alpha"):
        sma.ExplicitSolid(p)


def test_rejects_bad_precision_and_block():
    p = _prob()
    with pytest.raises(KeyError):
        sma.ExplicitSolid(p, precision="fp16")
    with pytest.raises(sma.SmaError, match="block"):
        sma.ExplicitSolid(p, block=100)


def test_null_arguments_are_errors():
    L = sma.lib()
    assert L.sma_ctx_create(None, None, None, None) == -1
    assert L.sma_explicit_step(None, 1) == -1
    assert L.sma_eval_law160(-1, None, C.c_double(0.0), None, None, None, None, None, None, 0, None) == -1
    assert L.sma_eval_law160_tangent(-1, None, C.c_double(0.0), None, None, None, None, None, None,
                                     None, None) == -1
    props = np.ascontiguousarray(P.nitinol_props(**P.NITI))
    assert L.sma_eval_law160_tangent(0, props.ctypes.data, C.c_double(0.0), None, None, None, None,
                                     None, None, None, None) == 0                 # n = 0: nothing to do
    assert L.sma_eval_law160_tangent(4, props.ctypes.data, C.c_double(0.0), None, None, None, None,
                                     None, None, None, None) == -1                # NULL device arrays


def test_rejects_empty_mesh():
    p = _prob()
    p.lnods = p.lnods[:0]
    with pytest.raises(sma.SmaError, match="empty mesh"):
        sma.ExplicitSolid(p)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(sma.SmaError, match="device"):
        sma.ExplicitSolid(_prob())


def test_surrogate_entry_points_reject_bad_input_before_the_device():
    """The surrogate's C-ABI calls check their arguments on the host first:
    NULL pointers, empty batches, an unaligned weight image, an out-of-range
    wait limit and a NULL context come back as SMA_ERR_ARG with no device
    call."""
    from alya_sma_b200 import surrogate as S
    ERR_ARG = -1                                   # SMA_ERR_ARG, include/alya_sma.h
    L = S._bind()
    st = C.c_int32(-1)
    assert L.sma_sur_wait_check(0, C.byref(st)) == ERR_ARG
    assert L.sma_sur_wait_check(1 << 21, C.byref(st)) == ERR_ARG
    assert L.sma_sur_wait_check(10, None) == ERR_ARG
    assert L.sma_sur_forward(None, None, 0, None, None, None, None, None) == ERR_ARG
    assert L.sma_sur_forward(C.c_void_p(16), C.c_void_p(16), 8, None, None, None, None, None) == ERR_ARG
    assert L.sma_sur_forward(C.c_void_p(17), C.c_void_p(16), 8, C.c_void_p(16), C.c_void_p(16), None,
                             C.c_void_p(16), None) == ERR_ARG
    assert b"aligned" in L.sma_last_error()
    L.sma_set_surrogate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                    C.c_int32, C.c_int32]
    assert L.sma_set_surrogate(None, None, None, 3.0, 1e-3, 10.0, 64, 1) == ERR_ARG
    L.sma_launch_info.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    assert L.sma_launch_info(None, None, None, None) == ERR_ARG
