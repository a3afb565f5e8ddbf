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
