"""The C ABI from a compiled C program (tests/c/sma_c_client.c), the way a
Fortran bind(C) caller uses it: compiled with gcc against include/alya_sma.h
and the shipped library.  Its argument checks run without a GPU; on a GPU its
100-step run must equal, bit for bit, the same run through the Python mirror
(FP64, coloured scatter: deterministic)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import alya_sma_b200 as sma
from alya_sma_b200 import problem as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def client(tmp_path_factory):
    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    libdir = os.path.join(ROOT, "alya_sma_b200")
    assert os.path.exists(os.path.join(libdir, "libalya_sma_b200.so")), "build the library first"
    exe = str(tmp_path_factory.mktemp("cclient") / "sma_c_client")
    cmd = [gcc, "-O2", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c", "sma_c_client.c"), "-L", libdir, "-lalya_sma_b200",
           f"-Wl,-rpath,{libdir}", "-lm", "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def test_c_client_argument_checks(client):
    res = subprocess.run([client, "reject"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "reject ok" in res.stdout


@pytest.mark.gpu
def test_c_client_run_equals_python_mirror(client, tmp_path):
    out = tmp_path / "c_run.bin"
    res = subprocess.run([client, "run", str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    raw = np.fromfile(out, dtype=np.float64)
    dt, u_c = raw[0], raw[1:].reshape(-1, 3)
    # the same bar through the Python mirror of the ABI
    coord, lnods = P.structured_box(8, 2, 2, 8.0, 2.0, 2.0)
    props = np.zeros((1, 18))
    props[0, :11] = [60000.0, 0.33, 0.05 * np.sqrt(1.5), 400.0, 500.0, 0, 0, 0, 0, 250.0, 150.0]
    npoin = coord.shape[0]
    fixno = np.zeros((npoin, 3), np.int32)
    bcfun = np.full(npoin, -1, np.int32)
    fixno[coord[:, 0] == 0.0] = 1
    tip = coord[:, 0] == 8.0
    fixno[tip, 0] = 1
    bcfun[tip] = 0
    T = 200 * dt
    tab = np.array([[0.0, 0.0, 0.0, 0.0], [0.5 * T, 0.4, 0.4, 0.4], [T, 0.0, 0.0, 0.0]])
    p = P.Problem(coord=coord, lnods=lnods, props=props, e_mart=np.zeros(1), densi=np.array([6.45e-9]),
                  fixno=fixno, bcfun=bcfun, fun_npts=np.array([3], np.int32),
                  fun_smooth=np.array([1], np.int32), fun_tab=tab, dtime=dt, nsteps=100)
    g = sma.ExplicitSolid(p, precision="fp64", scatter="color")
    g.step(100)
    u_py = g.get("displ")
    assert np.abs(u_c).max() > 0.0
    assert np.array_equal(u_c, u_py)
