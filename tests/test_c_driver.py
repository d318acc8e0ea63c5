"""tests/c_driver.c, a C restatement of the reference driver's time loop that
calls libnsegpu.so through include/nsegpu.h only: it compiles warning-free
against the header (CPU), and on the GPU its fields after a few steps equal
the CPU oracle's restatement of the same loop (nse_dominik.f:246-446 with the
reference's own parameters: body force and heat source 1, walls at T = 0,
uniform grid).

Tolerance: the tier-2 routines round like the oracle; MKP's transforms differ
at the 1e-15 level, so the fields after N steps agree within 1e-10 relative L2.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import rel_l2
from vtkmakecompare_b200 import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_driver.c")


def compile_driver(out_dir):
    exe = os.path.join(out_dir, "c_driver")
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror", "-I",
           os.path.join(ROOT, "include"), SRC, "-o", exe, LIB_PATH,
           "-Wl,-rpath," + os.path.dirname(LIB_PATH)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_c_driver_compiles_against_the_header(tmp_path):
    exe = compile_driver(str(tmp_path))
    assert os.path.exists(exe)


def write_input(path, nx, ny, nz, nsteps, par, f, c1):
    with open(path, "wb") as fh:
        np.array([nx, ny, nz, nsteps], dtype=np.int32).tofile(fh)
        np.array(par, dtype=np.float64).tofile(fh)
        for k in ("u", "v", "w", "T"):
            np.asfortranarray(f[k]).ravel(order="F").tofile(fh)
        np.asfortranarray(c1).ravel(order="F").tofile(fh)


@pytest.mark.gpu
@pytest.mark.parametrize("n,nsteps", [((16, 12, 10), 4), ((32, 24, 16), 3)])
def test_c_driver_time_loop_matches_oracle(tmp_path, n, nsteps):
    nx, ny, nz = n
    dt, Re, Sc, eta, xl, yl, zl = 2.0e-3, 200.0, 0.71, 1.0e3, 2.0, 1.0, 1.5
    rng = np.random.default_rng(31)
    f = {}
    for k in ("u", "v", "w", "T"):
        a = np.zeros((nx + 2, ny + 2, nz + 2), order="F")
        a[1:-1, 1:-1, 1:-1] = 0.1 * rng.standard_normal((nx, ny, nz))
        f[k] = a
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    r = np.sqrt((X - nx / 2) ** 2 + (Y - ny / 2) ** 2 + (Z - nz / 2) ** 2)
    c1 = np.asfortranarray(np.clip((3.0 - r) / 2.0, 0.0, 1.0))
    exe = compile_driver(str(tmp_path))
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    write_input(inp, nx, ny, nz, nsteps, (dt, Re, Sc, eta, xl, yl, zl), f, c1)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = (nx + 2) * (ny + 2) * (nz + 2)
    got = np.fromfile(out, dtype=np.float64).reshape(5, m)
    g = O.Grid(nx, ny, nz, xl, yl, zl)
    s = O.Solver(g, dt, Re, Sc, eta)
    for k in ("u", "v", "w", "T"):
        s.f[k][...] = f[k]
    s.cellvalue[..., 0] = c1
    s.start()
    s.step(nsteps)
    for q, k in enumerate(("u", "v", "w", "p", "T")):
        ref = s.f[k].ravel(order="F")
        assert rel_l2(got[q], ref) < 1e-10, k
