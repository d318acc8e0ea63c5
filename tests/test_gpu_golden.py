"""GPU path against the committed golden fixtures (tests/golden/*.npz,
generated by tests/golden/make_golden.py from the oracle)."""
import math
import os

import numpy as np
import pytest

from tests._helpers import bit_equal, rel_l2
from vtkmakecompare_b200 import legacy as G
from vtkmakecompare_b200 import solver as S
from vtkmakecompare_b200 import workload as W

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(HERE, name + ".npz"))


def grid(nx, ny, nz):
    return W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)


def test_golden_p2s():
    d = load("p2s")
    nx, ny, nz = 12, 4, 10
    FPT = np.zeros_like(d["FPT"], order="F")
    G.p2s(np.asfortranarray(d["FP"]), FPT, nx, ny, nz)
    sl = (slice(None), slice(1, ny + 1), slice(0, nz))
    assert rel_l2(FPT[sl], d["FPT"][sl]) < 1e-14


def test_golden_mkp():
    d = load("mkp")
    nx, ny, nz = 10, 8, 6
    g = grid(nx, ny, nz)
    f = {k[3:]: np.asfortranarray(d[k]).copy(order="F") for k in d.files if k.startswith("in_")}
    G.mkp(f["p"], f["u_temp"], f["v_temp"], f["w_temp"], 0.02, g["dx"], g["dy"], g["dz"],
          g["dx12"], g["dy12"], g["dz12"], 1.0, nx, ny, nz, 1, f["u_ta"], f["v_ta"], f["w_ta"],
          f["u_ep2"], f["v_ep2"], f["w_ep2"], f["divu"], f["u"], f["v"], f["w"], g["xl"],
          g["zl"])
    for k in f:
        assert rel_l2(f[k], d["out_" + k]) < 1e-12, k


def test_golden_lines():
    d = load("lines")
    n = 20
    g = grid(n, n, n)
    Re, Sc, dt, eta = 200.0, 0.71, 0.01, 1.0e4
    cu, s0, ll, rr = d["cu"], d["s0"], d["ll"], d["rr"]
    cu2 = np.concatenate([[0.0], cu, [0.0]])
    a = s0.copy()
    G.implicit_solver(a, n, g["dx"], g["dx12"], Re, dt, 0.0, 0.0, eta, cu)
    assert bit_equal(a, d["solver"])
    a = s0.copy()
    G.implicit_uy(a, n, g["dy"], g["dy12"], Re, dt, 0.0, 0.0, eta, cu)
    assert bit_equal(a, d["uy"])
    a = s0.copy()
    G.implicit_vy(a, n, g["dy"], g["dy12"], Re, dt, 0.0, 0.0, eta, cu)
    assert bit_equal(a, d["vy"])
    a = s0.copy()
    G.implicit_ty(a, n, g["dy"], g["dy12"], Re, Sc, dt, ll, rr, 2.0, 0.0, cu2, eta)
    assert bit_equal(a, d["ty"])
    a = s0.copy()
    G.implicit_tx(a, n, g["dx"], g["dx12"], Re, Sc, dt, ll, rr, 0.0, 0.0, eta, cu2)
    assert bit_equal(a, d["tx"])


def test_golden_levelset():
    d = load("levelset")
    nx, ny, nz = 12, 10, 8
    cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0)
    with S.Context(cfg) as ctx:
        phi = ctx.levelset(d["phi0"], nnn=40, width=1.5)
        c1 = ctx.download("cellvalue")
    assert bit_equal(phi, d["phi"])
    assert np.abs(c1 - d["c1"]).max() < 4e-16


def test_golden_step():
    d = load("step")
    nx, ny, nz = 16, 12, 8
    Re = 3000.0
    cfg = S.Config(nx, ny, nz, 0.01, Re, 0.71, 1.0e4, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0, body_force=3.0 / Re, heat_source=0.0, t_bot=1.0, t_top=0.0,
                   t_solid=1.0)
    with S.Context(cfg) as ctx:
        for k in ("u", "v", "w", "T"):
            ctx.upload(k, d["in_" + k])
        ctx.upload("cellvalue", d["c1"])
        ctx.start()
        ctx.step(3)
        for k in ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre",
                  "T_pre"):
            assert rel_l2(ctx.download(k), d["out_" + k]) < 1e-10, k
        # the divergence is round-off in both: compare absolutely
        assert np.abs(ctx.download("divu") - d["out_divu"]).max() < 1e-11
