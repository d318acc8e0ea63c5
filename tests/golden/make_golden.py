"""Generate the golden fixtures of tests/golden from the CPU oracle.

The reference (DominikHenzel/vtkmakeCompare) ships no golden vectors and its
Fortran + FFTW build is not available in this image, so these fixtures are
outputs of the oracle (oracle/nse_oracle.cpp) on small seeded inputs.  They
freeze the oracle's behaviour (tests/test_oracle.py regenerates and compares
bit for bit) and give the GPU tests fixed expected values.

    python tests/golden/make_golden.py      # rewrites the .npz files
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def _grid(nx, ny, nz):
    return O.Grid(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)


def _rand(rng, g):
    return np.asfortranarray(rng.standard_normal((g.nx + 2, g.ny + 2, g.nz + 2)))


def case_p2s():
    nx, ny, nz = 12, 4, 10
    rng = np.random.default_rng(101)
    FP = np.asfortranarray(rng.standard_normal((nx + 2, ny + 2, nz + 2)))
    FPT = O.p2s(FP, nx, ny, nz)
    back = O.s2p(FPT, nx, ny, nz)
    return {"FP": FP, "FPT": FPT, "back": back}


def case_mkp():
    g = _grid(10, 8, 6)
    rng = np.random.default_rng(102)
    names = ("p", "u_temp", "v_temp", "w_temp", "u_ta", "v_ta", "w_ta", "u_ep2", "v_ep2",
             "w_ep2", "divu", "u", "v", "w")
    f = {k: _rand(rng, g) for k in names}
    out = {"in_" + k: v.copy(order="F") for k, v in f.items()}
    O.mkp(g, f["p"], f["u_temp"], f["v_temp"], f["w_temp"], 0.02, f["u_ta"], f["v_ta"],
          f["w_ta"], f["u_ep2"], f["v_ep2"], f["w_ep2"], f["divu"], f["u"], f["v"], f["w"])
    out.update({"out_" + k: v for k, v in f.items()})
    return out


def case_lines():
    rng = np.random.default_rng(103)
    n = 20
    g = _grid(n, n, n)
    Re, Sc, dt, eta = 200.0, 0.71, 0.01, 1.0e4
    cu = rng.random(n)
    cu[cu < 0.5] = 0.0
    s0 = rng.standard_normal(n + 2)
    ll = 0.5 + rng.random(n + 2)
    rr = 0.5 + rng.random(n + 2)
    cu2 = np.concatenate([[0.0], cu, [0.0]])
    out = {"s0": s0, "cu": cu, "ll": ll, "rr": rr}
    a = s0.copy()
    O.implicit_solver(a, n, g.dx, g.dx12, Re, dt, 0.0, 0.0, eta, cu)
    out["solver"] = a
    a = s0.copy()
    O.implicit_uy(a, n, g.dy, g.dy12, Re, dt, 0.0, 0.0, eta, cu)
    out["uy"] = a
    a = s0.copy()
    O.implicit_vy(a, n, g.dy, g.dy12, Re, dt, 0.0, 0.0, eta, cu)
    out["vy"] = a
    a = s0.copy()
    O.implicit_ty(a, n, g.dy, g.dy12, Re, Sc, dt, ll, rr, 2.0, 0.0, cu2, eta)
    out["ty"] = a
    a = s0.copy()
    O.implicit_tx(a, n, g.dx, g.dx12, Re, Sc, dt, ll, rr, 0.0, 0.0, eta, cu2)
    out["tx"] = a
    return out


def case_levelset():
    nx, ny, nz = 12, 10, 8
    g = _grid(nx, ny, nz)
    X, Y, Z = np.meshgrid(g.x[1:-1], g.y[1:-1], g.z[1:-1], indexing="ij")
    phi0 = O.field(nx, ny, nz)
    phi0[1:-1, 1:-1, 1:-1] = 0.9 - np.sqrt((X - math.pi) ** 2 + Y ** 2 + (Z - 1.5) ** 2)
    phi, cv = O.set_levelset(g, phi0, nnn=40, width=1.5)
    return {"phi0": phi0, "phi": phi, "c1": np.asfortranarray(cv[..., 0])}


def case_step():
    nx, ny, nz = 16, 12, 8
    g = _grid(nx, ny, nz)
    rng = np.random.default_rng(104)
    Re = 3000.0
    s = O.Solver(g, 0.01, Re, 0.71, 1.0e4, force=3.0 / Re, source=0.0, tbot=1.0, ttop=0.0,
                 tsolid=1.0)
    yy = g.y[1:-1]
    s.f["u"][1:-1, 1:-1, 1:-1] = (1.5 * (1 - yy ** 2))[None, :, None] + \
        0.05 * rng.standard_normal((nx, ny, nz))
    s.f["v"][1:-1, 1:-1, 1:-1] = 0.05 * rng.standard_normal((nx, ny, nz))
    s.f["v"][:, ny, :] = 0.0
    s.f["w"][1:-1, 1:-1, 1:-1] = 0.05 * rng.standard_normal((nx, ny, nz))
    s.f["T"][1:-1, 1:-1, 1:-1] = ((1 - yy) / 2)[None, :, None]
    X, Y, Z = np.meshgrid(g.x[1:-1], g.y[1:-1], g.z[1:-1], indexing="ij")
    r = np.sqrt((X - math.pi) ** 2 + Y ** 2 + (Z - math.pi / 2) ** 2)
    s.cellvalue[..., 0] = np.clip((0.6 - r) / 0.3 + 0.5, 0.0, 1.0)
    out = {"in_" + k: s.f[k].copy(order="F") for k in ("u", "v", "w", "T")}
    out["c1"] = s.cellvalue[..., 0].copy(order="F")
    s.start()
    s.step(3)
    for k in ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre",
              "T_pre", "divu"):
        out["out_" + k] = s.f[k].copy(order="F")
    return out


CASES = {"p2s": case_p2s, "mkp": case_mkp, "lines": case_lines, "levelset": case_levelset,
         "step": case_step}


if __name__ == "__main__":
    for name, fn in CASES.items():
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fn())
        print(path, os.path.getsize(path))
