"""Synthetic channel workloads (seeded) in the reference's variables.

The channel is periodic in x and z (lengths xl, zl) with walls at y = y0 and
y = y0 + yl.  Mapping of the benchmark description onto the reference:

* Re_bulk -> Re, Pr -> Sc (nse_dominik.f:6, used at :999, :1736, :1794)
* body force F = 3/Re so that u = 1.5(1 - y^2) is the laminar state for
  walls at y = -1, 1 (the reference hard-codes 1.0, nse_dominik.f:785)
* heat source Q = 0 (reference 1.0, :879); wall temperatures T(y=-1) = 1,
  T(y=1) = 0 through the ghost rule T0 = 2 Tw - T1 (reference Tw = 0)
* penalisation permeability 1e-4 -> eta = 1e4 (the reference's eta is the
  inverse permeability, eta = 1e2/dt at :15)
* level set phi = R - |x - c| (positive inside the solid, the reference's
  convention, set_levelset.f:160-166); "no obstacle" -> mask c1 = 0
* CFL 0.5 -> one fixed dt = 0.5 / max(|u|/dx + |v|/dy + |w|/dz) from the
  initial field (the reference uses a fixed dt and only reports Courant).
"""
import ctypes as C
import math

import numpy as np

from . import lib


def grid_arrays(nx, ny, nz, xl, yl, zl, y0=0.0, gamma=0.0):
    """SET_C (nse_dominik.f:553-607) or its tanh-stretched y variant, computed by
    the library's host routine nse_set_c_stretched."""
    g = {k: np.zeros(n + 2) for k, n in (("x", nx), ("x12", nx), ("y", ny), ("y12", ny),
                                        ("z", nz), ("z12", nz), ("dx", nx), ("dx12", nx),
                                        ("dy", ny), ("dy12", ny), ("dz", nz), ("dz12", nz))}
    L = lib()
    L.nse_set_c_stretched.argtypes = [C.c_int] * 3 + [C.c_void_p] * 12 + [C.c_double] * 5
    L.nse_set_c_stretched(nx, ny, nz, *[g[k].ctypes.data for k in
                                        ("x", "x12", "y", "y12", "z", "z12", "dx", "dx12", "dy",
                                         "dy12", "dz", "dz12")], xl, yl, zl, y0, gamma)
    g.update(nx=nx, ny=ny, nz=nz, xl=xl, yl=yl, zl=zl)
    return g


def padded(g, fill=0.0):
    return np.full((g["nx"] + 2, g["ny"] + 2, g["nz"] + 2), fill, order="F")


def sphere_phi0(g, center, radius):
    """phi0 = R - |x - c| at cell centres (interior), zero ghosts (as readgrid3d
    leaves them)."""
    phi0 = padded(g)
    X = g["x"][1:-1, None, None]
    Y = g["y"][None, 1:-1, None]
    Z = g["z"][None, None, 1:-1]
    phi0[1:-1, 1:-1, 1:-1] = radius - np.sqrt((X - center[0]) ** 2 + (Y - center[1]) ** 2 +
                                              (Z - center[2]) ** 2)
    return phi0


def smoothed_mask(g, phi0, width):
    """Cell mask c1 of set_levelset.f:157-170 applied directly to a level set
    phi0 (padded, interior used) that is already a signed distance, without
    the reinitialisation sweeps: 1 where phi >= w*dx_i, 0 where phi <= -w*dx_i,
    (sin(pi phi / (2 w dx_i)) + 1)/2 between, with the reference's
    pi = 3.1415926535 (set_levelset.f:7).  numpy only (no library call), so
    the GPU run and the CPU reference run start from the same mask."""
    phi = phi0[1:-1, 1:-1, 1:-1]
    h = width * g["dx"][1:-1, None, None]
    c = (np.sin(3.1415926535 * phi / 2.0 / h) + 1.0) / 2.0
    return np.asfortranarray(np.where(phi >= h, 1.0, np.where(phi <= -h, 0.0, c)))


def channel_state(g, seed, noise=0.05, t_bot=1.0, t_top=0.0, bulk=True):
    """u = 1.5(1 - y^2) + N(0, noise^2), v, w ~ N(0, noise^2) on interior cells
    (y measured so that the walls are at -1, 1), T linear from t_bot to t_top."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    y0 = g["y12"][0]
    yl = g["y12"][ny] - y0
    eta_y = 2.0 * (g["y"][1:-1] - y0) / yl - 1.0  # in [-1, 1]
    f = {k: padded(g) for k in ("u", "v", "w", "T")}
    base = 1.5 * (1.0 - eta_y ** 2) if bulk else np.zeros(ny)
    f["u"][1:-1, 1:-1, 1:-1] = base[None, :, None] + noise * rng.standard_normal((nx, ny, nz))
    f["v"][1:-1, 1:-1, 1:-1] = noise * rng.standard_normal((nx, ny, nz))
    f["w"][1:-1, 1:-1, 1:-1] = noise * rng.standard_normal((nx, ny, nz))
    f["v"][:, ny, :] = 0.0
    f["T"][1:-1, 1:-1, 1:-1] = (t_bot + (t_top - t_bot) * (eta_y + 1.0) / 2.0)[None, :, None]
    return f


def cfl_dt(g, u, v, w, cfl=0.5):
    s = (np.abs(u[1:-1, 1:-1, 1:-1]) / g["dx"][1:-1, None, None] +
         np.abs(v[1:-1, 1:-1, 1:-1]) / g["dy"][None, 1:-1, None] +
         np.abs(w[1:-1, 1:-1, 1:-1]) / g["dz"][None, None, 1:-1])
    return cfl / float(s.max())


def poisson_rhs(g, seed):
    """Seeded N(0,1) right-hand side with its dy-weighted plane mean removed
    (so the mean-mode marching of SP0B, mkp.f:284-287, stays compatible),
    periodic sample fill as in MKP (mkp.f:101-121)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    f = padded(g)
    r = rng.standard_normal((nx, ny, nz))
    dy = g["dy"][1:-1]
    r -= (r.mean(axis=(0, 2)) * dy).sum() / dy.sum()
    f[1:-1, 1:-1, 1:-1] = r
    f[1:nx + 1, 1:ny + 1, 0] = f[1:nx + 1, 1:ny + 1, nz]
    f[0, 1:ny + 1, 1:nz + 1] = f[nx, 1:ny + 1, 1:nz + 1]
    f[0, 1:ny + 1, 0] = f[nx, 1:ny + 1, nz]
    return f


# named workloads of the benchmark description (sizes, geometry, physics)
CONFIGS = {
    "channel64": dict(nx=64, ny=64, nz=64, Re=3000.0, Pr=0.71, sphere=None, steps=10),
    "sphere256": dict(nx=256, ny=192, nz=256, Re=3000.0, Pr=0.71,
                      sphere=((math.pi, 0.0, math.pi / 2), 0.25), eta=1.0e4, width=1.5,
                      t_solid=1.0, steps=200),
}


# ---------------------------------------------------------------- ensemble
# grids of the ensemble workload (cases drawn uniformly among them)
ENSEMBLE_GRIDS = ((64, 64, 64), (96, 64, 96), (128, 96, 128), (160, 128, 160))


def box_phi0(g, center, half):
    """phi0 = minus the signed distance to an axis-aligned cube of half-side
    `half` (positive inside, the reference's sign), interior cells."""
    phi0 = padded(g)
    X = g["x"][1:-1, None, None]
    Y = g["y"][None, 1:-1, None]
    Z = g["z"][None, None, 1:-1]
    q = [np.abs(X - center[0]) - half, np.abs(Y - center[1]) - half,
         np.abs(Z - center[2]) - half]
    q = np.broadcast_arrays(*q)
    outside = np.sqrt(sum(np.maximum(a, 0.0) ** 2 for a in q))
    inside = np.minimum(np.maximum(np.maximum(q[0], q[1]), q[2]), 0.0)
    phi0[1:-1, 1:-1, 1:-1] = -(outside + inside)
    return phi0


def ensemble_case(seed):
    """One case of the batched ensemble: a grid drawn among ENSEMBLE_GRIDS,
    1-3 spheres or cubes (radius or half-side 0.1-0.3) at seeded positions in
    the 2pi x 2 x pi channel, Re_bulk uniform in [1000, 5000], its own noise.
    Returns (grid, fields, phi0, Re, obstacles)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = ENSEMBLE_GRIDS[int(rng.integers(len(ENSEMBLE_GRIDS)))]
    g = grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = channel_state(g, seed=int(rng.integers(1 << 30)), t_bot=1.0, t_top=0.0)
    Re = float(rng.uniform(1000.0, 5000.0))
    obst = []
    phi0 = None
    for _ in range(int(rng.integers(1, 4))):
        size = float(rng.uniform(0.1, 0.3))
        c = (float(rng.uniform(0, 2 * math.pi)), float(rng.uniform(-1 + size + 0.1, 1 - size - 0.1)),
             float(rng.uniform(0, math.pi)))
        kind = "sphere" if rng.random() < 0.5 else "box"
        p = sphere_phi0(g, c, size) if kind == "sphere" else box_phi0(g, c, size)
        phi0 = p if phi0 is None else np.maximum(phi0, p)
        obst.append((kind, c, size))
    return g, f, np.asfortranarray(phi0), Re, obst

