"""Shared test helpers: seeded inputs and comparisons."""
import numpy as np

from oracle import oracle as O


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    n = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0)


def oracle_grid(g):
    """oracle.Grid-like object from a workload grid dict."""
    class G:
        pass
    o = G()
    for k in ("nx", "ny", "nz", "xl", "yl", "zl", "x", "x12", "y", "y12", "z", "z12",
              "dx", "dx12", "dy", "dy12", "dz", "dz12"):
        setattr(o, k, g[k])
    return o


def rand_field(rng, nx, ny, nz, scale=1.0):
    return np.asfortranarray(scale * rng.standard_normal((nx + 2, ny + 2, nz + 2)))


def bit_equal(a, b):
    """Equal as IEEE bit patterns (NaN == NaN, -0 != +0 is ignored)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def maxdiff(a, b):
    return float(np.nanmax(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0
