"""Pins of the CPU oracle (no GPU).

The reference ships no tests or golden vectors, so the oracle is pinned by
known answers that follow from the reference's own mathematics:
* the FFT restatement against numpy.fft (pocketfft) and a direct DFT;
* every line solver against a dense numpy solve of the matrix the reference
  assembles (implicit_uy/vy/Ty rows, the augmented cyclic system, SPN's
  Neumann-folded system);
* a manufactured discrete Poisson solution (P2S->SPN->SP0B->S2P inverts the
  7-point operator of solve_p, nse_dominik.f:1988-1993, with PHIBC ghosts);
* the laminar Poiseuille profile of check_convergence (nse_dominik.f:2883);
* the committed golden fixtures (tests/golden, made by make_golden.py).
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))


def dft2_half(plane):
    """direct O(N^2) r2c DFT of plane[i, k] (i = x), kx = 0..NX/2, sign -1"""
    NX, NZ = plane.shape
    i = np.arange(NX)
    k = np.arange(NZ)
    Ex = np.exp(-2j * np.pi * np.outer(np.arange(NX // 2 + 1), i) / NX)
    Ez = np.exp(-2j * np.pi * np.outer(k, k) / NZ)
    return Ex @ plane @ Ez.T


@pytest.mark.parametrize("n", [(8, 3, 6), (12, 2, 10), (96, 2, 20), (30, 2, 160)])
def test_p2s_matches_numpy_and_dft(n):
    nx, ny, nz = n
    rng = np.random.default_rng(1)
    FP = O.field(nx, ny, nz)
    FP[...] = rng.standard_normal(FP.shape)
    FPT = O.p2s(FP, nx, ny, nz)
    for J in range(1, ny + 1):
        pl = FP[0:nx, J, 0:nz]
        ref = np.fft.rfft2(pl.T).T / (nx * nz)
        assert np.abs(FPT[:, J, 0:nz] - ref).max() < 1e-14
        if nx * nz <= 2000:
            assert np.abs(FPT[:, J, 0:nz] - dft2_half(pl) / (nx * nz)).max() < 1e-13
    back = O.s2p(FPT, nx, ny, nz)
    assert np.abs(back[0:nx, 1:ny + 1, 0:nz] - FP[0:nx, 1:ny + 1, 0:nz]).max() < 1e-13
    # the S2P wrap (p2s_fftw2d.f:211-216)
    assert np.array_equal(back[nx, 1:ny + 1, 0:nz + 1], back[0, 1:ny + 1, 0:nz + 1])
    assert np.array_equal(back[0:nx + 1, 1:ny + 1, nz], back[0:nx + 1, 1:ny + 1, 0])


def test_s2p_is_c2r_of_hermitian_extension():
    nx, ny, nz = 8, 1, 6
    rng = np.random.default_rng(2)
    FPT = np.zeros((nx // 2 + 1, ny + 2, nz + 2), complex, order="F")
    FPT[:, 1, 0:nz] = rng.standard_normal((5, nz)) + 1j * rng.standard_normal((5, nz))
    FP = O.s2p(FPT, nx, ny, nz)
    ref = np.fft.irfft2(FPT[:, 1, 0:nz].T, s=(nz, nx)).T * (nx * nz)
    assert np.abs(FP[0:nx, 1, 0:nz] - ref).max() < 1e-12


def test_ctridiag_tridiag_trid2_dense():
    rng = np.random.default_rng(3)
    NN = 11
    A = np.asfortranarray(rng.standard_normal((NN, 3)))
    A[:, 1] += 5.0
    M = np.diag(A[:, 1]) + np.diag(A[1:, 0], -1) + np.diag(A[:-1, 2], 1)
    B = rng.standard_normal(NN) + 1j * rng.standard_normal(NN)
    A1, B1 = A.copy(order="F"), B.copy()
    O.ctridiag(A1, B1)
    assert np.abs(B1 - np.linalg.solve(M, B)).max() < 1e-13
    Br = B.real.copy()
    A1 = A.copy(order="F")
    O.tridiag(A1, Br)
    assert np.abs(Br - np.linalg.solve(M, B.real)).max() < 1e-13
    BB = np.asfortranarray(rng.standard_normal((4, NN)))
    A1 = A.copy(order="F")
    X = BB.copy(order="F")
    O.trid2(A1, X)
    assert np.abs(X - np.linalg.solve(M, BB.T).T).max() < 1e-13


def test_cyclic_is_the_periodic_system():
    """implicit_solver's augmented system (periodic_implicit.f:1-44) equals the
    periodic tridiagonal system on 1..n with x0 = xn, x(n+1) = x1."""
    rng = np.random.default_rng(4)
    n = 9
    g = O.Grid(n, 4, 4, 2 * math.pi, 1.0, 1.0)
    Re, dt, eta = 50.0, 0.05, 30.0
    cux = rng.random(n)
    s = np.zeros(n + 2)
    s[1:n + 1] = rng.standard_normal(n)
    rhs = s[1:n + 1].copy()
    O.implicit_solver(s, n, g.dx, g.dx12, Re, dt, 0.0, 0.0, eta, cux)
    beta = dt / Re / 2
    M = np.zeros((n, n))
    for i in range(1, n + 1):
        al = dt * eta * cux[i - 1] + 1
        a = -beta / al / g.dx[i] / g.dx12[i]
        c = -beta / al / g.dx[i + 1] / g.dx12[i]
        b = 1 + beta / al * (1 / g.dx[i + 1] + 1 / g.dx[i]) / g.dx12[i]
        M[i - 1, i - 1] += b
        M[i - 1, (i - 2) % n] += a
        M[i - 1, i % n] += c
    x = np.linalg.solve(M, rhs)
    assert np.abs(s[1:n + 1] - x).max() < 1e-13
    assert abs(s[0] - s[n]) < 1e-13 and abs(s[n + 1] - s[1]) < 1e-13


def test_ul_solvers_match_dense():
    rng = np.random.default_rng(5)
    ny = 10
    g = O.Grid(4, ny, 4, 1.0, 2.0, 1.0, y0=-1.0, gamma=2.0)
    Re, dt, eta = 30.0, 0.02, 100.0
    cu = rng.random(ny)
    s = rng.standard_normal(ny + 2)
    x = s.copy()
    O.implicit_uy(x, ny, g.dy, g.dy12, Re, dt, 0.3, -0.2, eta, cu)
    beta = dt / Re / 2
    M = np.zeros((ny + 2, ny + 2))
    r = np.zeros(ny + 2)
    M[0, 0] = M[0, 1] = 1.0
    M[ny + 1, ny + 1] = M[ny + 1, ny] = 1.0
    r[0], r[ny + 1] = 0.3, -0.2
    for j in range(1, ny + 1):
        al = dt * eta * cu[j - 1] + 1
        M[j, j - 1] = -beta / al / g.dy12[j - 1] / g.dy[j]
        M[j, j] = 1 + beta / al * (1 / g.dy12[j] + 1 / g.dy12[j - 1]) / g.dy[j]
        M[j, j + 1] = -beta / al / g.dy12[j] / g.dy[j]
        r[j] = s[j]
    assert np.abs(x - np.linalg.solve(M, r)).max() < 1e-13
    # implicit_vy: rows 0..ny with Dirichlet rows 0 and ny
    x = s.copy()
    O.implicit_vy(x, ny, g.dy, g.dy12, Re, dt, 0.0, 0.0, eta, cu)
    M = np.zeros((ny + 1, ny + 1))
    r = np.zeros(ny + 1)
    M[0, 0] = M[ny, ny] = 1.0
    for j in range(1, ny):
        al = dt * eta * cu[j - 1] + 1
        M[j, j - 1] = -beta / al / g.dy[j] / g.dy12[j]
        M[j, j] = 1 + beta / al * (1 / g.dy[j + 1] + 1 / g.dy[j]) / g.dy12[j]
        M[j, j + 1] = -beta / al / g.dy[j + 1] / g.dy12[j]
        r[j] = s[j]
    assert np.abs(x[:ny + 1] - np.linalg.solve(M, r)).max() < 1e-13


def lap(g, P):
    nx, ny, nz = g.nx, g.ny, g.nz
    i, j, k = slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1)
    X = ((P[2:nx + 2, j, k] - P[i, j, k]) / g.dx12[1:nx + 1, None, None] -
         (P[i, j, k] - P[0:nx, j, k]) / g.dx12[0:nx, None, None]) / g.dx[1:nx + 1, None, None]
    Y = ((P[i, 2:ny + 2, k] - P[i, j, k]) / g.dy12[None, 1:ny + 1, None] -
         (P[i, j, k] - P[i, 0:ny, k]) / g.dy12[None, 0:ny, None]) / g.dy[None, 1:ny + 1, None]
    Z = ((P[i, j, 2:nz + 2] - P[i, j, k]) / g.dz12[None, None, 1:nz + 1] -
         (P[i, j, k] - P[i, j, 0:nz]) / g.dz12[None, None, 0:nz]) / g.dz[None, None, 1:nz + 1]
    return X + Y + Z


@pytest.mark.parametrize("n,gam", [((16, 8, 12), 0.0), ((32, 24, 20), 2.0), ((30, 10, 18), 2.0)])
def test_manufactured_poisson(n, gam):
    nx, ny, nz = n
    g = O.Grid(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=gam)
    rng = np.random.default_rng(6)
    phi = O.field(nx, ny, nz)
    phi[1:-1, 1:-1, 1:-1] = rng.standard_normal((nx, ny, nz))
    phi[1:-1, 1:-1, 1:-1] -= phi[1:-1, 1, 1:-1].mean()
    O.phibc(nx, ny, nz, phi)
    f = O.field(nx, ny, nz)
    f[1:-1, 1:-1, 1:-1] = lap(g, phi)
    f[1:nx + 1, 1:ny + 1, 0] = f[1:nx + 1, 1:ny + 1, nz]
    f[0, 1:ny + 1, 1:nz + 1] = f[nx, 1:ny + 1, 1:nz + 1]
    f[0, 1:ny + 1, 0] = f[nx, 1:ny + 1, nz]
    AC, KXZ = O.mkp_coeffs(g)
    PT = O.p2s(f, nx, ny, nz)
    O.spn(nx, ny, nz, AC, KXZ, PT)
    O.sp0b(nx, ny, nz, AC, PT)
    sol = O.s2p(PT, nx, ny, nz)
    O.phibc(nx, ny, nz, sol)
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    assert rel_l2(sol[I], phi[I]) < 1e-12


def test_mkp_projection_is_divergence_free():
    nx, ny, nz = 24, 16, 12
    g = O.Grid(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rng = np.random.default_rng(7)
    f = {k: O.field(nx, ny, nz) for k in ("p", "ut", "vt", "wt", "a", "b", "c", "e1", "e2",
                                           "e3", "divu", "u", "v", "w")}
    for k in ("ut", "vt", "wt"):
        f[k][1:-1, 1:-1, 1:-1] = rng.standard_normal((nx, ny, nz))
    f["vt"][:, ny, :] = 0.0
    f["vt"][:, 0, :] = 0.0
    for k in ("ut", "wt"):  # periodic ghosts of u*, w* (set_bc)
        a = f[k]
        a[0], a[nx + 1] = a[nx], a[1]
        a[:, :, 0], a[:, :, nz + 1] = a[:, :, nz], a[:, :, 1]
    a = f["vt"]
    a[0], a[nx + 1] = a[nx], a[1]
    a[:, :, 0], a[:, :, nz + 1] = a[:, :, nz], a[:, :, 1]
    O.mkp(g, f["p"], f["ut"], f["vt"], f["wt"], 0.01, f["a"], f["b"], f["c"], f["e1"], f["e2"],
          f["e3"], f["divu"], f["u"], f["v"], f["w"])
    assert np.abs(f["divu"][1:-1, 1:-1, 1:-1]).max() < 1e-11


def test_poiseuille_profile_is_steady_in_the_oracle():
    nx, ny, nz, Re, yl, dt = 4, 32, 4, 20.0, 4.0, 1.0e-3
    g = O.Grid(nx, ny, nz, 0.25, yl, 4.0)
    dy = yl / ny
    A = np.diag(-2.0 * np.ones(ny)) + np.diag(np.ones(ny - 1), 1) + np.diag(np.ones(ny - 1), -1)
    A[0, 0] -= 1
    A[-1, -1] -= 1
    us = np.linalg.solve(A / dy ** 2, -Re * np.ones(ny))
    s = O.Solver(g, dt, Re, 1.0, 0.0)
    s.f["u"][1:-1, 1:-1, 1:-1] = us[None, :, None]
    s.start()
    s.step(10)
    assert np.abs(s.f["u"][1:-1, 1:-1, 1:-1] - us[None, :, None]).max() < 1e-10 * us.max()
    y = g.y[1:-1]
    assert np.abs(us + Re / 2 * y * (y - yl)).max() < Re * dy ** 2


def test_levelset_keeps_a_signed_distance_and_nan_at_zero():
    nx, ny, nz = 16, 16, 16
    g = O.Grid(nx, ny, nz, 2.0, 2.0, 2.0)
    X, Y, Z = np.meshgrid(g.x[1:-1], g.y[1:-1], g.z[1:-1], indexing="ij")
    phi0 = O.field(nx, ny, nz)
    phi0[1:-1, 1:-1, 1:-1] = 0.55 - np.sqrt((X - 1) ** 2 + (Y - 1) ** 2 + (Z - 1) ** 2)
    phi, cv = O.set_levelset(g, phi0, nnn=200)
    inner = np.abs(phi0[1:-1, 1:-1, 1:-1]) < 0.3
    assert np.abs(phi[1:-1, 1:-1, 1:-1][inner] - phi0[1:-1, 1:-1, 1:-1][inner]).max() < 0.05
    c = cv[..., 0]
    assert c.min() >= 0.0 and c.max() <= 1.0 and c[8, 8, 8] == 1.0 and c[0, 0, 0] == 0.0
    # epsilon = 1.0d0-1 = 0 (set_levelset.f:6): S(0) = 0/0 = NaN, as in the reference
    phi0[5, 5, 5] = 0.0
    phi, cv = O.set_levelset(g, phi0, nnn=0)
    assert np.isnan(phi[5, 5, 5]) and np.isnan(cv[4, 4, 4, 0])


GOLDEN = sorted(f for f in os.listdir(os.path.join(HERE, "golden")) if f.endswith(".npz"))


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_reproduces_golden(name):
    from tests.golden import make_golden
    d = np.load(os.path.join(HERE, "golden", name))
    out = make_golden.CASES[name[:-4]]()
    for k in d.files:
        assert np.array_equal(d[k], out[k], equal_nan=True), (name, k)
