"""Parity of the resident GPU step with the CPU oracle on the benchmark
workloads themselves, from identical seeded inputs:

* the 64^3 plain channel (2pi x 2 x pi, tanh stretching 2, Re 3000, Pr 0.71,
  noise 0.05 on u, v, w, T linear from 1 to 0, no obstacle, CFL 0.5) after
  its initial projection and 10 steps;
* the seeded N(0,1) Poisson right-hand side with its dy-weighted mean
  removed, through the resident solve and through the tier-1 drop-ins
  (p2s_ -> spn_ -> sp0b_ -> s2p_ -> phibc_), against the oracle's
  P2S/SPN/SP0B/S2P/PHIBC (mkp.f:223-320, p2s_fftw2d.f);
* the ensemble grids 96x64x96 and 160x128x160 (x lines through the
  partitioned solver with 3 and 5 rows per lane) with obstacles;
* the 256x192x256 sphere workload of the benchmark for 3 steps.

Bounds (north star): state after N steps within 1e-10 relative L2,
Poisson solution within 1e-12 relative L2, post-projection divergence
at most 1e-12 (scaled by max|u|/dx, the size of one difference quotient).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import oracle_grid, rel_l2
from vtkmakecompare_b200 import legacy as G
from vtkmakecompare_b200 import solver as S
from vtkmakecompare_b200 import workload as W

pytestmark = pytest.mark.gpu

STATE = ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre", "T_pre",
         "u_ep2", "v_ep2", "w_ep2")


def channel(nx, ny, nz, seed, t_bot, t_top):
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = W.channel_state(g, seed=seed, t_bot=t_bot, t_top=t_top)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    return g, f, dt


def run_pair(g, f, dt, c1, Re, Pr, t_bot, t_top, t_solid, nsteps):
    """Both sides: upload/copy the same fields and mask, project, copy into the
    AB2 history, step nsteps times.  Returns (gpu fields, gpu monitor, oracle)."""
    kw = dict(force=3.0 / Re, source=0.0, tbot=t_bot, ttop=t_top, tsolid=t_solid)
    s = O.Solver(oracle_grid(g), dt, Re, Pr, 1.0e4, **kw)
    for k in ("u", "v", "w", "T"):
        s.f[k][...] = f[k]
    s.cellvalue[..., 0] = c1
    s.project()
    s.start()
    s.step(nsteps)
    cfg = S.Config(g["nx"], g["ny"], g["nz"], dt, Re, Pr, 1.0e4, g["xl"], g["yl"], g["zl"],
                   y0=-1.0, ystretch=2.0, body_force=3.0 / Re, heat_source=0.0, t_bot=t_bot,
                   t_top=t_top, t_solid=t_solid)
    with S.Context(cfg) as ctx:
        for k in ("u", "v", "w", "T"):
            ctx.upload(k, f[k])
        ctx.upload("cellvalue", c1)
        ctx.project()
        ctx.start()
        ctx.step(nsteps)
        got = {k: ctx.download(k) for k in STATE + ("divu",)}
        mon = ctx.monitor()
    return got, mon, s


def check_state(got, mon, s, g, bound=1e-10):
    scale = max(1.0, np.abs(s.f["u"]).max() / g["dx"][1])
    errs = {k: rel_l2(got[k], s.f[k]) for k in STATE}
    bad = {k: e for k, e in errs.items() if not e <= bound}
    assert not bad, bad
    assert mon["nonfinite"] == 0
    assert mon["max_divu"] <= 1e-12 * scale, mon
    assert np.abs(s.f["divu"]).max() <= 1e-12 * scale
    assert np.abs(got["divu"] - s.f["divu"]).max() <= 1e-12 * scale
    return errs


def test_channel64_plain_10_steps():
    """64^3 plain channel, no obstacle (mask 0), T = 1 at y = -1 and 0 at
    y = 1: projection and 10 FP64 steps against the oracle."""
    n = 64
    g, f, dt = channel(n, n, n, seed=11, t_bot=1.0, t_top=0.0)
    c1 = np.zeros((n, n, n), order="F")
    got, mon, s = run_pair(g, f, dt, c1, 3000.0, 0.71, 1.0, 0.0, 0.0, 10)
    check_state(got, mon, s, g)


def oracle_poisson(g, rhs):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    og = oracle_grid(g)
    AC, KXZ = O.mkp_coeffs(og)
    PT = O.p2s(rhs, nx, ny, nz)
    O.spn(nx, ny, nz, AC, KXZ, PT)
    O.sp0b(nx, ny, nz, AC, PT)
    phi = O.s2p(PT, nx, ny, nz)
    O.phibc(nx, ny, nz, phi)
    return phi, AC, KXZ


@pytest.mark.parametrize("n", [(64, 64, 64), (256, 192, 256)])
def test_seeded_poisson_rhs(n):
    """The seeded N(0,1) right-hand side with its dy-weighted mean removed
    (W.poisson_rhs): the resident solve and the tier-1 drop-in chain against
    the oracle's P2S -> SPN -> SP0B -> S2P -> PHIBC to 1e-12 relative L2."""
    nx, ny, nz = n
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rhs = W.poisson_rhs(g, seed=7)
    ref, AC, KXZ = oracle_poisson(g, rhs)
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0)
    with S.Context(cfg) as ctx:
        ctx.upload("phi", rhs)
        ctx.poisson()
        sol = ctx.download("phi")
    assert rel_l2(sol[I], ref[I]) < 1e-12
    if nx > 64:
        return
    # the same chain through the reference's own subroutine names
    PT = np.zeros((nx // 2 + 1, ny + 2, nz + 2), dtype=np.complex128, order="F")
    G.p2s(rhs.copy(order="F"), PT, nx, ny, nz)
    G.spn(nx, ny, nz, AC, KXZ, PT)
    G.sp0b(nx, ny, nz, AC, PT)
    phi = W.padded(g)
    G.s2p(PT, phi, nx, ny, nz)
    G.phibc(nx, ny, nz, phi)
    assert rel_l2(phi[I], ref[I]) < 1e-12


@pytest.mark.parametrize("seed", [7000, 7001, 7002, 7005])
def test_ensemble_cases_match_oracle(seed):
    """Cases of the batched-ensemble workload (grids 64^3 .. 160x128x160,
    1-3 spheres or cubes, own Re and noise, T = 1 at y = -1 and 0 at y = 1,
    obstacles at T = 1) stepped alone: projection and 4 FP64 steps against
    the oracle."""
    g, f, phi0, Re, _ = W.ensemble_case(seed)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    c1 = W.smoothed_mask(g, phi0, 1.5)
    got, mon, s = run_pair(g, f, dt, c1, Re, 0.71, 1.0, 0.0, 1.0, 4)
    check_state(got, mon, s, g)


@pytest.mark.parametrize("n", [(96, 64, 96), (160, 128, 160)])
def test_ensemble_grids_with_sphere(n):
    """The two ensemble grids whose x lines take the partitioned solver with
    3 and 5 rows per lane, with the benchmark sphere, 5 FP64 steps."""
    g, f, dt = channel(*n, seed=21, t_bot=1.0, t_top=0.0)
    c1 = W.smoothed_mask(g, W.sphere_phi0(g, (math.pi, 0.0, math.pi / 2), 0.25), 1.5)
    got, mon, s = run_pair(g, f, dt, c1, 3000.0, 0.71, 1.0, 0.0, 1.0, 5)
    check_state(got, mon, s, g)


def test_benchmark_workload_3_steps():
    """The 256x192x256 benchmark workload (sphere R = 0.25 at (pi, 0, pi/2),
    walls T = 0, sphere T = 1): projection and 3 FP64 steps against the
    oracle."""
    g, f, dt = channel(256, 192, 256, seed=2024, t_bot=0.0, t_top=0.0)
    c1 = W.smoothed_mask(g, W.sphere_phi0(g, (math.pi, 0.0, math.pi / 2), 0.25), 1.5)
    got, mon, s = run_pair(g, f, dt, c1, 3000.0, 0.71, 0.0, 0.0, 1.0, 3)
    check_state(got, mon, s, g)


@pytest.mark.parametrize("ny", [48, 192, 256])
def test_three_pass_poisson_matches_five_pass_and_oracle(ny):
    """The three-pass solve (NSE_FLAG_POISSON3: each plane's P2S and S2P + PHIBC
    in one cluster launch, partitioned SPN) against the five-pass default and
    the oracle, on the seeded right-hand side, over the whole padded array
    (ghosts included: both write exactly PHIBC's entries)."""
    nx, nz = 256, 256
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rhs = W.poisson_rhs(g, seed=ny)
    out = []
    for flags in (S.FLAG_POISSON3, 0):
        cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                       ystretch=2.0, flags=flags)
        with S.Context(cfg) as ctx:
            ctx.upload("phi", rhs)
            ctx.poisson()
            out.append(ctx.download("phi"))
    assert rel_l2(out[0], out[1]) < 1e-12
    ref, _, _ = oracle_poisson(g, rhs)
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    assert rel_l2(out[0][I], ref[I]) < 1e-12
    # the entries PHIBC and S2P never write keep the uploaded values
    assert np.array_equal(out[0][nx + 1, 0, :], rhs[nx + 1, 0, :])
    assert np.array_equal(out[0][:, ny + 1, 0], rhs[:, ny + 1, 0])


@pytest.mark.parametrize("n", [(256, 192, 256), (96, 64, 96), (160, 128, 160), (64, 48, 60)])
def test_tma_tile_spn_matches_default_and_oracle(n):
    """NSE_FLAG_SPN_TMA (SPN + SP0B through TMA tiles of 16 kx columns,
    partitioned over 16 warps) against the default two-ended solver and the
    oracle on the seeded right-hand side, and through 3 steps of the
    penalised step."""
    nx, ny, nz = n
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rhs = W.poisson_rhs(g, seed=nx + ny)
    out = []
    for flags in (S.FLAG_SPN_TMA, 0):
        cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                       ystretch=2.0, flags=flags)
        with S.Context(cfg) as ctx:
            ctx.upload("phi", rhs)
            ctx.poisson()
            ctx.sync()
            out.append(ctx.download("phi"))
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    assert rel_l2(out[0][I], out[1][I]) < 1e-12
    ref, _, _ = oracle_poisson(g, rhs)
    assert rel_l2(out[0][I], ref[I]) < 1e-12
    gg, f, dt = channel(*n, seed=5, t_bot=1.0, t_top=0.0)
    c1 = W.smoothed_mask(gg, W.sphere_phi0(gg, (math.pi, 0.0, math.pi / 2), 0.25), 1.5)
    res = []
    for flags in (S.FLAG_SPN_TMA, 0):
        cfg = S.Config(nx, ny, nz, dt, 3000.0, 0.71, 1.0e4, gg["xl"], gg["yl"], gg["zl"],
                       y0=-1.0, ystretch=2.0, body_force=1e-3, heat_source=0.0, t_bot=1.0,
                       t_solid=1.0, flags=flags)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.project()
            ctx.start()
            ctx.step(3)
            ctx.sync()
            res.append({k: ctx.download(k) for k in ("u", "v", "w", "p", "T")})
            assert ctx.monitor()["max_divu"] < 1e-10
    for k in res[0]:
        assert rel_l2(res[0][k], res[1][k]) < 1e-10, k


@pytest.mark.parametrize("n", [(256, 192, 256), (64, 48, 256)])
def test_sliced_middle_passes_are_bit_identical(n):
    """The z transforms and SPN in kx slices (NSE_FLAG_MID_SLICES: 3 slices,
    each slice's three passes back to back) give the same bits as the
    unsliced passes (NSE_FLAG_NO_AUTOTUNE), in the solve on the seeded
    right-hand side and through 2 penalised steps, FP64 and mixed; the
    autotuned default agrees too and reports a slice count."""
    nx, ny, nz = n
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rhs = W.poisson_rhs(g, seed=nx + 7)
    out = []
    for flags in (S.FLAG_NO_AUTOTUNE, S.FLAG_MID_SLICES, 0):
        cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                       ystretch=2.0, flags=flags)
        with S.Context(cfg) as ctx:
            ctx.upload("phi", rhs)
            ctx.poisson()
            ctx.sync()
            out.append(ctx.download("phi"))
            if flags == S.FLAG_MID_SLICES:
                assert ctx.line_shapes()["mid"] == 3
            if flags == 0:
                assert ctx.line_shapes()["mid"] in (1, 2, 3, 5, 9)
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[0], out[2])
    ref, _, _ = oracle_poisson(g, rhs)
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    assert rel_l2(out[1][I], ref[I]) < 1e-12
    gg, f, dt = channel(*n, seed=9, t_bot=1.0, t_top=0.0)
    c1 = W.smoothed_mask(gg, W.sphere_phi0(gg, (math.pi, 0.0, math.pi / 2), 0.25), 1.5)
    for prec in (S.FP64, S.MIXED):
        res = []
        for flags in (S.FLAG_NO_AUTOTUNE, S.FLAG_MID_SLICES | S.FLAG_NO_AUTOTUNE):
            cfg = S.Config(nx, ny, nz, dt, 3000.0, 0.71, 1.0e4, gg["xl"], gg["yl"], gg["zl"],
                           y0=-1.0, ystretch=2.0, body_force=1e-3, heat_source=0.0,
                           t_bot=1.0, t_solid=1.0, precision=prec, flags=flags)
            with S.Context(cfg) as ctx:
                for k in ("u", "v", "w", "T"):
                    ctx.upload(k, f[k])
                ctx.upload("cellvalue", c1)
                ctx.project()
                ctx.start()
                ctx.step(2)
                ctx.sync()
                res.append({k: ctx.download(k) for k in ("u", "v", "w", "p", "T")})
        for k in res[0]:
            assert np.array_equal(res[0][k], res[1][k]), (prec, k)


@pytest.mark.parametrize("n", [(256, 192, 256), (64, 48, 256), (48, 37, 40)])
def test_spn_tile_and_cpasync_forms_give_the_same_bits(n):
    """The two-ended SPN on TMA tiles of 16 kx columns (the default) and with
    per-thread cp.async staging (NSE_FLAG_SPN_CPASYNC) give the same bits in
    the solve on the seeded right-hand side, whole and in 3 kx slices (odd ny
    and a partial last column group included), and agree with the oracle."""
    nx, ny, nz = n
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rhs = W.poisson_rhs(g, seed=nx + 11)
    out = []
    for flags in (S.FLAG_NO_AUTOTUNE, S.FLAG_NO_AUTOTUNE | S.FLAG_SPN_CPASYNC,
                  S.FLAG_MID_SLICES, S.FLAG_MID_SLICES | S.FLAG_SPN_CPASYNC):
        cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                       ystretch=2.0, flags=flags)
        with S.Context(cfg) as ctx:
            ctx.upload("phi", rhs)
            ctx.poisson()
            ctx.sync()
            out.append(ctx.download("phi"))
    for o in out[1:]:
        assert np.array_equal(out[0], o)
    ref, _, _ = oracle_poisson(g, rhs)
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    assert rel_l2(out[0][I], ref[I]) < 1e-12
