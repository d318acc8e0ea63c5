"""Resident time step (nse_ctx_*) against the CPU oracle's restatement of the
reference time loop, plus the known-answer and size-independent checks.

Tolerance: velocity, pressure and temperature after N steps within 1e-10
relative L2 of the oracle (the stencils and line solves round identically;
the FFT transform differs at the 1e-15 level).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import oracle_grid, rel_l2
from vtkmakecompare_b200 import solver as S
from vtkmakecompare_b200 import workload as W

pytestmark = pytest.mark.gpu

STATE = ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre", "T_pre",
         "divu", "u_ep2", "v_ep2", "w_ep2")


def smooth_mask(g, center, radius, width):
    """Smoothed-Heaviside mask of set_levelset.f:157-170 applied to the exact
    signed distance (no reinitialisation)."""
    phi = W.sphere_phi0(g, center, radius)[1:-1, 1:-1, 1:-1]
    h = width * g["dx"][1:-1, None, None]
    c = (np.sin(3.1415926535 * phi / 2.0 / h) + 1.0) / 2.0
    c = np.where(phi >= h, 1.0, np.where(phi <= -h, 0.0, c))
    return np.asfortranarray(c)


def make_case(nx, ny, nz, seed=3, sphere=True, Re=3000.0, Pr=0.71, eta=1.0e4):
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = W.channel_state(g, seed)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    c1 = smooth_mask(g, (math.pi, 0.0, math.pi / 2), 0.6, 1.5) if sphere else np.zeros(
        (nx, ny, nz), order="F")
    par = dict(dt=dt, Re=Re, Sc=Pr, eta=eta, force=3.0 / Re, source=0.0, tbot=1.0, ttop=0.0,
               tsolid=1.0 if sphere else 0.0)
    return g, f, c1, par


def run_oracle(g, f, c1, par, nsteps):
    s = O.Solver(oracle_grid(g), par["dt"], par["Re"], par["Sc"], par["eta"],
                 force=par["force"], source=par["source"], tbot=par["tbot"], ttop=par["ttop"],
                 tsolid=par["tsolid"])
    for k in ("u", "v", "w", "T"):
        s.f[k][...] = f[k]
    s.cellvalue[..., 0] = c1
    s.start()
    s.step(nsteps)
    return s


def make_ctx(g, f, c1, par, exact=False):
    cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                   g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0, body_force=par["force"],
                   heat_source=par["source"], t_bot=par["tbot"], t_top=par["ttop"],
                   t_solid=par["tsolid"], flags=S.FLAG_EXACT if exact else 0)
    ctx = S.Context(cfg)
    for k in ("u", "v", "w", "T"):
        ctx.upload(k, f[k])
    ctx.upload("cellvalue", c1)
    ctx.start()
    return ctx


def test_context_grid_matches_oracle_grid():
    g = W.grid_arrays(24, 16, 12, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    og = O.Grid(24, 16, 12, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    for k in ("dx", "dy", "dz", "dx12", "dy12", "dz12", "y", "y12"):
        assert np.array_equal(g[k], getattr(og, k)), k


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("n,sphere,steps", [((16, 12, 8), True, 3), ((32, 24, 16), True, 10),
                                            ((24, 16, 20), False, 10), ((40, 33, 36), True, 4),
                                            # shapes the partitioned line solver takes
                                            ((96, 48, 64), True, 4), ((128, 40, 96), True, 3),
                                            ((64, 48, 64), True, 4),  # half-warp x lines
                                            ((256, 20, 24), False, 2),
                                            # fused z transforms + SPN (clusters)
                                            ((256, 32, 256), True, 2)])
def test_steps_match_oracle(n, sphere, steps, exact):
    g, f, c1, par = make_case(*n, sphere=sphere)
    ref = run_oracle(g, f, c1, par, steps)
    with make_ctx(g, f, c1, par, exact) as ctx:
        ctx.step(steps)
        assert ctx.step_index == steps + 1
        scale = max(1.0, np.abs(ref.f["u"]).max() / g["dx"][1])
        for k in STATE:
            got = ctx.download(k)
            if k == "divu":  # both are round-off (~1e-13): compare absolutely
                assert np.abs(got - ref.f[k]).max() < 1e-11 * scale
                continue
            err = rel_l2(got, ref.f[k])
            assert err < 1e-10, (k, err)
        mon = ctx.monitor()
        assert mon["nonfinite"] == 0
        assert mon["max_divu"] < 1e-12 * max(1.0, np.abs(ref.f["u"]).max() / g["dx"][1])


def test_step_bitexact_without_projection_effects():
    """With a zero velocity field and no body force the projection sees a zero
    right-hand side; the temperature then evolves through stencils and line
    solves only, which round identically to the oracle."""
    nx, ny, nz = 16, 12, 10
    g, f, c1, par = make_case(nx, ny, nz, sphere=True)
    par["force"] = 0.0
    for k in ("u", "v", "w"):
        f[k][...] = 0.0
    ref = run_oracle(g, f, c1, par, 2)
    with make_ctx(g, f, c1, par, exact=True) as ctx:
        ctx.step(2)
        T = ctx.download("T")
        assert np.array_equal(T, ref.f["T"])


def test_poiseuille_known_answer():
    """check_convergence (nse_dominik.f:2875-2891): with body force 1 and the
    reference's uniform grid the laminar profile -Re/2 y(y-yl) is steady.  The
    discrete steady state (ghost u0 = -u1) is reproduced to round-off and is
    within O(dy^2) of the analytic profile."""
    nx, ny, nz, Re, yl, dt = 4, 64, 8, 20.0, 4.0, 1.0e-3
    g = W.grid_arrays(nx, ny, nz, 0.25, yl, 4.0)
    y = g["y"][1:-1]
    dy = yl / ny
    # discrete steady state of D2 u = -Re (force 1) with u0 = -u1, u(ny+1) = -u(ny)
    A = np.zeros((ny, ny))
    for j in range(ny):
        A[j, j] = -2.0
        if j > 0:
            A[j, j - 1] = 1.0
        if j < ny - 1:
            A[j, j + 1] = 1.0
    A[0, 0] -= 1.0
    A[-1, -1] -= 1.0
    us = np.linalg.solve(A / dy ** 2, -Re * np.ones(ny))
    u = W.padded(g)
    u[1:-1, 1:-1, 1:-1] = us[None, :, None]
    cfg = S.Config(nx, ny, nz, dt, Re, 1.0, 0.0, 0.25, yl, 4.0)
    with S.Context(cfg) as ctx:
        ctx.upload("u", u)
        ctx.start()
        ctx.step(20)
        got = ctx.download("u")[1:-1, 1:-1, 1:-1]
        v = ctx.download("v")[1:-1, 1:-1, 1:-1]
    assert np.abs(got - us[None, :, None]).max() < 1e-9 * us.max()
    assert np.abs(v).max() < 1e-10
    analytic = -Re / 2 * y * (y - yl)
    assert np.abs(us - analytic).max() < Re * dy ** 2


def laplacian(g, P):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    i, j, k = slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1)
    dx, dy, dz = g["dx"], g["dy"], g["dz"]
    dx12, dy12, dz12 = g["dx12"], g["dy12"], g["dz12"]
    X = ((P[2:nx + 2, j, k] - P[i, j, k]) / dx12[1:nx + 1, None, None] -
         (P[i, j, k] - P[0:nx, j, k]) / dx12[0:nx, None, None]) / dx[1:nx + 1, None, None]
    Y = ((P[i, 2:ny + 2, k] - P[i, j, k]) / dy12[None, 1:ny + 1, None] -
         (P[i, j, k] - P[i, 0:ny, k]) / dy12[None, 0:ny, None]) / dy[None, 1:ny + 1, None]
    Z = ((P[i, j, 2:nz + 2] - P[i, j, k]) / dz12[None, None, 1:nz + 1] -
         (P[i, j, k] - P[i, j, 0:nz]) / dz12[None, None, 0:nz]) / dz[None, None, 1:nz + 1]
    return X + Y + Z


@pytest.mark.parametrize("n", [(64, 64, 64), (256, 192, 256), (256, 24, 256), (256, 48, 256)])
def test_poisson_manufactured(n):
    """P2S -> SPN -> SP0B -> S2P inverts the reference's 7-point operator
    (solve_p stencil nse_dominik.f:1988-1993 with PHIBC ghosts): a random phi
    with the SP0B gauge (plane mean at j=1 is zero) is recovered to 1e-12."""
    nx, ny, nz = n
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rng = np.random.default_rng(5)
    phi = W.padded(g)
    phi[1:-1, 1:-1, 1:-1] = rng.standard_normal((nx, ny, nz))
    phi[1:-1, 1:-1, 1:-1] -= phi[1:-1, 1, 1:-1].mean()
    O.phibc(nx, ny, nz, phi)
    rhs = W.padded(g)
    rhs[1:-1, 1:-1, 1:-1] = laplacian(g, phi)
    rhs[1:nx + 1, 1:ny + 1, 0] = rhs[1:nx + 1, 1:ny + 1, nz]
    rhs[0, 1:ny + 1, 1:nz + 1] = rhs[nx, 1:ny + 1, 1:nz + 1]
    rhs[0, 1:ny + 1, 0] = rhs[nx, 1:ny + 1, nz]
    cfg = S.Config(nx, ny, nz, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0)
    with S.Context(cfg) as ctx:
        ctx.upload("phi", rhs)
        ctx.poisson()
        sol = ctx.download("phi")
    I = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
    assert rel_l2(sol[I], phi[I]) < 1e-12


def test_full_size_step_properties():
    """The benchmark workload at 256x192x256 (sphere, heat): one step keeps
    every field finite and the projected velocity divergence-free."""
    nx, ny, nz = 256, 192, 256
    g, f, c1, par = make_case(nx, ny, nz, sphere=True)
    with make_ctx(g, f, c1, par) as ctx:
        ctx.step(2)
        mon = ctx.monitor()
    assert mon["nonfinite"] == 0
    assert mon["max_divu"] < 1e-10


def test_projection_is_divergence_free():
    """nse_project on a noisy field (noise also on the wall values of v): the
    boundary conditions are applied before MKP, so the projected field is
    divergence-free everywhere, including the last plane, where the mean mode's
    compatibility would otherwise fail (SP0B never enforces row NY)."""
    g, f, c1, par = make_case(96, 48, 64, sphere=True)
    for prec in (S.FP64, S.MIXED):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], precision=prec,
                       flags=0)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.project()
            mon = ctx.monitor()
            assert mon["max_divu"] < 1e-10, (prec, mon)



@pytest.mark.parametrize("prec,base", [(S.FP64, 0), (S.MIXED, 0), (S.MIXED, S.FLAG_POISSON32)])
@pytest.mark.parametrize("n", [(96, 48, 64), (128, 40, 96)])
def test_concurrent_line_chains_equal_serial(n, prec, base):
    """The fast and mixed forms run the four components' line chains on
    concurrent streams; every field after 4 steps is bit-identical to the
    order on one stream (NSE_FLAG_ONE_STREAM)."""
    g, f, c1, par = make_case(*n)
    out = []
    for flags in (base, base | S.FLAG_ONE_STREAM):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"], precision=prec, flags=flags)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.start()
            ctx.step(4)
            out.append({k: ctx.download(k) for k in STATE})
    for k in STATE:
        assert np.array_equal(out[0][k], out[1][k]), k



@pytest.mark.parametrize("n", [(96, 48, 64), (128, 40, 96), (256, 64, 256), (160, 128, 160)])
def test_line_launch_shapes_give_the_same_fields(n):
    """The line passes' launch shapes give the same bits after 4 steps of a
    penalised case (same arithmetic, same tables): the fixed shapes
    (NSE_FLAG_NO_AUTOTUNE), the TMA tiles for every FP64 y/z pass
    (NSE_FLAG_LINES_TMA) and the autotuner's choice (the default)."""
    g, f, c1, par = make_case(*n)
    out = []
    shapes = None
    for flags in (S.FLAG_NO_AUTOTUNE, S.FLAG_LINES_TMA, 0):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"], flags=flags)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.start()
            ctx.step(4)
            ctx.sync()
            out.append({k: ctx.download(k) for k in STATE})
            if flags == 0:
                shapes = ctx.line_shapes()
    for k in STATE:
        assert np.array_equal(out[1][k], out[0][k]), k
        assert np.array_equal(out[2][k], out[0][k]), k
    assert all(v in (0, 1, 2, 3) for v in shapes["y"] + shapes["z"]), shapes
    assert all(v in (1, 2, 3, 4) for v in shapes["x"]), shapes
    assert shapes["rhs"] in range(7), shapes
    assert shapes["correct"] in range(16), shapes


@pytest.mark.parametrize("n,prec,flags", [((96, 64, 96), S.FP64, 0), ((80, 40, 48), S.FP64, 0),
                                          ((96, 64, 96), S.MIXED, 0),
                                          ((80, 40, 48), S.MIXED, 32)])
def test_rhs_and_correction_shapes_give_the_same_bits(n, prec, flags):
    """Every launch shape of the right-hand side and of the pipelined
    correction, the cp.async rings (0-3) and the TMA rings (4-6; FP32
    storage: FP64 halo planes by TMA, history tiles by cp.async), gives the
    same bits after 3 penalised steps (partial x and y tiles in the 80x40x48
    case; FP64, mixed, and mixed with FP64 stencil arithmetic), with no ring
    wait reported by nse_sync."""
    g, f, c1, par = make_case(*n)
    out = []
    for rhs, corr in ((0, 0), (1, 2), (2, 1), (3, 3), (4, 4), (5, 5), (6, 6), (4, 7), (5, 8),
                      (4, 9), (5, 10), (4, 11), (5, 12), (4, 13), (5, 14), (4, 15)):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"], precision=prec, flags=flags)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.set_shapes(rhs, corr)
            ctx.project()
            ctx.start()
            ctx.step(3)
            ctx.sync()
            sh = ctx.line_shapes()
            assert (sh["rhs"], sh["correct"]) == (rhs, corr)
            out.append({k: ctx.download(k) for k in STATE})
    for o in out[1:]:
        for k in STATE:
            assert np.array_equal(o[k], out[0][k]), k


def test_set_shapes_rejects_bad_codes():
    g, f, c1, par = make_case(64, 48, 64)
    cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                   g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0)
    with S.Context(cfg) as ctx:
        with pytest.raises(Exception):
            ctx.set_shapes(7, 0)
        with pytest.raises(Exception):
            ctx.set_shapes(0, 16)
        with pytest.raises(Exception):
            ctx.set_shapes(0, -2)
        with pytest.raises(Exception):
            ctx.set_line_shapes(4, 2)
        with pytest.raises(Exception):
            ctx.set_line_shapes(0, 5)


@pytest.mark.parametrize("prec,flags", [(S.FP64, 0), (S.MIXED, 64)])
def test_autotuning_context_matches_fixed_shapes(prec, flags):
    """The first context of a grid runs every autotuner inside its first
    step (right-hand side, lines, correction); its fields after 4 penalised
    steps agree with a context that keeps the fixed shapes.  A grid no other
    test uses, so the tuning is not skipped by the per-process table."""
    g, f, c1, par = make_case(80, 48, 120, seed=11)
    out = []
    for fl in (flags, flags | S.FLAG_NO_AUTOTUNE):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"], precision=prec, flags=fl)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.project()
            ctx.start()
            ctx.step(4)
            ctx.sync()
            out.append({k: ctx.download(k) for k in ("u", "v", "w", "p", "T")})
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("prec", [S.FP64, S.MIXED])
def test_graph_replayed_steps_match_eager_steps(prec):
    """From the third step on, nse_step replays a captured one-step CUDA graph
    (one per temperature buffer a step starts from).  Ten steps with a mask
    change and a launch-shape change in between (each drops the graphs)
    give the same bits as the same steps run eagerly (profiled steps never
    replay).  The library counts a replayed step's kernels like a captured
    one's: four steps after the shape change (two captures, two replays)
    count the same launches each (the profiled steps run the passes in order
    on one stream, where set_bc is one launch instead of two)."""
    g, f, c1, par = make_case(64, 48, 64, seed=13)
    out, nk = [], []
    for eager in (False, True):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"], precision=prec)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.project()
            ctx.start()
            if eager:
                ctx.profile(20)
            ctx.step(5)
            ctx.upload("cellvalue", np.asfortranarray(0.5 * c1))
            ctx.step(2)
            ctx.set_shapes(2, 2)
            per = []
            for _ in range(4):
                n0 = S.launch_count()
                ctx.step(1)
                per.append(S.launch_count() - n0)
            ctx.sync()
            nk.append(per)
            out.append({k: ctx.download(k) for k in STATE})
    for k in STATE:
        assert np.array_equal(out[0][k], out[1][k]), k
    for per in nk:
        assert len(set(per)) == 1 and per[0] > 0, per


def test_levelset_leaves_the_poisson_work_field_clean():
    """A context whose mask comes from nse_levelset steps exactly like one
    given the same mask by upload: the level set does not stay behind in the
    Poisson work field, whose never-written ghost entries the correction's
    face pass reads (zero, as in the oracle)."""
    g, f, c1, par = make_case(96, 48, 64, seed=5)
    phi0 = W.sphere_phi0(g, (math.pi, 0.0, math.pi / 2), 0.4)
    out = []
    mask = None
    for use_levelset in (True, False):
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"])
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            if use_levelset:
                ctx.levelset(phi0, nnn=50, width=1.5, want_phi=False)
                mask = ctx.download("cellvalue")
            else:
                ctx.upload("cellvalue", mask)
            ctx.project()
            ctx.start()
            ctx.step(5)
            ctx.sync()
            out.append({k: ctx.download(k) for k in STATE})
    for k in STATE:
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("n,prec,flags", [((256, 48, 64), S.FP64, 0), ((128, 40, 96), S.FP64, 0),
                                          ((192, 48, 64), S.MIXED, 0),
                                          ((256, 48, 64), S.MIXED, 64)])
def test_every_line_shape_gives_the_same_bits(n, prec, flags):
    """Every fixed line launch shape (nse_ctx_set_line_shapes: y/z 16, 8, 32
    lines per CTA or the FP64 TMA tiles; x one or two lines per warp
    iteration, direct or through shared memory) gives the same bits after 3
    penalised steps, in FP64, mixed, and mixed with FP64 line arithmetic
    (nx = 256, 128, 192: 8, 4 and 6 rows per lane in x)."""
    g, f, c1, par = make_case(*n)
    out = []
    combos = [(0, 2), (1, 1), (3, 3), (0, 4)] + ([(2, 2)] if prec == S.FP64 else [])
    for yz, xl in combos:
        cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                       g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0,
                       body_force=par["force"], heat_source=par["source"], t_bot=par["tbot"],
                       t_top=par["ttop"], t_solid=par["tsolid"], precision=prec, flags=flags)
        with S.Context(cfg) as ctx:
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.set_line_shapes(yz, xl)
            ctx.project()
            ctx.start()
            ctx.step(3)
            ctx.sync()
            sh = ctx.line_shapes()
            assert sh["x"] == [xl] * 4 and sh["y"] == [yz] * 4 and sh["z"] == [yz] * 4
            out.append({k: ctx.download(k) for k in STATE})
    for o in out[1:]:
        for k in STATE:
            assert np.array_equal(o[k], out[0][k]), k
