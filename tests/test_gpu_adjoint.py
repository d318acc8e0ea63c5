"""The GPU discrete adjoint (nse_adjoint_*, k_adjoint.cu) and the adjoint.f
drop-ins.

* J, dJ/dc1 and the adjoint of every initial-state field equal the numpy
  adjoint of oracle/adjoint.py (which finite differences of the C oracle pin,
  tests/test_adjoint_oracle.py) to 1e-8 relative L2;
* central finite differences of the GPU's own J (step 1e-6 along seeded
  N(0,1) directions) agree with the adjoint gradient to 1e-6 relative;
* the checkpoint interval does not change the gradient (replays are
  deterministic: bit-identical);
* set_adj_convect_, set_adj_convection_for_scalar_ and set_adj_ns_scalar_
  equal the restated adjoint.f routines.
"""
import math

import numpy as np
import pytest

from oracle import adjoint as A
from tests._helpers import oracle_grid, rel_l2
from vtkmakecompare_b200 import legacy as LG
from vtkmakecompare_b200 import solver as S
from vtkmakecompare_b200 import workload as W

pytestmark = pytest.mark.gpu

PAR = dict(dt=0.01, Re=300.0, Sc=0.71, eta=1.0e3, force=0.01, source=0.0, tbot=1.0, ttop=0.0,
           tsolid=1.0)


def make_case(nx, ny, nz, seed=3, radius=0.6):
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    rng = np.random.default_rng(seed)
    y = g["y"][1:-1]
    st = {}
    st["u"] = 1.5 * (1 - y ** 2)[None, :, None] + 0.05 * rng.standard_normal((nx, ny, nz))
    st["v"] = 0.05 * rng.standard_normal((nx, ny, nz))
    st["v"][:, -1] = 0.0
    st["w"] = 0.05 * rng.standard_normal((nx, ny, nz))
    st["T"] = np.broadcast_to((1 - (y + 1) / 2)[None, :, None], (nx, ny, nz)).copy()
    st["T"] += 0.01 * rng.standard_normal((nx, ny, nz))
    for k in ("u_ta", "v_ta", "w_ta"):
        st[k] = 0.01 * rng.standard_normal((nx, ny, nz))
    st["v_ta"][:, -1] = 0.0
    for k in ("u", "v", "w", "T"):
        st[k + "_pre"] = 0.1 * rng.standard_normal((nx, ny, nz))
    phi = W.sphere_phi0(g, (math.pi, 0.0, math.pi / 2), radius)[1:-1, 1:-1, 1:-1]
    h = 1.5 * g["dx"][1]
    c1 = np.where(phi >= h, 1.0,
                  np.where(phi <= -h, 0.0, (np.sin(3.1415926535 * phi / 2 / h) + 1) / 2))
    P = A.Params(oracle_grid(g), dt=PAR["dt"], Re=PAR["Re"], Sc=PAR["Sc"], eta=PAR["eta"],
                 force=PAR["force"], source=PAR["source"], tbot=PAR["tbot"], ttop=PAR["ttop"],
                 tsolid=PAR["tsolid"])
    return g, P, st, np.asfortranarray(c1)


def make_ctx(g, flags=0):
    cfg = S.Config(g["nx"], g["ny"], g["nz"], PAR["dt"], PAR["Re"], PAR["Sc"], PAR["eta"],
                   g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0, body_force=PAR["force"],
                   heat_source=PAR["source"], t_bot=PAR["tbot"], t_top=PAR["ttop"],
                   t_solid=PAR["tsolid"], flags=flags)
    return S.Context(cfg)


def load(ctx, st, c1):
    for k, v in st.items():
        f = np.zeros(ctx.shape, order="F")
        f[1:-1, 1:-1, 1:-1] = v
        ctx.upload(k, f)
    ctx.upload("cellvalue", c1)
    ctx.step_index = 1


def padded_weights(shape, interior):
    w = np.zeros(shape, order="F")
    w[1:-1, 1:-1, 1:-1] = interior
    return w


@pytest.mark.parametrize("flags", [0, S.FLAG_EXACT])
@pytest.mark.parametrize("n", [(32, 16, 24), (64, 24, 32)])
def test_gradient_matches_numpy_adjoint(n, flags):
    g, P, st, c1 = make_case(*n)
    rng = np.random.default_rng(11)
    extra = {k: rng.standard_normal(n) for k in ("u", "v", "w", "T", "u_ta")}
    extra["v"][:, -1] = 0.0
    N, avg = 4, 2
    J_ref, g_ref, bar_ref = A.gradient(P, st, c1, N, avg, extra)
    with make_ctx(g, flags) as ctx:
        load(ctx, st, c1)
        with S.Adjoint(ctx, N, checkpoint_every=3, avg_from=avg) as adj:
            for k, v in extra.items():
                adj.set_weight(k, padded_weights(ctx.shape, v))
            J, grad = adj.gradient()
            assert abs(J - J_ref) <= 1e-11 * abs(J_ref)
            assert rel_l2(grad, g_ref) < 1e-8
            for k in A.STATE:
                got = adj.initial_adjoint(k)[1:-1, 1:-1, 1:-1]
                assert rel_l2(got, bar_ref[k]) < 1e-8, k
        assert ctx.step_index == 1 + N


def test_gradient_matches_finite_differences():
    n = (32, 16, 24)
    g, P, st, c1 = make_case(*n, seed=5)
    N, avg = 6, 3
    with make_ctx(g) as ctx:
        load(ctx, st, c1)
        with S.Adjoint(ctx, N, checkpoint_every=2, avg_from=avg) as adj:
            J, grad = adj.gradient()
            Tb = adj.initial_adjoint("T")[1:-1, 1:-1, 1:-1]
            rng = np.random.default_rng(7)
            eps = 1e-6

            def J_at(c, stx):
                load(ctx, stx, c)
                return adj.objective()

            for _ in range(3):
                d = rng.standard_normal(n)
                fd = (J_at(c1 + eps * d, st) - J_at(c1 - eps * d, st)) / (2 * eps)
                ad = float(np.sum(grad * d))
                assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
            d = rng.standard_normal(n)
            sp = {k: v.copy() for k, v in st.items()}
            sm = {k: v.copy() for k, v in st.items()}
            sp["T"] += eps * d
            sm["T"] -= eps * d
            fd = (J_at(c1, sp) - J_at(c1, sm)) / (2 * eps)
            ad = float(np.sum(Tb * d))
            assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


def test_checkpoint_interval_does_not_change_the_gradient():
    n = (32, 16, 24)
    g, P, st, c1 = make_case(*n, seed=9)
    N = 7
    grads = []
    with make_ctx(g) as ctx:
        for K in (1, 3, 7):
            load(ctx, st, c1)
            with S.Adjoint(ctx, N, checkpoint_every=K, avg_from=4) as adj:
                grads.append(adj.gradient())
    for J, gr in grads[1:]:
        assert J == grads[0][0]
        assert np.array_equal(gr, grads[0][1])


def test_adjoint_refuses_mixed_and_bad_config():
    g, P, st, c1 = make_case(32, 16, 24)
    cfg = S.Config(96, 16, 16, 0.01, 300.0, 0.71, 1e3, g["xl"], g["yl"], g["zl"], y0=-1.0,
                   ystretch=2.0, precision=S.MIXED)
    with S.Context(cfg) as ctx:
        with pytest.raises(S.NseError, match="FP64"):
            S.Adjoint(ctx, 4)
    with make_ctx(g) as ctx:
        with pytest.raises(S.NseError, match="avg_from"):
            S.Adjoint(ctx, 4, avg_from=5)


def rand_padded(rng, n, scale=1.0):
    return np.asfortranarray(scale * rng.standard_normal((n[0] + 2, n[1] + 2, n[2] + 2)))


def test_adjoint_f_dropins_match_restatement():
    n = (12, 10, 8)
    g = W.grid_arrays(*n, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    og = oracle_grid(g)
    rng = np.random.default_rng(3)
    u, v, w, uf, vf, wf, T, Tf = (rand_padded(rng, n) for _ in range(8))
    R = np.asfortranarray(1.0 + 0.1 * np.abs(rand_padded(rng, n)))
    dt = 0.013
    grid = [g[k] for k in ("dx", "dy", "dz", "dx12", "dy12", "dz12")]
    u_v, v_v, w_v = (np.zeros_like(u) for _ in range(3))
    LG.set_adj_convect(u, u_v, v, v_v, w, w_v, 300.0, dt, *n, *grid, uf, vf, wf)
    ref = A.set_adj_convect(u, v, w, uf, vf, wf, og, dt)
    for got, r in zip((u_v, v_v, w_v), ref):
        assert rel_l2(got[1:-1, 1:-1, 1:-1], r) < 1e-14
    u_vT = np.zeros_like(u)
    LG.set_adj_convection_for_scalar(u, v, w, 300.0, dt, *n, *grid, T, u_vT, R, uf, vf, wf)
    assert rel_l2(u_vT[1:-1, 1:-1, 1:-1], A.set_adj_convection_for_scalar(uf, vf, wf, T, R, og, dt)) < 1e-14
    us, vs, ws = (np.ones_like(u) for _ in range(3))
    LG.set_adj_ns_scalar(dt, *n, g["dx12"], g["dy12"], g["dz12"], T, us, vs, ws, uf, vf, wf)
    for a in (us, vs, ws):
        assert not a[1:-1, 1:-1, 1:-1].any()
    got = S.adj_ns_scalar(dt, g, T, Tf)
    for a, r in zip(got, A.set_adj_ns_scalar(T, Tf, og, dt)):
        assert rel_l2(a[1:-1, 1:-1, 1:-1], r) < 1e-14
