"""Run the resident step on a synthetic case, for profiling captures.

    python -m vtkmakecompare_b200.profile_step --grid 128 96 128 --steps 2 [--exact]
    python -m vtkmakecompare_b200.profile_step --poisson 5
    python -m vtkmakecompare_b200.profile_step --grid 128 128 128 --adjoint 6

Builds the penalised channel-with-sphere case of bench.py at the given size
(level-set mask, initial projection), runs --warmup steps, then --steps
steps (or --poisson solves, or the discrete adjoint of --adjoint steps:
checkpoints every half, wall flux averaged over the second half) and prints
the wall time.  Kernel launches before the measured part: the level set
(2*2001+1), the projection (8) and the warm-up steps (24 each).
"""
import argparse
import math
import time

from . import solver as S
from . import workload as W


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[128, 96, 128])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--poisson", type=int, default=0)
    ap.add_argument("--exact", action="store_true")
    ap.add_argument("--adjoint", type=int, default=0)
    ap.add_argument("--flags", type=int, default=0,
                    help="extra nse_config flags (e.g. 256 = NSE_FLAG_POISSON3)")
    ap.add_argument("--shapes", type=int, nargs=2, default=[-1, -1],
                    help="right-hand-side and correction launch shapes (nse_ctx_set_shapes; "
                         "-1: autotuned), so a profiler sees no tuning launches of them")
    a = ap.parse_args()
    nx, ny, nz = a.grid
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = W.channel_state(g, seed=2024, t_bot=0.0, t_top=0.0)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    Re = 3000.0
    cfg = S.Config(nx, ny, nz, dt, Re, 0.71, 1.0e4, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0, body_force=3.0 / Re, heat_source=0.0, t_solid=1.0,
                   flags=(S.FLAG_EXACT if a.exact else 0) | a.flags)
    with S.Context(cfg) as ctx:
        for k in ("u", "v", "w", "T"):
            ctx.upload(k, f[k])
        ctx.levelset(W.sphere_phi0(g, (math.pi, 0.0, math.pi / 2), 0.25), width=1.5,
                     want_phi=False)
        ctx.set_shapes(*a.shapes)
        ctx.project()
        ctx.start()
        ctx.step(a.warmup)
        ctx.sync()
        t0 = time.perf_counter()
        if a.poisson:
            ctx.upload("phi", W.poisson_rhs(g, 7))
            for _ in range(a.poisson):
                ctx.poisson()
        elif a.adjoint:
            n = a.adjoint
            with S.Adjoint(ctx, n, checkpoint_every=max(1, n // 2), avg_from=n // 2 + 1) as adj:
                J, _ = adj.gradient()
            print(f"adjoint of {n} steps: J = {J:.12e}")
        else:
            ctx.step(a.steps)
        ctx.sync()
        el = time.perf_counter() - t0
        print(f"grid {nx}x{ny}x{nz}: {el * 1e3:.2f} ms, monitor {ctx.monitor()}")


if __name__ == "__main__":
    main()
