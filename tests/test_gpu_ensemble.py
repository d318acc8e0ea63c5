"""Ensemble of independent cases (nse_ensemble_*): heterogeneous grids, masks
and precisions stepped together on several streams, the steps after the first
replayed from a captured CUDA graph.  Every case must end bit-identical to the
same case stepped on its own (same kernels in the same order per case), for
even and odd step counts."""
import numpy as np
import pytest

from tests.test_gpu_step import make_case
from vtkmakecompare_b200 import solver as S

pytestmark = pytest.mark.gpu

SHAPES = [((64, 48, 64), S.FP64), ((96, 48, 64), S.FP64), ((128, 40, 96), S.MIXED),
          ((64, 64, 64), S.MIXED), ((40, 33, 36), S.FP64)]
KEYS = ("u", "v", "w", "p", "T", "u_ta", "u_pre", "T_pre", "divu")


def make(n, prec, seed):
    g, f, c1, par = make_case(*n, seed=seed, sphere=True)
    cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                   g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0, body_force=par["force"],
                   heat_source=par["source"], t_bot=par["tbot"], t_top=par["ttop"],
                   t_solid=par["tsolid"], precision=prec)
    c = S.Context(cfg)
    for k in ("u", "v", "w", "T"):
        c.upload(k, f[k])
    c.upload("cellvalue", c1)
    c.project()
    c.start()
    return c


def test_ensemble_matches_cases_stepped_alone():
    ens_cases = [make(n, p, 10 + i) for i, (n, p) in enumerate(SHAPES)]
    solo = [make(n, p, 10 + i) for i, (n, p) in enumerate(SHAPES)]
    try:
        with S.Ensemble(ens_cases, nstreams=3) as ens:
            for n_steps in (7, 4, 1, 5):
                ens.step(n_steps)
                ens.sync()
                for c in solo:
                    c.step(n_steps)
                    c.sync()
                for i, (a, b) in enumerate(zip(ens_cases, solo)):
                    assert a.step_index == b.step_index
                    for k in KEYS:
                        assert np.array_equal(a.download(k), b.download(k)), (i, k, n_steps)
    finally:
        for c in ens_cases + solo:
            c.close()
