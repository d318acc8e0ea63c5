"""Resident output and restart files: nse_ctx_write_output writes the same
bytes as the reference's OUTPUT (the library's gfortran-ABI output_) given
the downloaded fields; the level set is the one of the last nse_levelset and
cellvalue 2..4 the face masks of SET_IMMERSED_BOUNDARY (nse_dominik.f:
1037-1080); READFIELD's file restores the state of a fresh context."""
import filecmp
import math
import os

import numpy as np
import pytest

from oracle import fortran_io as FIO
from tests.test_gpu_step import make_case
from vtkmakecompare_b200 import legacy as G
from vtkmakecompare_b200 import solver as S
from vtkmakecompare_b200 import workload as W

pytestmark = pytest.mark.gpu


def face_masks(c1):
    nx, ny, nz = c1.shape
    cv = np.zeros((nx, ny, nz, 4), order="F")
    cv[..., 0] = c1
    cv[:-1, :, :, 1] = (c1[:-1] + c1[1:]) * 0.50
    cv[-1, :, :, 1] = c1[-1]
    cv[:, :-1, :, 2] = (c1[:, :-1] + c1[:, 1:]) * 0.50
    cv[:, -1, :, 2] = c1[:, -1]
    cv[:, :, :-1, 3] = (c1[:, :, :-1] + c1[:, :, 1:]) * 0.50
    cv[:, :, -1, 3] = c1[:, :, -1]
    return cv


@pytest.mark.parametrize("precision", [S.FP64, S.MIXED])
def test_write_output_matches_output_on_downloaded_fields(tmp_path, precision):
    g, f, c1, par = make_case(96, 48, 64, sphere=False)
    cfg = S.Config(g["nx"], g["ny"], g["nz"], par["dt"], par["Re"], par["Sc"], par["eta"],
                   g["xl"], g["yl"], g["zl"], y0=-1.0, ystretch=2.0, body_force=par["force"],
                   heat_source=par["source"], precision=precision)
    with S.Context(cfg) as ctx:
        for k in ("u", "v", "w", "T"):
            ctx.upload(k, f[k])
        phi = ctx.levelset(W.sphere_phi0(g, (math.pi, 0.0, math.pi / 2), 0.5), nnn=20,
                           width=1.5)
        ctx.project()
        ctx.start()
        ctx.step(3)
        a = tmp_path / "resident"
        a.mkdir()
        ctx.write_output(a)
        d = {k: ctx.download(k) for k in ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta",
                                         "divu")}
        cv = face_masks(ctx.download("cellvalue"))
        b = tmp_path / "legacy"
        b.mkdir()
        cwd = os.getcwd()
        os.chdir(b)
        try:
            G.output(d["u"], d["v"], d["w"], d["p"], g["x"], g["y"], g["z"], g["nx"], g["ny"],
                     g["nz"], d["T"], cv, d["u_ta"], d["v_ta"], d["w_ta"], phi, d["divu"])
        finally:
            os.chdir(cwd)
        for n in sorted(os.listdir(b / "nseoutput2")):
            assert filecmp.cmp(a / "nseoutput2" / n, b / "nseoutput2" / n, shallow=False), n
        assert (a / "temperature_check.dat").read_text() == \
            (b / "temperature_check.dat").read_text()
        # OUTFIELD with the time record
        ctx.write_field(tmp_path / "field.u", 0.75, tmp_path / "grid.u")
        recs = FIO.read_records(tmp_path / "field.u")
        assert np.frombuffer(recs[0], "<f8")[0] == 0.75
        # READFIELD into a fresh context restores the state
        with S.Context(cfg) as c2:
            c2.read_field(a / "nseoutput2" / "field.u")
            for k in ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta"):
                assert np.array_equal(c2.download(k), d[k]), k
            c2.write_field(tmp_path / "field2.u", 0.75)
            assert filecmp.cmp(tmp_path / "field.u", tmp_path / "field2.u", shallow=False)
