"""The reference's output and restart files (OUTPUT, OUTFIELD, READFIELD of
nse_dominik.f:2606-2794) written by the library's gfortran-ABI entry points,
byte for byte against the oracle's independent restatement
(oracle/fortran_io.py), plus the READFIELD round trip.  Host code only: runs
without a GPU."""
import filecmp
import os

import numpy as np
import pytest

from oracle import fortran_io as FIO
from vtkmakecompare_b200 import NseError
from vtkmakecompare_b200 import legacy as G

N = (6, 5, 4)


def fields(seed=3):
    nx, ny, nz = N
    rng = np.random.default_rng(seed)
    pad = (nx + 2, ny + 2, nz + 2)
    f = {k: np.asfortranarray(rng.standard_normal(pad)) for k in
         ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "phi", "divu")}
    f["u"][2, 2, 2] = 1e-31   # averages below 1e-30 are written as 0
    f["u"][1, 2, 2] = -1e-31
    f["T"][nx, 3, nz // 2] = 1.0e-5    # E editing in temperature_check.dat
    f["T"][nx, 2, nz // 2] = 0.0
    f["cellvalue"] = np.asfortranarray(rng.random((nx, ny, nz, 4)))
    g = {k: np.linspace(-0.3, 1.7, n + 2) for k, n in zip("xyz", N)}
    return f, g


def run_in(path, fn):
    cwd = os.getcwd()
    os.chdir(path)
    try:
        fn()
    finally:
        os.chdir(cwd)


def test_output_matches_the_oracle_byte_for_byte(tmp_path):
    nx, ny, nz = N
    f, g = fields()
    a, b = tmp_path / "lib", tmp_path / "oracle"
    a.mkdir()
    b.mkdir()
    run_in(a, lambda: G.output(f["u"], f["v"], f["w"], f["p"], g["x"], g["y"], g["z"], nx, ny,
                               nz, f["T"], f["cellvalue"], f["u_ta"], f["v_ta"], f["w_ta"],
                               f["phi"], f["divu"]))
    FIO.output(str(b), f["u"], f["v"], f["w"], f["p"], g["x"], g["y"], g["z"], nx, ny, nz,
               f["T"], f["cellvalue"], f["u_ta"], f["v_ta"], f["w_ta"], f["phi"], f["divu"])
    names = sorted(os.listdir(b / "nseoutput2"))
    assert len(names) == 15 and sorted(os.listdir(a / "nseoutput2")) == names
    for n in names:
        assert filecmp.cmp(a / "nseoutput2" / n, b / "nseoutput2" / n, shallow=False), n
    assert (a / "temperature_check.dat").read_text() == (b / "temperature_check.dat").read_text()
    # record structure: one 24-byte record per interior cell, zero where |avg| < 1e-30
    recs = FIO.read_records(a / "nseoutput2" / "velocity.dat")
    assert len(recs) == nx * ny * nz and all(len(r) == 24 for r in recs)
    assert FIO.read_records(a / "nseoutput2" / "gridnumber.dat") == [
        np.array([nx, ny, nz], "<i4").tobytes()]


def test_outfield_and_readfield_round_trip(tmp_path):
    nx, ny, nz = N
    f, g = fields(5)
    run_in(tmp_path, lambda: G.outfield(g["x"], g["y"], g["z"], f["u"], f["v"], f["w"], f["p"],
                                        nx, ny, nz, 12.5, f["T"], f["phi"], f["u_ta"],
                                        f["v_ta"], f["w_ta"]))
    recs = FIO.read_records(tmp_path / "field.u")
    assert np.frombuffer(recs[0], "<f8")[0] == 12.5
    assert len(recs) == 1 + (nx + 2) * (ny + 2) * (nz + 2)
    FIO.grid_u(str(tmp_path / "grid_oracle.u"), g["x"], g["y"], g["z"], nx, ny, nz)
    assert filecmp.cmp(tmp_path / "nseoutput2" / "grid.u", tmp_path / "grid_oracle.u",
                       shallow=False)
    # READFIELD reads OUTPUT's field.u (no time record)
    FIO.field_u(str(tmp_path / "nseoutput2" / "field.u"), None, f["u"], f["v"], f["w"], f["p"],
                f["T"], f["phi"], f["u_ta"], f["v_ta"], f["w_ta"])
    out = {k: np.zeros_like(f[k]) for k in ("u", "v", "w", "p", "T", "phi", "u_ta", "v_ta",
                                            "w_ta")}
    run_in(tmp_path, lambda: G.readfield(out["u"], out["v"], out["w"], out["p"], nx, ny, nz,
                                         out["T"], out["phi"], out["u_ta"], out["v_ta"],
                                         out["w_ta"]))
    for k, v in out.items():
        assert np.array_equal(v, f[k]), k


def test_readfield_rejects_a_truncated_file(tmp_path):
    nx, ny, nz = N
    f, _ = fields()
    (tmp_path / "nseoutput2").mkdir()
    path = tmp_path / "nseoutput2" / "field.u"
    FIO.field_u(str(path), None, f["u"], f["v"], f["w"], f["p"], f["T"], f["phi"], f["u_ta"],
                f["v_ta"], f["w_ta"])
    data = path.read_bytes()
    path.write_bytes(data[: len(data) // 2])
    out = {k: np.zeros_like(f["u"]) for k in range(9)}
    with pytest.raises(NseError, match="record"):
        run_in(tmp_path, lambda: G.readfield(out[0], out[1], out[2], out[3], nx, ny, nz, out[4],
                                             out[5], out[6], out[7], out[8]))
