"""Test infrastructure (the oracle): Python restatement of the reference's
output and restart routines, OUTPUT / OUTFIELD / READFIELD of
nse_dominik.f:2606-2794, written from the Fortran source independently of the
library's C++ writer, to check it byte for byte.

gfortran sequential unformatted files: each WRITE statement is one record,
framed before and after by its length in bytes (int32, little endian).
temperature_check.dat is list-directed: each REAL(8) item is a blank followed
by G25.17E3 editing (F editing with four trailing exponent blanks when
0.1 <= |v| < 1e17 or v == 0, E editing with a three-digit exponent
otherwise) -- a restatement of gfortran's documented list-directed layout,
not checked against a gfortran run (no Fortran compiler here).
"""
import os
import struct

import numpy as np


def _rec(f, *vals, fmt="d"):
    data = struct.pack("<" + fmt * len(vals), *vals)
    f.write(struct.pack("<i", len(data)) + data + struct.pack("<i", len(data)))


def read_records(path):
    """list of raw record payloads (bytes)"""
    out = []
    with open(path, "rb") as f:
        b = f.read()
    i = 0
    while i < len(b):
        (n,) = struct.unpack_from("<i", b, i)
        out.append(b[i + 4:i + 4 + n])
        (m,) = struct.unpack_from("<i", b, i + 4 + n)
        assert m == n, "bad record marker"
        i += 8 + n
    return out


def g25_17(v):
    v = float(v)
    if v == 0.0 or 0.1 <= abs(v) < 1e17:
        if v == 0.0:
            dec = 16
        else:
            ex = int(("%.16e" % v).split("e")[1])
            dec = 17 - (ex + 1)
        if v == 0.0 or (0 <= dec and ex >= -1 and ex + 1 <= 17):
            return " " + ("%.*f" % (dec, v)).rjust(20) + "     "
    mant, ex = ("%.16E" % v).split("E")
    ex = int(ex)
    return " " + ("%sE%s%03d" % (mant, "-" if ex < 0 else "+", abs(ex))).rjust(25)


def output(root, u, v, w, p, x, y, z, nx, ny, nz, T, cellvalue, u_ta, v_ta, w_ta, phi, divu):
    """OUTPUT, nse_dominik.f:2606-2723 (arrays: padded fields, Fortran order)"""
    od = os.path.join(root, "nseoutput2")
    os.makedirs(od, exist_ok=True)
    names = ["velocity", "temperature", "pressure", "divergence", "gridx", "gridy", "gridz",
             "gridnumber", "phi", "cellvalue1", "cellvalue2", "cellvalue3", "cellvalue4"]
    fs = {n: open(os.path.join(od, n + ".dat"), "wb") for n in names}
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                ua = (u[i - 1, j, k] + u[i, j, k]) * 0.50
                va = (v[i, j - 1, k] + v[i, j, k]) * 0.50
                wa = (w[i, j, k - 1] + w[i, j, k]) * 0.50
                ua = 0.0 if abs(ua) < 1.0e-30 else ua
                va = 0.0 if abs(va) < 1.0e-30 else va
                wa = 0.0 if abs(wa) < 1.0e-30 else wa
                _rec(fs["velocity"], ua, va, wa)
                _rec(fs["pressure"], p[i, j, k])
                _rec(fs["temperature"], T[i, j, k])
                _rec(fs["divergence"], divu[i, j, k])
                _rec(fs["phi"], phi[i, j, k])
                for q in range(4):
                    _rec(fs["cellvalue%d" % (q + 1)], cellvalue[i - 1, j - 1, k - 1, q])
    with open(os.path.join(root, "temperature_check.dat"), "w") as tc:
        for j in range(0, ny + 2):
            tc.write(g25_17(y[j]) + g25_17(T[nx, j, nz // 2]) + "\n")
    for i in range(1, nx + 1):
        _rec(fs["gridx"], x[i])
    for j in range(1, ny + 1):
        _rec(fs["gridy"], y[j])
    for k in range(1, nz + 1):
        _rec(fs["gridz"], z[k])
    _rec(fs["gridnumber"], nx, ny, nz, fmt="i")
    for f in fs.values():
        f.close()
    field_u(os.path.join(od, "field.u"), None, u, v, w, p, T, phi, u_ta, v_ta, w_ta)
    grid_u(os.path.join(od, "grid.u"), x, y, z, nx, ny, nz)


def field_u(path, tid, u, v, w, p, T, phi, u_ta, v_ta, w_ta):
    with open(path, "wb") as f:
        if tid is not None:
            _rec(f, tid)
        nx2, ny2, nz2 = u.shape
        for k in range(nz2):
            for j in range(ny2):
                for i in range(nx2):
                    _rec(f, u[i, j, k], v[i, j, k], w[i, j, k], p[i, j, k], T[i, j, k],
                         phi[i, j, k], u_ta[i, j, k], v_ta[i, j, k], w_ta[i, j, k])


def grid_u(path, x, y, z, nx, ny, nz):
    with open(path, "wb") as f:
        for i in range(1, nx + 1):
            _rec(f, x[i])
        for j in range(1, ny + 1):
            _rec(f, y[j])
        for k in range(1, nz + 1):
            _rec(f, z[k])


def read_field(path, nx, ny, nz):
    """READFIELD: dict of the nine padded fields"""
    recs = read_records(path)
    assert len(recs) == (nx + 2) * (ny + 2) * (nz + 2)
    a = np.array([struct.unpack("<9d", r) for r in recs])
    names = ("u", "v", "w", "p", "T", "phi", "u_ta", "v_ta", "w_ta")
    return {n: np.asfortranarray(a[:, q].reshape((nx + 2, ny + 2, nz + 2), order="F"))
            for q, n in enumerate(names)}
