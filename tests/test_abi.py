"""The C-ABI library (no GPU needed): it loads, exports every symbol that
include/nsegpu.h declares, the Python mirror's argument tables agree with the
prototypes, the host-side grid routines agree with the oracle, and compute
entry points fail loudly (NseError) when no GPU is usable."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from vtkmakecompare_b200 import NseError, legacy, lib
from vtkmakecompare_b200 import workload as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nsegpu.h")


def prototypes():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{()]*)\)\s*;", text):
        name, args = m.group(1), m.group(2)
        if name in ("if", "while", "sizeof"):
            continue
        out[name] = [a.strip() for a in args.split(",") if a.strip() and a.strip() != "void"]
    return out


def test_library_exports_every_declared_symbol():
    L = lib()
    protos = prototypes()
    assert len(protos) >= 45
    missing = [n for n in protos if not hasattr(L, n)]
    assert not missing, missing


def test_config_flags_match_header():
    """Every NSE_FLAG_* of include/nsegpu.h has the same value as the Python
    mirror's FLAG_* constant, and the flags are distinct bits."""
    from vtkmakecompare_b200 import solver as S
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    flags = {m.group(1): int(m.group(2))
             for m in re.finditer(r"\bNSE_FLAG_([A-Z0-9_]+)\s*=\s*(\d+)", text)}
    assert len(flags) >= 14
    for name, v in flags.items():
        assert getattr(S, "FLAG_" + name) == v, name
        assert v & (v - 1) == 0, name
    assert len(set(flags.values())) == len(flags)
    mirror = {n[5:] for n in dir(S) if n.startswith("FLAG_")}
    assert mirror == set(flags), mirror ^ set(flags)


def test_legacy_signature_tables_match_header():
    protos = prototypes()
    for name, sig in legacy._SIG.items():
        args = protos[name + "_"]
        assert len(args) == len(sig), name
        for kind, a in zip(sig, args):
            if kind == "i":
                assert "int*" in a.replace(" ", "") or "void*" in a.replace(" ", ""), (name, a)
            elif kind in "do":
                assert "double*" in a.replace(" ", ""), (name, a)


def test_set_c_matches_oracle():
    nx, ny, nz = 12, 10, 8
    for (y0, gam) in ((0.0, 0.0), (-1.0, 2.0), (-1.0, 0.0)):
        g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=y0, gamma=gam)
        og = O.Grid(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=y0, gamma=gam)
        for k in ("x", "x12", "y", "y12", "z", "z12", "dx", "dx12", "dy", "dy12", "dz", "dz12"):
            assert np.array_equal(g[k], getattr(og, k)), (y0, gam, k)
    arr = {k: np.zeros(n + 2) for k, n in (("x", nx), ("x12", nx), ("y", ny), ("y12", ny),
                                          ("z", nz), ("z12", nz), ("dx", nx), ("dx12", nx),
                                          ("dy", ny), ("dy12", ny), ("dz", nz), ("dz12", nz))}
    legacy.set_c(nx, ny, nz, *[arr[k] for k in ("x", "x12", "y", "y12", "z", "z12", "dx",
                                                "dx12", "dy", "dy12", "dz", "dz12")],
                 0.25, 4.0, 4.0)
    og = O.Grid(nx, ny, nz, 0.25, 4.0, 4.0)
    for k, v in arr.items():
        assert np.array_equal(v, getattr(og, k)), k


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_compute_without_gpu_fails_loudly():
    n = 8
    A = np.asfortranarray(np.ones((n, 3)))
    B = np.ones(n)
    with pytest.raises(NseError):
        legacy.tridiag(A, B, n)
    from vtkmakecompare_b200 import solver as S
    with pytest.raises(NseError):
        S.Context(S.Config(8, 8, 8, 0.01, 100.0, 1.0, 0.0, 1.0, 1.0, 1.0))


def test_bad_arguments_are_rejected_by_the_mirror():
    with pytest.raises(TypeError):
        legacy.tridiag(np.ones((3, 3), dtype=np.float32), np.ones(3), 3)
    with pytest.raises(TypeError):
        legacy.p2s(np.ones(3))
