"""The reference's Fortran subroutines, one for one, on the GPU.

Each function has the name, argument order and in-place semantics of the
reference subroutine it replaces (file:line in the signature table) and calls
the gfortran-mangled entry point of libnsegpu.so.  Arrays are numpy arrays in
the reference layout:

* padded field: float64, Fortran order, shape (nx+2, ny+2, nz+2)
* cellvalue: float64, Fortran order, shape (nx, ny, nz, 4)
* spectrum PHIT/FPT: complex128, Fortran order, shape (nx/2+1, ny+2, nz+2)
* 1-D grid arrays: float64 (n+2)

Output arrays are modified in place, exactly the entries the reference
routine writes.  Integer arguments are INTEGER*4, the others REAL*8.
"""
import ctypes as C

import numpy as np

from . import check_legacy, lib

_D = C.POINTER(C.c_double)

# argument kinds: 'a' array (in/out), 'i' INTEGER, 'd' REAL*8, 'o' REAL*8 out
_SIG = {
    "p2s": "aaiii",                        # p2s_fftw2d.f:5
    "s2p": "aaiii",                        # p2s_fftw2d.f:116
    "tridiag": "aai",                      # tridiag.f:5
    "trid2": "aaii",                       # tridiag.f:21
    "ctridiag": "aai",                     # tridiag.f:43
    "implicit_solver": "aiaaddddda",       # periodic_implicit.f:1
    "tdma": "aaaaai",                      # periodic_implicit.f:47
    "cyclic": "aaaddaai",                  # periodic_implicit.f:67
    "mkp": "aaaadaaaaaadiiiiaaaaaaaaaadd",   # mkp.f:9 (ompnthreads ignored)
    "spn": "iiiaaa",                       # mkp.f:223
    "sp0b": "iiiaa",                       # mkp.f:263
    "phibc": "iiia",                       # mkp.f:293
    "set_levelset": "iiiaaaaaaaaaa",       # set_levelset.f:1
    "readgrid3d": "iiia",                  # set_levelset.f:202
    "set_c": "iiiaaaaaaaaaaaaddd",         # nse_dominik.f:553
    "set_bc": "aaaaiiia",                  # nse_dominik.f:611
    "set_convect": "aaaaaadiiiaaaaaa",     # nse_dominik.f:757
    "set_convection_for_scalar": "aaadiiiaaaaaaaaa",  # nse_dominik.f:834
    "set_conduction": "aaaaaaddiiiaaaaaa",  # nse_dominik.f:888
    "set_diffusion_for_scalar": "ddiiiaaaaaaaadaa",   # nse_dominik.f:950
    "set_immersed_boundary": "diiidaaaaaaaaaaaio",    # nse_dominik.f:1011
    "set_explicit": "aaaaaaaaaaaaaaaiiii",  # nse_dominik.f:1132
    "set_explicit_for_tempreture": "aaaaaiiii",        # nse_dominik.f:1291
    "solve_u_temp": "aaaiiiaaaaaadddaaaa",  # nse_dominik.f:1344
    "solve_t": "aiiiaaaaaadddaaad",        # nse_dominik.f:1465
    "implicit_uy": "aiaaddddda",           # nse_dominik.f:1505
    "implicit_vy": "aiaaddddda",           # nse_dominik.f:1583
    "implicit_tx": "aiaadddaaddda",        # nse_dominik.f:1725
    "implicit_ty": "aiaadddaaddad",        # nse_dominik.f:1784
    "parallel_uy": "iiaaiiiaadddi",        # nse_dominik.f:2893
    "parallel_z": "iiaaiiiaadddi",         # nse_dominik.f:2912
    "parallel_x": "iiaaiiiaadddi",         # nse_dominik.f:2931
    "parallel_vy": "iiaaiiiaadddi",        # nse_dominik.f:2950
    "parallel_tx": "iiiiiaaaaaadddd",      # nse_dominik.f:2969
    "parallel_ty": "iiiiiaaaaaadddd",      # nse_dominik.f:2995
    "parallel_tz": "iiiiiaaaaaadddd",      # nse_dominik.f:3021
    "output": "aaaaaaaiiiaaaaaaa",         # nse_dominik.f:2606 (files under ./)
    "outfield": "aaaaaaaiiidaaaaa",        # nse_dominik.f:2726
    "readfield": "aaaaiiiaaaaa",           # nse_dominik.f:2769
    "set_adj_convect": "aaaaaaddiiiaaaaaaaaa",                  # adjoint.f:1
    "set_adj_convection_for_scalar": "aaaddiiiaaaaaaaaaaaa",    # adjoint.f:128
    "set_adj_ns_scalar": "diiiaaaaaaaaaa",                      # adjoint.f:185
}


def _ptr(a, name, k):
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{name}: argument {k} must be a numpy array")
    if a.dtype not in (np.float64, np.complex128):
        raise TypeError(f"{name}: argument {k} must be float64 or complex128, not {a.dtype}")
    if not (a.flags.f_contiguous or a.ndim == 1 and a.flags.c_contiguous):
        raise ValueError(f"{name}: argument {k} must be Fortran-contiguous")
    return a.ctypes.data_as(_D)


def _call(name, args):
    sig = _SIG[name]
    if len(args) != len(sig):
        raise TypeError(f"{name} takes {len(sig)} arguments ({len(args)} given)")
    cargs, keep, outs = [], [], []
    for k, (kind, a) in enumerate(zip(sig, args)):
        if kind == "a":
            cargs.append(_ptr(a, name, k))
        elif kind == "i":
            v = C.c_int(int(a))
            keep.append(v)
            cargs.append(C.byref(v))
        elif kind == "d":
            v = C.c_double(float(a))
            keep.append(v)
            cargs.append(C.byref(v))
        else:  # scalar output: a 1-element float64 array or None
            v = C.c_double(0.0 if a is None else float(np.asarray(a).ravel()[0]))
            keep.append(v)
            outs.append((a, v))
            cargs.append(C.byref(v))
    getattr(lib(), name + "_")(*cargs)
    check_legacy()
    res = []
    for a, v in outs:
        if isinstance(a, np.ndarray):
            a.ravel()[0] = v.value
        res.append(v.value)
    return res[0] if len(res) == 1 else None


def _make(name):
    def f(*args):
        return _call(name, args)

    f.__name__ = name
    f.__doc__ = f"GPU drop-in for the reference subroutine {name.upper()} (see module table)."
    return f


for _n in _SIG:
    globals()[_n] = _make(_n)

__all__ = list(_SIG)
