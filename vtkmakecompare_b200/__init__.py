"""B200-native drop-in for the fractional-step hot path of
DominikHenzel/vtkmakeCompare (3-D incompressible Navier-Stokes + heat with
volume penalisation).

The product is libnsegpu.so (CUDA kernels for sm_100a behind a C-ABI that
exports the reference's Fortran subroutine names).  This package is the
Python host side: `legacy` mirrors the reference subroutines one for one
(same names, arguments and in-place semantics, numpy arrays in the
reference layout) and `solver` wraps the resident API.

There is no CPU fallback: importing the library on a machine without a
usable sm_100 GPU succeeds, but every compute call raises NseError.
"""
import ctypes as _C
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_HERE, "libnsegpu.so")
_lib = None


class NseError(RuntimeError):
    """A libnsegpu call failed (status code and message from nse_last_error)."""

    def __init__(self, status, msg):
        super().__init__(f"nsegpu status {status}: {msg}")
        self.status = status


def lib():
    """Load libnsegpu.so (built in-tree by build.py); raise if it is missing."""
    global _lib
    if _lib is None:
        if not _os.path.exists(LIB_PATH):
            raise NseError(-1, f"{LIB_PATH} is missing: run vtkmakecompare_b200/build.py")
        _lib = _C.CDLL(LIB_PATH)
        _lib.nse_last_error.restype = _C.c_char_p
        _lib.nse_last_status.restype = _C.c_int
    return _lib


def last_error():
    L = lib()
    return L.nse_last_status(), L.nse_last_error().decode(errors="replace")


def check_legacy():
    """Raise NseError if the previous legacy (void) call recorded an error."""
    st, msg = last_error()
    if st != 0:
        lib().nse_clear_error()
        raise NseError(st, msg)


def check(status):
    if status != 0:
        st, msg = last_error()
        lib().nse_clear_error()
        raise NseError(status, msg)
