"""nse_spn_noalloc: the spectral tridiagonal solve for callers that cannot
allocate GPU memory (their device arrays belong to a framework or to a
Fortran data region, or their time loop must not hit cudaMalloc, which
stalls the whole device).  The caller passes device pointers; the solve's
scratch is a fixed array inside the library.

Checked through the C-ABI against the host-array entry point spn_ and the
CPU oracle's SPN (mkp.f:223-260) on two calls in a row (the fixed scratch
keeps the previous call's contents), including an odd size; a size beyond
the fixed scratch, or beyond the launch grid's limit in z, must be refused
with NSE_ERR_LIMIT.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import rel_l2
from vtkmakecompare_b200 import legacy as G
from vtkmakecompare_b200 import lib

pytestmark = pytest.mark.gpu

NSE_OK, NSE_ERR_LIMIT = 0, 5


def entry():
    f = lib().nse_spn_noalloc
    f.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 4
    f.restype = ctypes.c_int
    return f


def to_device(torch, a):
    flat = np.ascontiguousarray(np.asarray(a).ravel(order="F"))
    if flat.dtype == np.complex128:
        flat = flat.view(np.float64)
    return torch.from_numpy(flat.copy()).to("cuda:0")


@pytest.mark.parametrize("n", [(32, 24, 20), (6, 5, 3)])
def test_noalloc_spn_matches_spn_on_two_calls(n):
    import torch
    nx, ny, nz = n
    g = O.Grid(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    AC, KXZ = O.mkp_coeffs(g)
    dAC, dK = to_device(torch, AC), to_device(torch, KXZ)
    H = nx // 2 + 1
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rng = np.random.default_rng(100 + call)
        PT = np.asfortranarray(rng.standard_normal((H, ny + 2, nz + 2)) +
                               1j * rng.standard_normal((H, ny + 2, nz + 2)))
        ref = PT.copy(order="F")
        G.spn(nx, ny, nz, AC, KXZ, ref)
        cpu = PT.copy(order="F")
        O.spn(nx, ny, nz, AC, KXZ, cpu)
        d = to_device(torch, PT)
        st = entry()(nx, ny, nz, dAC.data_ptr(), dK.data_ptr(), d.data_ptr(), stream)
        assert st == NSE_OK, lib().nse_last_error()
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(np.complex128).reshape(PT.shape, order="F")
        assert rel_l2(got, ref) < 1e-13
        assert rel_l2(got, cpu) < 1e-13
        # entries SPN does not write are untouched
        assert np.array_equal(got[:, 0, :], PT[:, 0, :])
        assert np.array_equal(got[:, ny + 1, :], PT[:, ny + 1, :])
        assert np.array_equal(got[0, :, 0], PT[0, :, 0])


def test_noalloc_spn_refuses_sizes_beyond_its_scratch():
    import torch
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = buf.data_ptr()
    st = entry()(512, 256, 512, p, p, p, torch.cuda.current_stream().cuda_stream)
    assert st == NSE_ERR_LIMIT
    lib().nse_clear_error()
    # fits the scratch (2 * 1 * 70000 values) but not the launch grid in z
    st = entry()(2, 1, 70000, p, p, p, torch.cuda.current_stream().cuda_stream)
    assert st == NSE_ERR_LIMIT
    lib().nse_clear_error()
    assert torch.all(buf == 0)
