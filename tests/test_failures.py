"""Failure detection of the C-ABI, without faulting a GPU: every failure is made
on the host (a bad argument, a non-finite value in an uploaded field, an
allocation cap set from the host) and must come back as a status code, with
the library still usable afterwards.

The reference checks nothing (it only prints the Courant number,
nse_dominik.f:2519-2600); the statuses are the library's own (nsegpu.h).
"""
import ctypes as C
import math

import numpy as np
import pytest

from vtkmakecompare_b200 import NseError, lib
from vtkmakecompare_b200 import legacy as G
from vtkmakecompare_b200 import solver as S
from vtkmakecompare_b200 import workload as W

NSE_OK, NSE_ERR_ARG, NSE_ERR_CUDA, NSE_ERR_NOMEM, NSE_ERR_NONFINITE = 0, 1, 2, 3, 4


def create(cfg):
    L = S._sig()
    h = C.c_void_p()
    st = L.nse_ctx_create(C.byref(cfg), C.byref(h))
    return st, h


def destroy(h):
    if h.value:
        S._sig().nse_ctx_destroy(h)


# sizes and parameters the resident API refuses before it touches a GPU
BAD_CONFIGS = [
    dict(nx=0, ny=16, nz=16),                # empty
    dict(nx=16, ny=2, nz=16),                # fewer than 3 cells between the walls
    dict(nx=77, ny=16, nz=16),               # 7 * 11: not a product of 2, 3 and 5
    dict(nx=16, ny=16, nz=14),               # 2 * 7
    dict(nx=16, ny=16, nz=16, dt=0.0),       # non-positive time step
    dict(nx=16, ny=16, nz=16, dt=float("nan")),
    dict(nx=16, ny=16, nz=16, Re=-1.0),
    dict(nx=16, ny=16, nz=16, precision=7),  # no such precision
]


def bad_config(kw):
    a = dict(nx=16, ny=16, nz=16, dt=0.01, Re=100.0, precision=S.FP64)
    a.update(kw)
    return S.Config(a["nx"], a["ny"], a["nz"], a["dt"], a["Re"], 0.71, 0.0, 2 * math.pi, 2.0,
                    math.pi, precision=a["precision"])


@pytest.mark.parametrize("kw", BAD_CONFIGS)
def test_bad_dimensions_are_refused_with_err_arg(kw):
    """NSE_ERR_ARG with or without a GPU: the arguments are checked first."""
    st, h = create(bad_config(kw))
    try:
        assert st == NSE_ERR_ARG, (kw, st, lib().nse_last_error())
        assert not h.value
    finally:
        destroy(h)
        lib().nse_clear_error()


def test_legacy_bad_dimensions_record_err_arg():
    """A legacy (void) entry point records NSE_ERR_ARG for bad sizes, which the
    Python mirror raises; mkp_ with nx = 0 and a parallel_uy_ line outside
    the field are refused before any device work."""
    z = np.zeros(8)
    f = np.zeros((3, 3, 3), order="F")
    with pytest.raises(NseError) as e:
        G.mkp(f, f, f, f, 0.1, z, z, z, z, z, z, 1.0, 0, 1, 1, 0, f, f, f, f, f, f, f, f, f, f,
              1.0, 1.0)
    assert e.value.status == NSE_ERR_ARG
    cv = np.zeros((4, 4, 4, 4), order="F")
    u = np.zeros((6, 6, 6), order="F")
    with pytest.raises(NseError) as e:
        G.parallel_uy(5, 1, u, cv, 4, 4, 4, np.ones(6), np.ones(6), 100.0, 0.01, 0.0, 1)
    assert e.value.status == NSE_ERR_ARG
    with pytest.raises(NseError) as e:  # k = 5 on a 4-cell axis
        G.parallel_tx(5, 1, 4, 4, 4, u, u, u, cv, np.ones(6), np.ones(6), 100.0, 1.0, 0.01,
                      0.0)
    assert e.value.status == NSE_ERR_ARG
    lib().nse_clear_error()


def test_alloc_limit_is_settable_without_a_gpu():
    L = lib()
    L.nse_set_alloc_limit.argtypes = [C.c_longlong]
    L.nse_alloc_bytes.restype = C.c_longlong
    L.nse_set_alloc_limit(1 << 20)
    L.nse_set_alloc_limit(0)
    assert L.nse_alloc_bytes() >= 0


# ------------------------------------------------------------------ GPU ----

def channel_ctx(n=(32, 24, 16), flags=0):
    g = W.grid_arrays(*n, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = W.channel_state(g, seed=9)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    cfg = S.Config(*n, dt, 3000.0, 0.71, 1.0e4, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0, body_force=1e-3, heat_source=0.0, t_bot=1.0, t_top=0.0,
                   flags=flags)
    ctx = S.Context(cfg)
    for k in ("u", "v", "w", "T"):
        ctx.upload(k, f[k])
    ctx.start()
    return ctx, f


@pytest.mark.gpu
@pytest.mark.parametrize("kw", BAD_CONFIGS[:4])
def test_bad_dimensions_on_a_gpu(kw):
    st, h = create(bad_config(kw))
    try:
        assert st == NSE_ERR_ARG
    finally:
        destroy(h)
        lib().nse_clear_error()


@pytest.mark.gpu
def test_nonfinite_value_is_detected_and_the_context_stays_usable():
    """NSE_FLAG_CHECK_FINITE: a NaN planted in the uploaded u (on the host)
    makes nse_step return NSE_ERR_NONFINITE after the step it spread in;
    after finite fields are uploaded again the same context steps normally."""
    ctx, f = channel_ctx(flags=S.FLAG_CHECK_FINITE)
    with ctx:
        ctx.step(2)
        bad = f["u"].copy(order="F")
        bad[5, 7, 3] = np.nan
        ctx.upload("u", bad)
        with pytest.raises(NseError) as e:
            ctx.step(1)
        assert e.value.status == NSE_ERR_NONFINITE
        assert ctx.monitor()["nonfinite"] > 0
        for k in ("u", "v", "w", "T"):
            ctx.upload(k, f[k])
        for k in ("u_pre", "v_pre", "w_pre", "T_pre"):
            ctx.upload(k, f[k[0]])
        for k in ("u_ta", "v_ta", "w_ta", "p"):
            ctx.upload(k, np.zeros_like(f["u"]))
        ctx.step(2)
        mon = ctx.monitor()
        assert mon["nonfinite"] == 0 and mon["max_divu"] < 1e-10
    # an infinity in the mask is caught the same way
    ctx, f = channel_ctx(flags=S.FLAG_CHECK_FINITE)
    with ctx:
        c1 = np.zeros((32, 24, 16), order="F")
        c1[3, 4, 5] = np.inf
        ctx.upload("cellvalue", c1)
        with pytest.raises(NseError) as e:
            ctx.step(1)
        assert e.value.status == NSE_ERR_NONFINITE


@pytest.mark.gpu
def test_allocation_cap_gives_err_nomem_and_releases_everything():
    """A cap on the library's device memory, set from the host, makes context
    creation fail with NSE_ERR_NOMEM; the partly built context is released
    (the library's byte count returns to where it was) and, with the cap
    lifted, the same configuration is created and steps."""
    L = lib()
    L.nse_set_alloc_limit.argtypes = [C.c_longlong]
    L.nse_alloc_bytes.restype = C.c_longlong
    n = (128, 96, 128)
    cfg = S.Config(*n, 1e-3, 1000.0, 0.71, 0.0, 2 * math.pi, 2.0, math.pi)
    before = L.nse_alloc_bytes()
    try:
        L.nse_set_alloc_limit(before + 200 * 1024 * 1024)  # 200 MB: less than one context
        st, h = create(cfg)
        assert st == NSE_ERR_NOMEM, (st, L.nse_last_error())
        assert not h.value
        assert L.nse_alloc_bytes() == before
        lib().nse_clear_error()
    finally:
        L.nse_set_alloc_limit(0)
    st, h = create(cfg)
    try:
        assert st == NSE_OK
        assert L.nse_alloc_bytes() > before + 200 * 1024 * 1024
        assert S._sig().nse_step(h, 1) == NSE_OK
    finally:
        destroy(h)
    assert L.nse_alloc_bytes() == before
