"""Resident solver: the fields stay in HBM across time steps (nse_ctx_* C-ABI).

`Context` owns one device context.  A step is the reference time-loop body
(nse_dominik.f:290-446): boundary conditions, fused explicit right-hand side,
penalised ADI line solves (u, v, w then T), and the FFT projection (MKP).
"""
import ctypes as C

import numpy as np

from . import NseError, check, lib

FIELDS = ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre",
          "T_pre", "divu", "u_ep2", "v_ep2", "w_ep2", "phi", "cellvalue")
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
FP64, MIXED = 0, 1
PHASES = ("set_bc", "rhs", "y_vel", "z_vel", "x_vel", "y_T", "x_T", "z_T", "set_bc_temp",
          "fft_x_fwd", "fft_z_fwd", "spn", "fft_z_inv", "fft_x_inv", "phibc", "refine",
          "correct")
FLAG_CHECK_FINITE = 1
FLAG_EXACT = 4
FLAG_REFINE2 = 8
FLAG_POISSON64 = 16
FLAG_MATH64 = 32
FLAG_LINES64 = 64
FLAG_ONE_STREAM = 128
FLAG_POISSON3 = 256
FLAG_POISSON32 = 512
FLAG_LINES_TMA = 1024
FLAG_NO_AUTOTUNE = 2048
FLAG_SPN_TMA = 4096
FLAG_MID_SLICES = 8192
FLAG_SPN_CPASYNC = 16384


class Config(C.Structure):
    """nse_config of include/nsegpu.h.  Defaults are the reference's values
    (body force and heat source 1, walls and solid at T = 0, rhoCp = thc = 1,
    uniform grid)."""

    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dt", C.c_double), ("Re", C.c_double), ("Sc", C.c_double),
                ("eta", C.c_double), ("xl", C.c_double), ("yl", C.c_double),
                ("zl", C.c_double), ("y0", C.c_double), ("ystretch", C.c_double),
                ("body_force", C.c_double), ("heat_source", C.c_double),
                ("t_bot", C.c_double), ("t_top", C.c_double), ("t_solid", C.c_double),
                ("rho_cp", C.c_double), ("thc", C.c_double),
                ("precision", C.c_int), ("flags", C.c_int)]

    def __init__(self, nx, ny, nz, dt, Re, Sc, eta, xl, yl, zl, y0=0.0, ystretch=0.0,
                 body_force=1.0, heat_source=1.0, t_bot=0.0, t_top=0.0, t_solid=0.0,
                 rho_cp=1.0, thc=1.0, precision=FP64, flags=0):
        super().__init__(nx, ny, nz, dt, Re, Sc, eta, xl, yl, zl, y0, ystretch, body_force,
                         heat_source, t_bot, t_top, t_solid, rho_cp, thc, precision, flags)


class AdjointConfig(C.Structure):
    """nse_adjoint_config of include/nsegpu.h"""

    _fields_ = [("nsteps", C.c_int), ("checkpoint_every", C.c_int), ("avg_from", C.c_int)]


def _sig():
    L = lib()
    vp = C.c_void_p
    L.nse_ctx_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    for n in ("nse_ctx_destroy", "nse_start", "nse_project", "nse_poisson", "nse_sync",
              "nse_ctx_get_step"):
        getattr(L, n).argtypes = [vp]
    L.nse_ctx_set_stream.argtypes = [vp, vp]
    L.nse_ctx_upload.argtypes = [vp, C.c_int, vp]
    L.nse_ctx_download.argtypes = [vp, C.c_int, vp]
    L.nse_ctx_set_step.argtypes = [vp, C.c_int]
    L.nse_step.argtypes = [vp, C.c_int]
    L.nse_monitor.argtypes = [vp, vp]
    L.nse_ctx_write_output.argtypes = [vp, C.c_char_p]
    L.nse_ctx_write_field.argtypes = [vp, C.c_char_p, C.c_double, C.c_char_p]
    L.nse_ctx_read_field.argtypes = [vp, C.c_char_p]
    L.nse_levelset.argtypes = [vp, vp, vp, C.c_int, C.c_double, C.c_double]
    L.nse_ctx_grid.argtypes = [vp] + [vp] * 12
    L.nse_ctx_profile.argtypes = [vp, C.c_int]
    L.nse_ctx_launch_shapes.argtypes = [vp, vp]
    L.nse_ctx_set_shapes.argtypes = [vp, C.c_int, C.c_int]
    L.nse_ctx_set_line_shapes.argtypes = [vp, C.c_int, C.c_int]
    L.nse_ctx_phase_times.argtypes = [vp, vp, C.c_int, vp]
    L.nse_launch_count.restype = C.c_longlong
    L.nse_ensemble_create.argtypes = [vp, C.c_int, C.c_int, C.POINTER(vp)]
    L.nse_ensemble_step.argtypes = [vp, C.c_int]
    L.nse_ensemble_set_stream.argtypes = [vp, vp]
    L.nse_ensemble_sync.argtypes = [vp]
    L.nse_ensemble_destroy.argtypes = [vp]
    L.nse_adjoint_create.argtypes = [vp, C.POINTER(AdjointConfig), C.POINTER(vp)]
    L.nse_adjoint_set_weight.argtypes = [vp, C.c_int, vp]
    L.nse_adjoint_objective.argtypes = [vp, vp]
    L.nse_adjoint_gradient.argtypes = [vp, vp, vp]
    L.nse_adjoint_download.argtypes = [vp, C.c_int, vp]
    L.nse_adjoint_destroy.argtypes = [vp]
    return L


def launch_count():
    """Kernel launches issued by libnsegpu.so in this process."""
    return int(_sig().nse_launch_count())


class Context:
    def __init__(self, cfg: Config):
        self.L = _sig()
        self.cfg = cfg
        h = C.c_void_p()
        check(self.L.nse_ctx_create(C.byref(cfg), C.byref(h)))
        self.h = h
        n = cfg.nx, cfg.ny, cfg.nz
        self.shape = (n[0] + 2, n[1] + 2, n[2] + 2)
        self.grid = {k: np.zeros(m + 2) for k, m in
                     (("x", n[0]), ("x12", n[0]), ("y", n[1]), ("y12", n[1]), ("z", n[2]),
                      ("z12", n[2]), ("dx", n[0]), ("dx12", n[0]), ("dy", n[1]),
                      ("dy12", n[1]), ("dz", n[2]), ("dz12", n[2]))}
        g = self.grid
        check(self.L.nse_ctx_grid(self.h, *[g[k].ctypes.data for k in
                                            ("x", "x12", "y", "y12", "z", "z12", "dx", "dx12",
                                             "dy", "dy12", "dz", "dz12")]))

    def close(self):
        if getattr(self, "h", None):
            self.L.nse_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _fshape(self, name):
        c = self.cfg
        return (c.nx, c.ny, c.nz) if name == "cellvalue" else self.shape

    def upload(self, name, arr):
        a = np.asfortranarray(arr, dtype=np.float64)
        want = self._fshape(name)
        if name == "cellvalue" and a.ndim == 4:
            a = np.asfortranarray(a[..., 0])
        if a.shape != want:
            raise ValueError(f"{name}: shape {a.shape}, expected {want}")
        check(self.L.nse_ctx_upload(self.h, FIELD_ID[name], a.ctypes.data))

    def upload_ptr(self, name, ptr):
        """Upload from a host address (e.g. a pinned torch buffer)."""
        check(self.L.nse_ctx_upload(self.h, FIELD_ID[name], ptr))

    def download(self, name, out=None):
        if out is None:
            out = np.zeros(self._fshape(name), order="F")
        check(self.L.nse_ctx_download(self.h, FIELD_ID[name], out.ctypes.data))
        return out

    def download_ptr(self, name, ptr):
        check(self.L.nse_ctx_download(self.h, FIELD_ID[name], ptr))

    def set_stream(self, stream_handle):
        check(self.L.nse_ctx_set_stream(self.h, stream_handle))

    @property
    def step_index(self):
        return self.L.nse_ctx_get_step(self.h)

    @step_index.setter
    def step_index(self, l):
        check(self.L.nse_ctx_set_step(self.h, int(l)))

    def start(self):
        check(self.L.nse_start(self.h))

    def step(self, n=1):
        check(self.L.nse_step(self.h, int(n)))

    def project(self):
        check(self.L.nse_project(self.h))

    def poisson(self):
        check(self.L.nse_poisson(self.h))

    def sync(self):
        check(self.L.nse_sync(self.h))

    def line_shapes(self):
        """Launch shapes the autotuner chose (after the first step): {"y": [u, v,
        w, T], "z": [...], "x": [...], "rhs": shape, "correct": shape, "mid": slices};
        y/z codes 0 = 16 lines per CTA, 1 = 8, 3 = 32, 2 = TMA tiles; x = lines per
        warp iteration; rhs, correct 0-3; mid = kx slices of the FP64 solve's z
        transforms and SPN (nsegpu.h, nse_ctx_launch_shapes)."""
        o = (C.c_int * 15)()
        check(self.L.nse_ctx_launch_shapes(self.h, o))
        return {"y": list(o[:4]), "z": list(o[4:8]), "x": list(o[8:12]), "rhs": o[12],
                "correct": o[13], "mid": o[14]}

    def set_line_shapes(self, yz, x):
        """Fix every partitioned line pass's launch shape (y/z code 0-3, x code
        1-4); nsegpu.h, nse_ctx_set_line_shapes."""
        check(self.L.nse_ctx_set_line_shapes(self.h, int(yz), int(x)))

    def set_shapes(self, rhs=-1, correct=-1):
        """Fix the right-hand-side and correction launch shapes (-1: autotuned);
        nsegpu.h, nse_ctx_set_shapes."""
        check(self.L.nse_ctx_set_shapes(self.h, int(rhs), int(correct)))

    def levelset(self, phi0, nnn=2000, dtau=1.0e-3, width=1.0, want_phi=True):
        a = np.asfortranarray(phi0, dtype=np.float64)
        out = np.zeros(self.shape, order="F") if want_phi else None
        check(self.L.nse_levelset(self.h, a.ctypes.data, out.ctypes.data if want_phi else None,
                                  int(nnn), float(dtau), float(width)))
        return out

    def profile(self, max_steps):
        """Record CUDA events around every phase of the next max_steps steps
        (those steps run every pass in order on the context's stream)."""
        check(self.L.nse_ctx_profile(self.h, int(max_steps)))

    def phase_times(self):
        """Summed milliseconds per phase over the profiled steps, and the step count."""
        ms = np.zeros(len(PHASES))
        n = C.c_int(0)
        check(self.L.nse_ctx_phase_times(self.h, ms.ctypes.data, len(PHASES),
                                         C.addressof(n)))
        return dict(zip(PHASES, ms.tolist())), n.value

    # the reference's output and restart files (OUTPUT / OUTFIELD / READFIELD)
    def write_output(self, root):
        """root/nseoutput2/*.dat, field.u, grid.u and root/temperature_check.dat"""
        check(self.L.nse_ctx_write_output(self.h, str(root).encode()))

    def write_field(self, path, tid, grid_path=None):
        """field.u with the time record first; grid.u at grid_path if given"""
        check(self.L.nse_ctx_write_field(self.h, str(path).encode(), float(tid),
                                         str(grid_path).encode() if grid_path else None))

    def read_field(self, path):
        """u, v, w, p, T, the level set and u_ta, v_ta, w_ta from a field.u
        without a time record (the one OUTPUT writes)"""
        check(self.L.nse_ctx_read_field(self.h, str(path).encode()))

    def monitor(self):
        out = np.zeros(6)
        check(self.L.nse_monitor(self.h, out.ctypes.data))
        return {"max_divu": out[0], "u_int": out[1], "v_int": out[2], "w_int": out[3],
                "T_int": out[4], "nonfinite": int(out[5])}


__all__ = ["Config", "Context", "FIELDS", "FP64", "MIXED", "FLAG_CHECK_FINITE", "FLAG_EXACT", "FLAG_ONE_STREAM",
           "NseError"]


class Ensemble:
    """Independent cases (Contexts) stepped together on `nstreams` streams,
    replaying a captured CUDA graph of two steps of all cases after the first
    step (nse_ensemble_*)."""

    def __init__(self, contexts, nstreams=8):
        self.L = _sig()
        self.cases = list(contexts)
        arr = (C.c_void_p * len(self.cases))(*[c.h.value for c in self.cases])
        h = C.c_void_p()
        check(self.L.nse_ensemble_create(arr, len(self.cases), int(nstreams), C.byref(h)))
        self.h = h

    def step(self, n=1):
        check(self.L.nse_ensemble_step(self.h, int(n)))

    def set_stream(self, stream):
        """graph replays on the caller's cudaStream_t (e.g. torch's cuda_stream)"""
        check(self.L.nse_ensemble_set_stream(self.h, stream))

    def sync(self):
        check(self.L.nse_ensemble_sync(self.h))

    def close(self):
        if self.h:
            self.L.nse_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def adj_ns_scalar(dt, g, T, T_final):
    """set_adj_NS_scalar (adjoint.f:185-211) with the adjoint temperature given
    (nse_adj_ns_scalar); g: grid dict with dx12, dy12, dz12.  Returns padded
    u_s, v_s, w_s (interior written)."""
    L = _sig()
    vp = C.c_void_p
    L.nse_adj_ns_scalar.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
    T = np.asfortranarray(T, dtype=np.float64)
    Tf = np.asfortranarray(T_final, dtype=np.float64)
    nx, ny, nz = (s - 2 for s in T.shape)
    out = [np.zeros(T.shape, order="F") for _ in range(3)]
    d = C.c_double(dt)
    check(L.nse_adj_ns_scalar(C.addressof(d), nx, ny, nz, g["dx12"].ctypes.data,
                              g["dy12"].ctypes.data, g["dz12"].ctypes.data, T.ctypes.data,
                              Tf.ctypes.data, *[o.ctypes.data for o in out]))
    return out


class Adjoint:
    """Discrete adjoint of `nsteps` FP64 steps of a Context (nse_adjoint_*).

    J = mean over steps avg_from..nsteps of the wall heat flux at y = y0 plus
    sum_f <W_f, f after nsteps> for the weights set with `set_weight`.
    `gradient()` returns (J, dJ/dc1) with dJ/dc1 shaped (nx, ny, nz); the
    adjoint of the initial state is then `initial_adjoint(name)`.  Both calls
    run from the context's current state and leave it after nsteps steps."""

    def __init__(self, ctx, nsteps, checkpoint_every=20, avg_from=None):
        self.L = _sig()
        self.ctx = ctx
        avg_from = nsteps if avg_from is None else avg_from
        self.cfg = AdjointConfig(int(nsteps), int(checkpoint_every), int(avg_from))
        h = C.c_void_p()
        check(self.L.nse_adjoint_create(ctx.h, C.byref(self.cfg), C.byref(h)))
        self.h = h

    def set_weight(self, name, weights):
        if weights is None:
            check(self.L.nse_adjoint_set_weight(self.h, FIELD_ID[name], None))
            return
        w = np.asfortranarray(weights, dtype=np.float64)
        if w.shape != self.ctx.shape:
            raise ValueError(f"weights of {name}: shape {w.shape}, expected {self.ctx.shape}")
        self._keep = getattr(self, "_keep", {})
        self._keep[name] = w
        check(self.L.nse_adjoint_set_weight(self.h, FIELD_ID[name], w.ctypes.data))

    def objective(self):
        J = C.c_double()
        check(self.L.nse_adjoint_objective(self.h, C.byref(J)))
        return J.value

    def gradient(self):
        c = self.ctx.cfg
        g = np.zeros((c.nx, c.ny, c.nz), order="F")
        J = C.c_double()
        check(self.L.nse_adjoint_gradient(self.h, C.byref(J), g.ctypes.data))
        return J.value, g

    def initial_adjoint(self, name):
        out = np.zeros(self.ctx.shape, order="F")
        check(self.L.nse_adjoint_download(self.h, FIELD_ID[name], out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.nse_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

