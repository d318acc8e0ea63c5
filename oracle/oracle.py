"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference arm of bench.py, as the checker or the timed CPU
baseline.  The product package never imports this module.

Arrays follow the reference layout: a padded field is a Fortran-ordered
float64 array of shape (nx+2, ny+2, nz+2); cellvalue is (nx, ny, nz, 4);
complex spectra are complex128 (nx/2+1, ny+2, nz+2).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

dp = C.POINTER(C.c_double)
ci = C.c_int
cd = C.c_double


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
    return _lib


def P(a):
    """Pointer to a contiguous float64/complex128 numpy array (no copy)."""
    if a is None:
        return None
    assert a.flags.f_contiguous or a.flags.c_contiguous
    assert a.dtype in (np.float64, np.complex128)
    return a.ctypes.data_as(dp)


def field(nx, ny, nz, fill=0.0):
    return np.full((nx + 2, ny + 2, nz + 2), fill, dtype=np.float64, order="F")


class Grid:
    """Grid arrays of SET_C (nse_dominik.f:553-607), optionally tanh-stretched in y."""

    def __init__(self, nx, ny, nz, xl, yl, zl, y0=0.0, gamma=0.0):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.xl, self.yl, self.zl = xl, yl, zl
        arr = {}
        for d, n in (("x", nx), ("y", ny), ("z", nz)):
            for suffix in ("", "12"):
                arr[d + suffix] = np.zeros(n + 2)
                arr["d" + d + suffix] = np.zeros(n + 2)
        self.__dict__.update(arr)
        L = lib()
        if gamma == 0.0 and y0 == 0.0:
            L.or_set_c(nx, ny, nz, P(self.x), P(self.x12), P(self.y), P(self.y12), P(self.z),
                       P(self.z12), P(self.dx), P(self.dx12), P(self.dy), P(self.dy12),
                       P(self.dz), P(self.dz12), cd(xl), cd(yl), cd(zl))
        else:
            L.or_set_c_stretched(nx, ny, nz, P(self.x), P(self.x12), P(self.y), P(self.y12),
                                 P(self.z), P(self.z12), P(self.dx), P(self.dx12), P(self.dy),
                                 P(self.dy12), P(self.dz), P(self.dz12), cd(xl), cd(yl), cd(zl),
                                 cd(y0), cd(gamma))


def set_bc(u, v, w, p, T, tbot=0.0, ttop=0.0):
    nx, ny, nz = (s - 2 for s in u.shape)
    lib().or_set_bc(P(u), P(v), P(w), P(p), nx, ny, nz, P(T), cd(tbot), cd(ttop))


def p2s(FP, nx, ny, nz, FPT=None):
    if FPT is None:
        FPT = np.zeros((nx // 2 + 1, ny + 2, nz + 2), dtype=np.complex128, order="F")
    lib().or_p2s(P(FP), P(FPT), nx, ny, nz)
    return FPT


def s2p(FPT, nx, ny, nz, FP=None):
    if FP is None:
        FP = field(nx, ny, nz)
    lib().or_s2p(P(FPT), P(FP), nx, ny, nz)
    return FP


def mkp_coeffs(g):
    AC = np.zeros((g.ny, 3), order="F")
    KXZ = np.zeros((g.nx // 2 + 1, g.nz + 1), order="F")
    lib().or_mkp_coeffs(g.nx, g.ny, g.nz, P(g.dx), P(g.dy), P(g.dz), P(g.dy12), cd(g.xl),
                        cd(g.zl), P(AC), P(KXZ))
    return AC, KXZ


def spn(nx, ny, nz, AC, KXZ, PHIT):
    lib().or_spn(nx, ny, nz, P(AC), P(KXZ), P(PHIT))


def sp0b(nx, ny, nz, AC, PHIT):
    lib().or_sp0b(nx, ny, nz, P(AC), P(PHIT))


def phibc(nx, ny, nz, PHI):
    lib().or_phibc(nx, ny, nz, P(PHI))


def ctridiag(A, B):
    lib().or_ctridiag(P(A), P(B), A.shape[0])


def tridiag(A, B):
    lib().or_tridiag(P(A), P(B), A.shape[0])


def trid2(A, B):
    M, N = B.shape
    lib().or_trid2(P(A), P(B), M, N)


def tdma(a, b, c, r, n):
    u = np.zeros(n + 2)
    lib().or_tdma(P(a), P(b), P(c), P(r), P(u), n)
    return u


def cyclic(a, b, c, alpha, beta, r, n):
    x = np.zeros(n + 2)
    lib().or_cyclic(P(a), P(b), P(c), cd(alpha), cd(beta), P(r), P(x), n)
    return x


def implicit_solver(SUX, nx, dx, dx12, Re, dt, ft, fb, eta, CUX):
    lib().or_implicit_solver(P(SUX), nx, P(dx), P(dx12), cd(Re), cd(dt), cd(ft), cd(fb),
                             cd(eta), P(CUX))


def implicit_uy(SUY, ny, dy, dy12, Re, dt, ft, fb, eta, CUY):
    lib().or_implicit_uy(P(SUY), ny, P(dy), P(dy12), cd(Re), cd(dt), cd(ft), cd(fb), cd(eta),
                         P(CUY))


def implicit_vy(SVY, ny, dy, dy12, Re, dt, ft, fb, eta, CVY):
    lib().or_implicit_vy(P(SVY), ny, P(dy), P(dy12), cd(Re), cd(dt), cd(ft), cd(fb), cd(eta),
                         P(CVY))


def mkp(g, p, u_temp, v_temp, w_temp, dt, u_ta, v_ta, w_ta, u_ep2, v_ep2, w_ep2, divu, u, v,
        w, phi_work=None, Re=1.0):
    if phi_work is None:
        phi_work = field(g.nx, g.ny, g.nz)
    lib().or_mkp(P(p), P(u_temp), P(v_temp), P(w_temp), cd(dt), P(g.dx), P(g.dy), P(g.dz),
                 P(g.dx12), P(g.dy12), P(g.dz12), cd(Re), g.nx, g.ny, g.nz, P(u_ta), P(v_ta),
                 P(w_ta), P(u_ep2), P(v_ep2), P(w_ep2), P(divu), P(u), P(v), P(w), cd(g.xl),
                 cd(g.zl), P(phi_work))
    return phi_work


def set_levelset(g, phi0, nnn=2000, dtau=1.0e-3, width=1.0):
    phi = np.zeros_like(phi0)
    cv = np.zeros((g.nx, g.ny, g.nz, 4), order="F")
    lib().or_set_levelset(g.nx, g.ny, g.nz, P(g.dx), P(g.dx12), P(g.dy12), P(g.dz12), P(phi0),
                          P(phi), P(cv), nnn, cd(dtau), cd(width))
    return phi, cv


class OrState(C.Structure):
    _fields_ = ([(n, ci) for n in ("nx", "ny", "nz", "l")] +
                [(n, cd) for n in ("dt", "Re", "Sc", "eta", "xl", "zl", "force", "source",
                                   "tbot", "ttop", "tsolid")] +
                [(n, dp) for n in ("dx", "dy", "dz", "dx12", "dy12", "dz12",
                                   "u", "v", "w", "p", "T",
                                   "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre", "T_pre",
                                   "divu", "u_ep2", "v_ep2", "w_ep2",
                                   "cellvalue", "rhoCp", "thc",
                                   "u_v", "v_v", "w_v", "u_d", "v_d", "w_d", "u_a", "v_a", "w_a",
                                   "u_l", "v_l", "w_l", "u_temp", "v_temp", "w_temp",
                                   "u_vT", "u_dT", "u_T", "T_l", "phi_work")])


STATE_FIELDS = ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre",
                "T_pre", "divu", "u_ep2", "v_ep2", "w_ep2")
SCRATCH_FIELDS = ("u_v", "v_v", "w_v", "u_d", "v_d", "w_d", "u_a", "v_a", "w_a", "u_l", "v_l",
                  "w_l", "u_temp", "v_temp", "w_temp", "u_vT", "u_dT", "u_T", "T_l",
                  "phi_work")


class Solver:
    """The reference time loop (nse_dominik.f:261-446) on the CPU oracle.

    `fields` holds every padded array of the reference main program that the
    step touches; `cellvalue` is (nx,ny,nz,4).  Parameters default to the
    reference values (body force and heat source 1, walls and solid at T=0,
    rhoCp = thc = 1)."""

    def __init__(self, g, dt, Re, Sc, eta, force=1.0, source=1.0, tbot=0.0, ttop=0.0,
                 tsolid=0.0):
        self.g = g
        nx, ny, nz = g.nx, g.ny, g.nz
        self.f = {n: field(nx, ny, nz) for n in STATE_FIELDS + SCRATCH_FIELDS}
        self.f["rhoCp"] = field(nx, ny, nz, 1.0)
        self.f["thc"] = field(nx, ny, nz, 1.0)
        self.cellvalue = np.zeros((nx, ny, nz, 4), order="F")
        self.params = dict(dt=dt, Re=Re, Sc=Sc, eta=eta, xl=g.xl, zl=g.zl, force=force,
                           source=source, tbot=tbot, ttop=ttop, tsolid=tsolid)
        self.l = 1

    def project(self):
        """Initial projection of the benchmark workloads (the seeded field is
        "then projected divergence-free"): SET_BC (nse_dominik.f:611-753) on
        copies of u, v, w, then MKP (mkp.f:9-220) with those copies as
        u_temp, v_temp, w_temp.  MKP writes u, v, w, p, u_ta, u_ep2 and divu;
        p's ghosts are left as they are (the time loop's first SET_BC sets
        them)."""
        g = self.g
        f = self.f
        tmp = {k: f[k].copy(order="F") for k in ("u", "v", "w", "p", "T")}
        set_bc(tmp["u"], tmp["v"], tmp["w"], tmp["p"], tmp["T"], self.params["tbot"],
               self.params["ttop"])
        mkp(g, f["p"], tmp["u"], tmp["v"], tmp["w"], self.params["dt"], f["u_ta"], f["v_ta"],
            f["w_ta"], f["u_ep2"], f["v_ep2"], f["w_ep2"], f["divu"], f["u"], f["v"], f["w"],
            phi_work=f["phi_work"], Re=self.params["Re"])

    def start(self):
        """Copy the state into the AB2 history, as nse_dominik.f:246-257 does."""
        for a, b in (("u", "u_pre"), ("v", "v_pre"), ("w", "w_pre"), ("T", "T_pre")):
            self.f[b][...] = self.f[a]

    def step(self, n=1):
        g = self.g
        st = OrState(nx=g.nx, ny=g.ny, nz=g.nz, l=self.l, **self.params)
        for n_ in ("dx", "dy", "dz", "dx12", "dy12", "dz12"):
            setattr(st, n_, P(getattr(g, n_)))
        for n_, a in self.f.items():
            setattr(st, n_, P(a))
        st.cellvalue = P(self.cellvalue)
        for _ in range(n):
            lib().or_step(C.byref(st))
        self.l = st.l


def set_faithful(on):
    lib().or_set_faithful(1 if on else 0)


def num_threads():
    return lib().or_num_threads()


def _dims(a):
    return tuple(s - 2 for s in a.shape)


def set_convect(u, u_v, v, v_v, w, w_v, dt, g, force=1.0):
    nx, ny, nz = _dims(u)
    lib().or_set_convect(P(u), P(u_v), P(v), P(v_v), P(w), P(w_v), cd(dt), nx, ny, nz,
                         P(g.dx), P(g.dy), P(g.dz), P(g.dx12), P(g.dy12), P(g.dz12), cd(force))


def set_convection_for_scalar(u, v, w, dt, g, T, u_vT, rhoCp, source=1.0):
    nx, ny, nz = _dims(u)
    lib().or_set_convection_for_scalar(P(u), P(v), P(w), cd(dt), nx, ny, nz, P(g.dx), P(g.dy),
                                       P(g.dz), P(g.dx12), P(g.dy12), P(g.dz12), P(T), P(u_vT),
                                       P(rhoCp), cd(source))


def set_conduction(u, u_d, v, v_d, w, w_d, Re, dt, g):
    nx, ny, nz = _dims(u)
    lib().or_set_conduction(P(u), P(u_d), P(v), P(v_d), P(w), P(w_d), cd(Re), cd(dt), nx, ny,
                            nz, P(g.dx), P(g.dy), P(g.dz), P(g.dx12), P(g.dy12), P(g.dz12))


def set_diffusion_for_scalar(Re, dt, g, T, u_dT, Sc, thc, rhoCp):
    nx, ny, nz = _dims(T)
    lib().or_set_diffusion_for_scalar(cd(Re), cd(dt), nx, ny, nz, P(g.dx), P(g.dy), P(g.dz),
                                      P(g.dx12), P(g.dy12), P(g.dz12), P(T), P(u_dT), cd(Sc),
                                      P(thc), P(rhoCp))


def set_immersed_boundary(eta, dt, u_l, v_l, w_l, T_l, cellvalue, u_ta, v_ta, w_ta, l):
    nx, ny, nz = _dims(u_l)
    lib().or_set_immersed_boundary(cd(eta), nx, ny, nz, cd(dt), P(u_l), P(v_l), P(w_l), P(T_l),
                                   P(cellvalue), P(u_ta), P(v_ta), P(w_ta), l)


def set_explicit(u_v, u_pre, u_d, u_a, v_v, v_pre, v_d, v_a, w_v, w_pre, w_d, w_a, u_l, v_l,
                 w_l, l):
    nx, ny, nz = _dims(u_v)
    lib().or_set_explicit(P(u_v), P(u_pre), P(u_d), P(u_a), P(v_v), P(v_pre), P(v_d), P(v_a),
                          P(w_v), P(w_pre), P(w_d), P(w_a), P(u_l), P(v_l), P(w_l), nx, ny, nz,
                          l)


def set_explicit_for_tempreture(u_vT, u_dT, u_T, T_pre, T_l, l):
    nx, ny, nz = _dims(u_vT)
    lib().or_set_explicit_for_tempreture(P(u_vT), P(u_dT), P(u_T), P(T_pre), P(T_l), nx, ny,
                                         nz, l)


def solve_u_temp(u_a, v_a, w_a, g, Re, dt, eta, cellvalue, u, v, w):
    nx, ny, nz = _dims(u_a)
    lib().or_solve_u_temp(P(u_a), P(v_a), P(w_a), nx, ny, nz, P(g.dx), P(g.dy), P(g.dz),
                          P(g.dx12), P(g.dy12), P(g.dz12), cd(Re), cd(dt), cd(eta),
                          P(cellvalue), P(u), P(v), P(w))


def solve_t(u_T, g, Re, Sc, dt, rhoCp, thc, cellvalue, eta, ft_y=0.0, fb_y=0.0):
    nx, ny, nz = _dims(u_T)
    lib().or_solve_t(P(u_T), nx, ny, nz, P(g.dx), P(g.dy), P(g.dz), P(g.dx12), P(g.dy12),
                     P(g.dz12), cd(Re), cd(Sc), cd(dt), P(rhoCp), P(thc), P(cellvalue), cd(eta),
                     cd(ft_y), cd(fb_y))


def implicit_ty(STY, ny, dy, dy12, Re, Sc, dt, lly, rry, ft, fb, CUY, eta):
    lib().or_implicit_ty(P(STY), ny, P(dy), P(dy12), cd(Re), cd(Sc), cd(dt), P(lly), P(rry),
                         cd(ft), cd(fb), P(CUY), cd(eta))


def implicit_tx(STX, nx, dx, dx12, Re, Sc, dt, llx, rrx, ft, fb, eta, CUX):
    lib().or_implicit_tx(P(STX), nx, P(dx), P(dx12), cd(Re), cd(Sc), cd(dt), P(llx), P(rrx),
                         cd(ft), cd(fb), cd(eta), P(CUX))
