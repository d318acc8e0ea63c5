"""The fractional time step and its exact discrete adjoint, restated with numpy.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU
adjoint.  The product package never imports this module.

Forward (`step`): one time step of nse_dominik.f:290-446 for the volume-
penalised channel with heat transfer, the same arithmetic as the C oracle's
or_step (oracle/nse_oracle.cpp):
  SET_BC :611-753, SET_CONVECT :757-831, SET_CONVECTION_FOR_SCALAR :834-884,
  SET_CONDUCTION :888-945, SET_DIFFUSION_FOR_SCALAR :950-1004,
  SET_IMMERSED_BOUNDARY :1011-1129, SET_EXPLICIT :1132-1341, the penalised
  updates :387-396 / :1358-1433, the ADI line solves implicit_uy/vy/Ty
  :1505-1870 and implicit_solver/cyclic periodic_implicit.f:1-93 (as the
  dense interior systems they are equivalent to), and MKP mkp.f:9-220.
It records what the adjoint needs: the state at the start of the step and the
input and output of every line-solve pass.

Adjoint (`adjoint_step`): the transpose of the step's Jacobian with respect to
the state (interior values of u, v, w, T, u_ta, v_ta, w_ta and the AB2
histories) and to the penalisation masks c2, c3, c4 (face averages) and c1,
applied in reverse order:
  * MKP: the correction's gradient transposed, the Poisson map transposed
    (P2S -> transposed SPN / SP0B -> S2P; the Hermitian weights of the
    half spectrum cancel per wavenumber), the divergence transposed;
  * each line pass x = A(c)^-1 r: r_bar = A^-T x_bar and, with
    alpha_j = 1 + dt eta c_j, c_bar_j += r_bar_j dt eta / alpha_j (r_j - x_j);
  * penalised updates, AB2, immersed boundary: pointwise transposes;
  * convection (bilinear), conduction and scalar diffusion (linear): the
    stencils' partial derivatives scattered to the cells they read;
  * SET_BC: ghost cells folded back onto the interior cells they copy.
Ghost values of the state are never state: every step starts with SET_BC.

`restated adjoint.f`: set_adj_convect (adjoint.f:1-125),
set_adj_convection_for_scalar (:128-181) and set_adj_NS_scalar (:185-211) as
the reference writes them (including its index slips, see the functions).
"""
import numpy as np

from oracle import oracle as O


# ------------------------------------------------------------------ helpers
def dims(a):
    return a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2


def V(a, di=0, dj=0, dk=0):
    """interior block of a padded array shifted by (di, dj, dk)"""
    nx, ny, nz = dims(a)
    return a[1 + di:nx + 1 + di, 1 + dj:ny + 1 + dj, 1 + dk:nz + 1 + dk]


def acc(a, di, dj, dk, val):
    """a[interior + (di,dj,dk)] += val"""
    t = V(a, di, dj, dk)
    t += val


def gx(a, o=0):
    n = len(a) - 2
    return a[1 + o:n + 1 + o][:, None, None]


def gy(a, o=0):
    n = len(a) - 2
    return a[1 + o:n + 1 + o][None, :, None]


def gz(a, o=0):
    n = len(a) - 2
    return a[1 + o:n + 1 + o][None, None, :]


def padded(nx, ny, nz):
    return np.zeros((nx + 2, ny + 2, nz + 2), order="F")


def embed(interior):
    nx, ny, nz = interior.shape
    p = padded(nx, ny, nz)
    V(p)[...] = interior
    return p


class Params:
    """Grid and physical parameters of a run (the reference's variables)."""

    def __init__(self, g, dt, Re, Sc, eta, force=1.0, source=1.0, tbot=0.0, ttop=0.0,
                 tsolid=0.0, rho_cp=1.0, thc=1.0):
        self.g = g
        self.nx, self.ny, self.nz = g.nx, g.ny, g.nz
        self.dt, self.Re, self.Sc, self.eta = dt, Re, Sc, eta
        self.force, self.source = force, source
        self.tbot, self.ttop, self.tsolid = tbot, ttop, tsolid
        self.R, self.L = rho_cp, thc
        self.AC, self.KXZ = O.mkp_coeffs(g)


# ---------------------------------------------------------------- SET_BC --
def set_bc(A, kind, tb=0.0, tt=0.0):
    """nse_dominik.f:611-753 in place; kind 'u' (u, w), 'v', 'T', 'p'."""
    nx, ny, nz = dims(A)
    A[0] = A[nx]
    A[nx + 1] = A[1]
    if kind == "u":
        A[:, 0] = -A[:, 1]
        A[:, ny + 1] = -A[:, ny]
    elif kind == "v":
        A[:, 0] = 0.0
        A[:, ny] = 0.0
    elif kind == "T":
        A[:, 0] = 2.0 * tb - A[:, 1] if tb != 0.0 else -A[:, 1]
        A[:, ny + 1] = 2.0 * tt - A[:, ny] if tt != 0.0 else -A[:, ny]
    else:
        A[:, 0] = A[:, 1]
        A[:, ny + 1] = A[:, ny]
    A[:, :, 0] = A[:, :, nz]
    A[:, :, nz + 1] = A[:, :, 1]


def set_bc_adj(B, kind):
    """transpose of set_bc (its statements reversed) on an adjoint array"""
    nx, ny, nz = dims(B)
    B[:, :, 1] += B[:, :, nz + 1]
    B[:, :, nz + 1] = 0.0
    B[:, :, nz] += B[:, :, 0]
    B[:, :, 0] = 0.0
    if kind in ("u", "T"):
        B[:, ny] -= B[:, ny + 1]
        B[:, ny + 1] = 0.0
        B[:, 1] -= B[:, 0]
        B[:, 0] = 0.0
    elif kind == "v":
        B[:, ny] = 0.0
        B[:, 0] = 0.0
    else:
        B[:, ny] += B[:, ny + 1]
        B[:, ny + 1] = 0.0
        B[:, 1] += B[:, 0]
        B[:, 0] = 0.0
    B[1] += B[nx + 1]
    B[nx + 1] = 0.0
    B[nx] += B[0]
    B[0] = 0.0


# ------------------------------------------------------ explicit stencils --
def convect(P, u, v, w):
    """SET_CONVECT nse_dominik.f:757-831 (interior u_v, v_v, w_v)"""
    g, dt = P.g, P.dt
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    uc, vc, wc = V(u), V(v), V(w)
    U1 = ((uc + V(u, 1)) * (uc + V(u, 1)) - (uc + V(u, -1)) * (uc + V(u, -1))) / gx(dx12)
    U2 = ((V(v, 1) * gx(dx, 1) + vc * gx(dx)) * (V(u, 0, 1) + uc) -
          (V(v, 1, -1) * gx(dx, 1) + V(v, 0, -1) * gx(dx)) * (uc + V(u, 0, -1))) / gx(dx12) / gy(dy)
    U3 = ((V(w, 1) * gx(dx, 1) + wc * gx(dx)) * (V(u, 0, 0, 1) + uc) -
          (V(w, 1, 0, -1) * gx(dx, 1) + V(w, 0, 0, -1) * gx(dx)) * (uc + V(u, 0, 0, -1))) / gx(dx12) / gz(dz)
    uv = 0.25 * (-U1 - U2 - U3) * dt + P.force * dt
    V1 = ((V(u, 0, 1) * gy(dy, 1) + uc * gy(dy)) * (V(v, 1) + vc) -
          (V(u, -1, 1) * gy(dy, 1) + V(u, -1) * gy(dy)) * (vc + V(v, -1))) / gy(dy12) / gx(dx)
    V2 = ((vc + V(v, 0, 1)) * (vc + V(v, 0, 1)) - (vc + V(v, 0, -1)) * (vc + V(v, 0, -1))) / gy(dy12)
    V3 = ((V(w, 0, 1) * gy(dy, 1) + wc * gy(dy)) * (V(v, 0, 0, 1) + vc) -
          (V(w, 0, 1, -1) * gy(dy, 1) + V(w, 0, 0, -1) * gy(dy)) * (vc + V(v, 0, 0, -1))) / gy(dy12) / gz(dz)
    vv = 0.25 * (-V1 - V2 - V3) * dt
    W1 = ((V(u, 0, 0, 1) * gz(dz, 1) + uc * gz(dz)) * (V(w, 1) + wc) -
          (V(u, -1, 0, 1) * gz(dz, 1) + V(u, -1) * gz(dz)) * (wc + V(w, -1))) / gz(dz12) / gx(dx)
    W2 = ((V(v, 0, 0, 1) * gz(dz, 1) + vc * gz(dz)) * (V(w, 0, 1) + wc) -
          (V(v, 0, -1, 1) * gz(dz, 1) + V(v, 0, -1) * gz(dz)) * (wc + V(w, 0, -1))) / gz(dz12) / gy(dy)
    W3 = ((wc + V(w, 0, 0, 1)) * (wc + V(w, 0, 0, 1)) - (wc + V(w, 0, 0, -1)) * (wc + V(w, 0, 0, -1))) / gz(dz12)
    wv = 0.25 * (-W1 - W2 - W3) * dt
    return uv, vv, wv


def convect_adj(P, u, v, w, uvb, vvb, wvb, ub, vb, wb):
    """adds (d convect / d(u,v,w))^T (uvb, vvb, wvb) to the padded ub, vb, wb"""
    g, dt = P.g, P.dt
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    uc, vc, wc = V(u), V(v), V(w)

    def square_term(fb, f, q, d12, e):
        # ((fc + f+)^2 - (fc + f-)^2) / d12 along unit offset e
        m = q / d12
        ap = V(f) + V(f, *e)
        am = V(f) + V(f, *[-x for x in e])
        acc(fb, 0, 0, 0, 2.0 * m * (ap - am))
        acc(fb, *e, 2.0 * m * ap)
        acc(fb, *[-x for x in e], -2.0 * m * am)

    def cross_term(fb, f, gb, gfield, q, e_f, e_g, wp, wc_, scale):
        # (Gp (f+ + fc) - Gm (fc + f-)) * scale with
        # Gp = g[e_g] wp + g[0] wc_, Gm = g[e_g - e_f] wp + g[-e_f] wc_
        m = q * scale
        neg_f = tuple(-x for x in e_f)
        gm_sh = tuple(a - b for a, b in zip(e_g, e_f))
        Gp = V(gfield, *e_g) * wp + V(gfield) * wc_
        Gm = V(gfield, *gm_sh) * wp + V(gfield, *neg_f) * wc_
        sp = V(f, *e_f) + V(f)
        sm = V(f) + V(f, *neg_f)
        acc(fb, *e_f, m * Gp)
        acc(fb, 0, 0, 0, m * (Gp - Gm))
        acc(fb, *neg_f, -m * Gm)
        acc(gb, *e_g, m * wp * sp)
        acc(gb, 0, 0, 0, m * wc_ * sp)
        acc(gb, *gm_sh, -m * wp * sm)
        acc(gb, *neg_f, -m * wc_ * sm)

    ex, ey, ez = (1, 0, 0), (0, 1, 0), (0, 0, 1)
    qu = -0.25 * dt * uvb
    qv = -0.25 * dt * vvb
    qw = -0.25 * dt * wvb
    # u_v: U1, U2 (v along x face pair, u along y), U3
    square_term(ub, u, qu, gx(dx12), ex)
    cross_term(ub, u, vb, v, qu, ey, ex, gx(dx, 1), gx(dx), 1.0 / gx(dx12) / gy(dy))
    cross_term(ub, u, wb, w, qu, ez, ex, gx(dx, 1), gx(dx), 1.0 / gx(dx12) / gz(dz))
    # v_v: V1 (u), V2, V3 (w)
    cross_term(vb, v, ub, u, qv, ex, ey, gy(dy, 1), gy(dy), 1.0 / gy(dy12) / gx(dx))
    square_term(vb, v, qv, gy(dy12), ey)
    cross_term(vb, v, wb, w, qv, ez, ey, gy(dy, 1), gy(dy), 1.0 / gy(dy12) / gz(dz))
    # w_v: W1 (u), W2 (v), W3
    cross_term(wb, w, ub, u, qw, ex, ez, gz(dz, 1), gz(dz), 1.0 / gz(dz12) / gx(dx))
    cross_term(wb, w, vb, v, qw, ey, ez, gz(dz, 1), gz(dz), 1.0 / gz(dz12) / gy(dy))
    square_term(wb, w, qw, gz(dz12), ez)
    _ = (uc, vc, wc)


def convect_scalar(P, u, v, w, T):
    """SET_CONVECTION_FOR_SCALAR nse_dominik.f:834-884 with rhoCp = R"""
    g, dt, R = P.g, P.dt, P.R
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    Tc = V(T)
    UT = (-((R * V(T, -1) * gx(dx) + R * Tc * gx(dx, -1)) * V(u, -1)) / 2.0 / gx(dx12, -1) +
          ((R * Tc * gx(dx, 1) + R * V(T, 1) * gx(dx)) * V(u)) / 2.0 / gx(dx12)) / gx(dx)
    VT = (-((R * V(T, 0, -1) * gy(dy) + R * Tc * gy(dy, -1)) * V(v, 0, -1)) / 2.0 / gy(dy12, -1) +
          ((R * Tc * gy(dy, 1) + R * V(T, 0, 1) * gy(dy)) * V(v)) / 2.0 / gy(dy12)) / gy(dy)
    WT = (-((R * V(T, 0, 0, -1) * gz(dz) + R * Tc * gz(dz, -1)) * V(w, 0, 0, -1)) / 2.0 / gz(dz12, -1) +
          ((R * Tc * gz(dz, 1) + R * V(T, 0, 0, 1) * gz(dz)) * V(w)) / 2.0 / gz(dz12)) / gz(dz)
    return (-UT - VT - WT) * dt / R + P.source * dt


def convect_scalar_adj(P, u, v, w, T, uvTb, ub, vb, wb, Tb):
    g, dt, R = P.g, P.dt, P.R
    q = -uvTb * dt / R
    for f, fb, e, D, D12 in ((u, ub, (1, 0, 0), (g.dx, gx), (g.dx12, gx)),
                             (v, vb, (0, 1, 0), (g.dy, gy), (g.dy12, gy)),
                             (w, wb, (0, 0, 1), (g.dz, gz), (g.dz12, gz))):
        d, G = D
        d12, _ = D12
        ne = tuple(-x for x in e)
        m1 = q / 2.0 / G(d12, -1) / G(d)
        m2 = q / 2.0 / G(d12) / G(d)
        # -(R T- d + R Tc d-) f- * m1
        acc(fb, *ne, -m1 * (R * V(T, *ne) * G(d) + R * V(T) * G(d, -1)))
        acc(Tb, *ne, -m1 * R * G(d) * V(f, *ne))
        acc(Tb, 0, 0, 0, -m1 * R * G(d, -1) * V(f, *ne))
        # +(R Tc d+ + R T+ d) fc * m2
        acc(fb, 0, 0, 0, m2 * (R * V(T) * G(d, 1) + R * V(T, *e) * G(d)))
        acc(Tb, 0, 0, 0, m2 * R * G(d, 1) * V(f))
        acc(Tb, *e, m2 * R * G(d) * V(f))


def _lap_terms(g, comp):
    """(axis offset, coefficient of f+, coefficient of f-) of the three second
    differences of SET_CONDUCTION for u (0), v (1), w (2) (nse_dominik.f:900-940)"""
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    X = ((1, 0, 0), 1.0 / gx(dx, 1) / gx(dx12), 1.0 / gx(dx) / gx(dx12))
    Xs = ((1, 0, 0), 1.0 / gx(dx12) / gx(dx), 1.0 / gx(dx12, -1) / gx(dx))
    Y = ((0, 1, 0), 1.0 / gy(dy12) / gy(dy), 1.0 / gy(dy12, -1) / gy(dy))
    Ys = ((0, 1, 0), 1.0 / gy(dy, 1) / gy(dy12), 1.0 / gy(dy) / gy(dy12))
    Z = ((0, 0, 1), 1.0 / gz(dz12) / gz(dz), 1.0 / gz(dz12, -1) / gz(dz))
    Zs = ((0, 0, 1), 1.0 / gz(dz, 1) / gz(dz12), 1.0 / gz(dz) / gz(dz12))
    return {0: (X, Y, Z), 1: (Xs, Ys, Z), 2: (Xs, Y, Zs)}[comp]


def conduction(P, f, comp):
    """SET_CONDUCTION nse_dominik.f:888-945, one component"""
    g = P.g
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    fc = V(f)
    if comp == 0:
        A = ((V(f, 1) - fc) / gx(dx, 1) - (fc - V(f, -1)) / gx(dx)) / gx(dx12)
        B = ((V(f, 0, 1) - fc) / gy(dy12) - (fc - V(f, 0, -1)) / gy(dy12, -1)) / gy(dy)
        C = ((V(f, 0, 0, 1) - fc) / gz(dz12) - (fc - V(f, 0, 0, -1)) / gz(dz12, -1)) / gz(dz)
    elif comp == 1:
        A = ((V(f, 1) - fc) / gx(dx12) - (fc - V(f, -1)) / gx(dx12, -1)) / gx(dx)
        B = ((V(f, 0, 1) - fc) / gy(dy, 1) - (fc - V(f, 0, -1)) / gy(dy)) / gy(dy12)
        C = ((V(f, 0, 0, 1) - fc) / gz(dz12) - (fc - V(f, 0, 0, -1)) / gz(dz12, -1)) / gz(dz)
    else:
        A = ((V(f, 1) - fc) / gx(dx12) - (fc - V(f, -1)) / gx(dx12, -1)) / gx(dx)
        B = ((V(f, 0, 1) - fc) / gy(dy12) - (fc - V(f, 0, -1)) / gy(dy12, -1)) / gy(dy)
        C = ((V(f, 0, 0, 1) - fc) / gz(dz, 1) - (fc - V(f, 0, 0, -1)) / gz(dz)) / gz(dz12)
    return P.dt / P.Re / 2.0 * (A + B + C)


def _lap_adj(fb, terms, m):
    for e, cp, cm in terms:
        ne = tuple(-x for x in e)
        acc(fb, *e, m * cp)
        acc(fb, 0, 0, 0, -m * (cp + cm))
        acc(fb, *ne, m * cm)


def conduction_adj(P, fdb, comp, fb):
    _lap_adj(fb, _lap_terms(P.g, comp), P.dt / P.Re / 2.0 * fdb)


def _harm(d, L, o):
    """harmonic-mean conductance factor of SET_DIFFUSION_FOR_SCALAR between
    cells i and i+o (o = +-1) for uniform conductivity L"""
    n = len(d) - 2
    a = d[1 + o:n + 1 + o]
    b = d[1:n + 1]
    return (a + b) / (a / L + b / L)


def _diffT_terms(P):
    g, L = P.g, P.L
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    hx = lambda o: _harm(dx, L, o)[:, None, None]
    hy = lambda o: _harm(dy, L, o)[None, :, None]
    hz = lambda o: _harm(dz, L, o)[None, None, :]
    return (((1, 0, 0), hx(1) / gx(dx12) / gx(dx), hx(-1) / gx(dx12, -1) / gx(dx)),
            ((0, 1, 0), hy(1) / gy(dy12) / gy(dy), hy(-1) / gy(dy12, -1) / gy(dy)),
            ((0, 0, 1), hz(1) / gz(dz12) / gz(dz), hz(-1) / gz(dz12, -1) / gz(dz)))


def diffusion_scalar(P, T):
    """SET_DIFFUSION_FOR_SCALAR nse_dominik.f:950-1004 for uniform thc, rhoCp"""
    tot = 0.0
    for e, cp, cm in _diffT_terms(P):
        ne = tuple(-x for x in e)
        tot = tot + (cp * (V(T, *e) - V(T)) - cm * (V(T) - V(T, *ne)))
    return tot / 2.0 / P.Re / P.Sc / P.R * P.dt


def diffusion_scalar_adj(P, udTb, Tb):
    _lap_adj(Tb, _diffT_terms(P), udTb / 2.0 / P.Re / P.Sc / P.R * P.dt)


def face_masks(c1):
    """SET_IMMERSED_BOUNDARY's face averages (nse_dominik.f:1036-1070); the
    last face of each direction copies its cell (no periodic wrap)"""
    c2 = c1.copy()
    c2[:-1] = 0.5 * (c1[:-1] + c1[1:])
    c3 = c1.copy()
    c3[:, :-1] = 0.5 * (c1[:, :-1] + c1[:, 1:])
    c4 = c1.copy()
    c4[:, :, :-1] = 0.5 * (c1[:, :, :-1] + c1[:, :, 1:])
    return c2, c3, c4


def face_masks_adj(c2b, c3b, c4b):
    c1b = np.zeros_like(c2b)
    for cb, ax in ((c2b, 0), (c3b, 1), (c4b, 2)):
        sl = [slice(None)] * 3
        lo = list(sl)
        lo[ax] = slice(0, -1)
        hi = list(sl)
        hi[ax] = slice(1, None)
        last = list(sl)
        last[ax] = slice(-1, None)
        c1b[tuple(lo)] += 0.5 * cb[tuple(lo)]
        c1b[tuple(hi)] += 0.5 * cb[tuple(lo)]
        c1b[tuple(last)] += cb[tuple(last)]
    return c1b


# ---------------------------------------------------------- line solves --
def _lines(X, axis):
    n = X.shape[axis]
    Xl = np.moveaxis(X, axis, -1)
    return Xl.reshape(-1, n), Xl.shape


def _unlines(Y, shape, axis):
    return np.moveaxis(Y.reshape(shape), -1, axis)


def _dense(lo, di, up, periodic):
    b, n = di.shape
    M = np.zeros((b, n, n))
    idx = np.arange(n)
    M[:, idx, idx] = di
    M[:, idx[1:], idx[:-1]] = lo[:, 1:]
    M[:, idx[:-1], idx[1:]] = up[:, :-1]
    if periodic:
        M[:, 0, n - 1] += lo[:, 0]
        M[:, n - 1, 0] += up[:, n - 1]
    return M


def _rows(P, kind, axis, alpha):
    """row coefficients (lo, di, up) of the interior rows along `axis` for the
    line family `kind`: 'u' (implicit_uy, u/w in y), 'v' (implicit_vy),
    'T' (implicit_Ty / implicit_Tx), 'c' (implicit_solver, velocity in x/z).
    alpha has the shape of the interior block; returns arrays of that shape."""
    g = P.g
    d, d12, G = {0: (g.dx, g.dx12, gx), 1: (g.dy, g.dy12, gy), 2: (g.dz, g.dz12, gz)}[axis]
    if kind == "T":
        beta = P.dt / P.Re / P.Sc / 2.0
        n = len(d) - 2
        hp = _harm(d, P.L, 1)
        hm = _harm(d, P.L, -1)
        sh = [1, 1, 1]
        sh[axis] = n
        hp = hp.reshape(sh)
        hm = hm.reshape(sh)
        lo = -beta / alpha * hm / G(d12, -1) / G(d) / P.R
        di = 1.0 + beta / alpha * (hp / G(d12) / G(d) + hm / G(d12, -1) / G(d)) / P.R
        up = -beta / alpha * hp / G(d12) / G(d) / P.R
        return lo, di, up
    beta = P.dt / P.Re / 2.0
    if kind == "u":
        lo = -beta / alpha / G(d12, -1) / G(d)
        di = 1.0 + beta / alpha * (1.0 / G(d12) + 1.0 / G(d12, -1)) / G(d)
        up = -beta / alpha / G(d12) / G(d)
    else:  # 'v' and 'c' share the form of implicit_vy / implicit_solver
        lo = -beta / alpha / G(d) / G(d12)
        di = 1.0 + beta / alpha * (1.0 / G(d, 1) + 1.0 / G(d)) / G(d12)
        up = -beta / alpha / G(d, 1) / G(d12)
    return lo, di, up


class LinePass:
    """One ADI pass x = A(c)^-1 r over all lines of a direction.

    kind 'u' / 'T' along y: ghost rows x0 + x1 = ft, x_n + x_n+1 = fb folded
    into the interior system; 'v' along y: rows 1..ny-1 with x0 = x_ny = 0;
    periodic ('c', or 'T' along x/z): x0 = x_n, x_n+1 = x_1.
    vrows: the v component, whose lines and rows are j = 1..ny-1 only."""

    def __init__(self, P, kind, axis, c, ft=0.0, fb=0.0, vrows=False):
        self.P, self.kind, self.axis = P, kind, axis
        self.ft, self.fb = ft, fb
        self.vrows = vrows          # v component: only rows/lines j = 1..ny-1
        cc = c[:, :-1] if vrows else c
        self.alpha = P.dt * P.eta * cc + 1.0
        lo, di, up = _rows(P, kind, axis, self.alpha) if not vrows else \
            _rows_v(P, kind, axis, self.alpha)
        self.lo3, self.up3 = lo, up
        L, self.shape = _lines(np.broadcast_to(lo, self.alpha.shape), axis)
        D, _ = _lines(np.broadcast_to(di, self.alpha.shape), axis)
        U, _ = _lines(np.broadcast_to(up, self.alpha.shape), axis)
        self.periodic = axis != 1
        D = D.copy()
        self.f = np.zeros_like(D)
        if axis == 1 and kind in ("u", "T"):
            D[:, 0] -= L[:, 0]
            D[:, -1] -= U[:, -1]
            self.f[:, 0] = L[:, 0] * ft
            self.f[:, -1] = U[:, -1] * fb
        self.M = _dense(L, D, U, self.periodic)

    def _sub(self, X):
        return X[:, :-1] if self.vrows else X

    def solve(self, R):
        r, _ = _lines(self._sub(R), self.axis)
        x = np.linalg.solve(self.M, (r - self.f)[..., None])[..., 0]
        out = R.copy()
        if self.vrows:
            out[:, :-1] = _unlines(x, self.shape, self.axis)
            if self.axis == 1:
                out[:, -1] = 0.0   # implicit_vy writes x(ny) = fb = 0
        else:
            out[...] = _unlines(x, self.shape, self.axis)
        return out

    def adjoint(self, Xb, R, X):
        """returns (R_bar, c_bar) for the pass R -> X given X_bar"""
        xb, _ = _lines(self._sub(Xb), self.axis)
        y = np.linalg.solve(np.transpose(self.M, (0, 2, 1)), xb[..., None])[..., 0]
        yb = _unlines(y, self.shape, self.axis)
        cb_sub = yb * self.P.dt * self.P.eta / self.alpha * (self._sub(R) - self._sub(X))
        Rb = np.zeros_like(Xb)
        cb = np.zeros_like(Xb)
        if self.vrows:
            Rb[:, :-1] = yb
            cb[:, :-1] = cb_sub
            if self.axis != 1:
                Rb[:, -1] = Xb[:, -1]   # row ny passes through the x and z passes
        else:
            Rb[...] = yb
            cb[...] = cb_sub
        return Rb, cb


def _rows_v(P, kind, axis, alpha):
    """rows of the v component: implicit_vy along y, implicit_solver along x/z,
    on the block j = 1..ny-1"""
    g = P.g
    beta = P.dt / P.Re / 2.0
    if axis == 1:
        d, d12 = g.dy, g.dy12
        ny = g.ny
        dd = d[1:ny][None, :, None]
        dp = d[2:ny + 1][None, :, None]
        dd12 = d12[1:ny][None, :, None]
        lo = -beta / alpha / dd / dd12
        di = 1.0 + beta / alpha * (1.0 / dp + 1.0 / dd) / dd12
        up = -beta / alpha / dp / dd12
        return lo, di, up
    return _rows(P, "c", axis, alpha)


# ------------------------------------------------------------------ MKP --
def _spn_matrix(P):
    """SPN's Neumann-folded real matrices per (kx, kz) (mkp.f:239-254), dense
    (H, nz, ny, ny); the (0,0) entry is unused (SP0B)"""
    ny, H, nz = P.ny, P.nx // 2 + 1, P.nz
    AC = P.AC
    lo = np.broadcast_to(AC[:, 0], (H, nz, ny)).copy()
    up = np.broadcast_to(AC[:, 2], (H, nz, ny)).copy()
    di = AC[None, None, :, 1] - P.KXZ[:H, :nz][:, :, None]
    di = di.copy()
    di[:, :, 0] += lo[:, :, 0]
    di[:, :, -1] += up[:, :, -1]
    M = _dense(lo.reshape(-1, ny), di.reshape(-1, ny), up.reshape(-1, ny), False)
    return M.reshape(H, nz, ny, ny)


def _sp0b(P, D):
    """SP0B mkp.f:263-290 on D[1..ny] (complex), returns phi[1..ny]"""
    ny = P.ny
    AC = P.AC
    ph = np.zeros(ny + 2, dtype=complex)
    for J in range(1, ny):
        ph[J + 1] = (D[J - 1] - AC[J - 1, 0] * ph[J - 1] - AC[J - 1, 1] * ph[J]) / AC[J - 1, 2]
    return ph[1:ny + 1]


def _sp0b_adj(P, phb):
    ny = P.ny
    AC = P.AC
    pb = np.zeros(ny + 2, dtype=complex)
    pb[1:ny + 1] = phb
    Db = np.zeros(ny, dtype=complex)
    for J in range(ny - 1, 0, -1):
        t = pb[J + 1] / AC[J - 1, 2]
        Db[J - 1] += t
        pb[J - 1] -= AC[J - 1, 0] * t
        pb[J] -= AC[J - 1, 1] * t
        pb[J + 1] = 0.0
    return Db


def _p2s(samples):
    """P2S: samples (nx, ny, nz) -> half spectrum (H, ny, nz) / (nx nz)"""
    nx, nz = samples.shape[0], samples.shape[2]
    return np.fft.rfft2(samples, axes=(2, 0)) / (nx * nz)


def _s2p(spec, nx, nz):
    """S2P: unnormalised c2r of the half spectrum -> samples (nx, ny, nz)"""
    return np.fft.irfft2(spec, s=(nz, nx), axes=(2, 0)) * (nx * nz)


def _spectral(P, Y, transpose):
    """SPN + SP0B on a half spectrum (H, ny, nz), or their transposes"""
    M = _spn_matrix(P)
    M[0, 0] = np.eye(P.ny)   # the mean mode is SP0B's
    if transpose:
        M = np.swapaxes(M, -1, -2)
    H, ny, nz = Y.shape
    Yl = np.moveaxis(Y, 1, -1)  # (H, nz, ny)
    Xr = np.linalg.solve(M, Yl.real[..., None])[..., 0]
    Xi = np.linalg.solve(M, Yl.imag[..., None])[..., 0]
    X = Xr + 1j * Xi
    X[0, 0] = _sp0b_adj(P, Yl[0, 0]) if transpose else _sp0b(P, Yl[0, 0])
    return np.moveaxis(X, -1, 1)


def poisson(P, rhs):
    """interior right-hand side -> padded phi (periodic sample fill of
    mkp.f:101-121, P2S, SPN, SP0B, S2P, PHIBC)"""
    nx, ny, nz = P.nx, P.ny, P.nz
    samp = np.roll(np.roll(rhs, 1, axis=0), 1, axis=2)   # sample 0 = cell n
    s = _s2p(_spectral(P, _p2s(samp), False), nx, nz)
    phi = padded(nx, ny, nz)
    ii = np.arange(nx + 2) % nx
    jj = np.clip(np.arange(ny + 2), 1, ny) - 1
    kk = np.arange(nz + 2) % nz
    phi[...] = s[np.ix_(ii, jj, kk)]
    return phi


def poisson_adj(P, phib):
    nx, ny, nz = P.nx, P.ny, P.nz
    sb = np.zeros((nx, ny, nz))
    ii = np.arange(nx + 2) % nx
    jj = np.clip(np.arange(ny + 2), 1, ny) - 1
    kk = np.arange(nz + 2) % nz
    np.add.at(sb, np.ix_(ii, jj, kk), phib)
    rb_s = _s2p(_spectral(P, _p2s(sb), True), nx, nz)
    return np.roll(np.roll(rb_s, -1, axis=0), -1, axis=2)


def mkp(P, us, vs, ws):
    """MKP on u* (padded, after SET_BC): returns interior u, v, w, u_ta, v_ta, w_ta"""
    g, dt = P.g, P.dt
    rhs = ((V(us) - V(us, -1)) / gx(g.dx) + (V(vs) - V(vs, 0, -1)) / gy(g.dy) +
           (V(ws) - V(ws, 0, 0, -1)) / gz(g.dz)) / dt
    phi = poisson(P, rhs)
    Gx = (V(phi, 1) - V(phi)) / gx(g.dx12)
    Gy = (V(phi, 0, 1) - V(phi)) / gy(g.dy12)
    Gz = (V(phi, 0, 0, 1) - V(phi)) / gz(g.dz12)
    return (V(us) - dt * Gx, V(vs) - dt * Gy, V(ws) - dt * Gz, dt * Gx, dt * Gy, dt * Gz)


def mkp_adj(P, ub, vb, wb, utab, vtab, wtab):
    """adjoint of mkp: interior adjoints of the outputs -> padded adjoints of
    u*, v*, w* (before the transposed SET_BC)"""
    g, dt = P.g, P.dt
    nx, ny, nz = P.nx, P.ny, P.nz
    usb, vsb, wsb = embed(ub), embed(vb), embed(wb)
    phib = padded(nx, ny, nz)
    for Gb, e, d12 in ((dt * (utab - ub), (1, 0, 0), gx(g.dx12)),
                       (dt * (vtab - vb), (0, 1, 0), gy(g.dy12)),
                       (dt * (wtab - wb), (0, 0, 1), gz(g.dz12))):
        acc(phib, *e, Gb / d12)
        acc(phib, 0, 0, 0, -Gb / d12)
    rb = poisson_adj(P, phib) / dt
    acc(usb, 0, 0, 0, rb / gx(g.dx))
    acc(usb, -1, 0, 0, -rb / gx(g.dx))
    acc(vsb, 0, 0, 0, rb / gy(g.dy))
    acc(vsb, 0, -1, 0, -rb / gy(g.dy))
    acc(wsb, 0, 0, 0, rb / gz(g.dz))
    acc(wsb, 0, 0, -1, -rb / gz(g.dz))
    return usb, vsb, wsb


# ----------------------------------------------------------------- step --
STATE = ("u", "v", "w", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre", "T_pre")


def step(P, st, c1, l):
    """One time step.  st: dict of interior arrays (nx, ny, nz) of STATE;
    c1: mask (nx, ny, nz); l: step counter (1 = Euler start).
    Returns (new state, record)."""
    nx, ny, nz = P.nx, P.ny, P.nz
    dt, eta = P.dt, P.eta
    u, v, w, T = (embed(st[k]) for k in ("u", "v", "w", "T"))
    set_bc(u, "u"); set_bc(v, "v"); set_bc(w, "u"); set_bc(T, "T", P.tbot, P.ttop)
    c2, c3, c4 = face_masks(c1)
    uv, vv, wv = convect(P, u, v, w)
    uvT = convect_scalar(P, u, v, w, T)
    a1, a2 = (1.0, 0.0) if l == 1 else (1.5, -0.5)
    ua = a1 * uv + a2 * st["u_pre"] + conduction(P, u, 0) + eta * c2 * st["u_ta"] * dt
    va = a1 * vv + a2 * st["v_pre"] + conduction(P, v, 1) + eta * c3 * st["v_ta"] * dt
    wa = a1 * wv + a2 * st["w_pre"] + conduction(P, w, 2) + eta * c4 * st["w_ta"] * dt
    uT = a1 * uvT + a2 * st["T_pre"] + diffusion_scalar(P, T)
    rec = dict(start={k: st[k].copy() for k in STATE}, l=l)
    ua0 = (V(u) + ua) / (1.0 + eta * c2 * dt)
    va0 = (V(v) + va) / (1.0 + eta * c3 * dt)
    wa0 = (V(w) + wa) / (1.0 + eta * c4 * dt)
    uT0 = (V(T) + uT + eta * c1 * dt * P.tsolid) / (1.0 + eta * c1 * dt)
    out = {}
    for name, x0, c, vrows in (("u", ua0, c2, False), ("v", va0, c3, True), ("w", wa0, c4, False)):
        passes = [LinePass(P, "v" if vrows else "u", 1, c, vrows=vrows),
                  LinePass(P, "c", 2, c, vrows=vrows), LinePass(P, "c", 0, c, vrows=vrows)]
        xs = [x0]
        for ps in passes:
            xs.append(ps.solve(xs[-1]))
        rec[name] = (passes, xs)
        out[name] = xs[-1]
    passes = [LinePass(P, "T", 1, c1, 2.0 * P.tbot, 2.0 * P.ttop), LinePass(P, "T", 0, c1),
              LinePass(P, "T", 2, c1)]
    xs = [uT0]
    for ps in passes:
        xs.append(ps.solve(xs[-1]))
    rec["T"] = (passes, xs)
    us, vs, ws = embed(out["u"]), embed(out["v"]), embed(out["w"])
    set_bc(us, "u"); set_bc(vs, "v"); set_bc(ws, "u")
    un, vn, wn, utn, vtn, wtn = mkp(P, us, vs, ws)
    new = dict(u=un, v=vn, w=wn, T=xs[-1], u_ta=utn, v_ta=vtn, w_ta=wtn, u_pre=uv, v_pre=vv,
               w_pre=wv, T_pre=uvT)
    rec["c"] = (c2, c3, c4)
    return new, rec


def adjoint_step(P, rec, bar, c1, cbar):
    """Reverse of one step.  bar: dict of interior adjoints of the state after
    the step (consumed); cbar: dict with 'c1', 'c2', 'c3', 'c4' accumulators.
    Returns the adjoint of the state at the start of the step."""
    nx, ny, nz = P.nx, P.ny, P.nz
    dt, eta = P.dt, P.eta
    st = rec["start"]
    l = rec["l"]
    c2, c3, c4 = rec["c"]
    # MKP
    usb, vsb, wsb = mkp_adj(P, bar["u"], bar["v"], bar["w"], bar["u_ta"], bar["v_ta"],
                            bar["w_ta"])
    set_bc_adj(usb, "u"); set_bc_adj(vsb, "v"); set_bc_adj(wsb, "u")
    # line passes in reverse
    xb = {"u": V(usb).copy(), "v": V(vsb).copy(), "w": V(wsb).copy(), "T": bar["T"].copy()}
    x0b = {}
    for name, ckey in (("u", "c2"), ("v", "c3"), ("w", "c4"), ("T", "c1")):
        passes, xs = rec[name]
        b = xb[name]
        for p in range(len(passes) - 1, -1, -1):
            b, cb = passes[p].adjoint(b, xs[p], xs[p + 1])
            cbar[ckey] += cb
        x0b[name] = b
    # penalised updates
    u, v, w, T = (embed(st[k]) for k in ("u", "v", "w", "T"))
    set_bc(u, "u"); set_bc(v, "v"); set_bc(w, "u"); set_bc(T, "T", P.tbot, P.ttop)
    out = {k: padded(nx, ny, nz) for k in ("u", "v", "w", "T")}
    ab = {}
    for name, c, ckey in (("u", c2, "c2"), ("v", c3, "c3"), ("w", c4, "c4")):
        den = 1.0 + eta * c * dt
        x0 = rec[name][1][0]
        ab[name] = x0b[name] / den
        acc(out[name], 0, 0, 0, x0b[name] / den)
        cbar[ckey] += -x0b[name] * x0 * eta * dt / den
    den = 1.0 + eta * c1 * dt
    tb = x0b["T"] / den
    acc(out["T"], 0, 0, 0, tb)
    cbar["c1"] += x0b["T"] * eta * dt * (P.tsolid - rec["T"][1][0]) / den
    # AB2, immersed boundary
    a1, a2 = (1.0, 0.0) if l == 1 else (1.5, -0.5)
    new = {}
    uvb = {}
    for name, c, ckey, ta in (("u", c2, "c2", "u_ta"), ("v", c3, "c3", "v_ta"),
                              ("w", c4, "c4", "w_ta")):
        uvb[name] = a1 * ab[name] + bar[name + "_pre"]
        new[name + "_pre"] = a2 * ab[name]
        new[ta] = eta * c * dt * ab[name]
        cbar[ckey] += eta * dt * st[ta] * ab[name]
    uvTb = a1 * tb + bar["T_pre"]
    new["T_pre"] = a2 * tb
    # conduction, scalar diffusion, convection
    for comp, name in enumerate(("u", "v", "w")):
        conduction_adj(P, ab[name], comp, out[name])
    diffusion_scalar_adj(P, tb, out["T"])
    convect_adj(P, u, v, w, uvb["u"], uvb["v"], uvb["w"], out["u"], out["v"], out["w"])
    convect_scalar_adj(P, u, v, w, T, uvTb, out["u"], out["v"], out["w"], out["T"])
    set_bc_adj(out["u"], "u"); set_bc_adj(out["v"], "v"); set_bc_adj(out["w"], "u")
    set_bc_adj(out["T"], "T")
    for k in ("u", "v", "w", "T"):
        new[k] = V(out[k]).copy()
    return new


def wall_flux_weights(P):
    """d J_n / d T(i,1,k) for J_n = area-weighted mean over the y = y0 wall of
    thc (T(i,1,k) - T(i,0,k)) / dy12(0) with the wall ghost T0 = 2 Tb - T1"""
    g = P.g
    a = (g.dx[1:P.nx + 1][:, None] * g.dz[1:P.nz + 1][None, :]) / (g.xl * g.zl)
    return 2.0 * P.L * a / g.dy12[0]


def wall_flux(P, T):
    """the objective's per-step term from the interior T (nx, ny, nz)"""
    g = P.g
    a = (g.dx[1:P.nx + 1][:, None] * g.dz[1:P.nz + 1][None, :]) / (g.xl * g.zl)
    return float(np.sum(a * P.L * (2.0 * T[:, 0, :] - 2.0 * P.tbot) / g.dy12[0]))


def gradient(P, st0, c1, nsteps, avg_from, extra=None):
    """J = mean over steps avg_from..nsteps of the wall flux, plus
    sum_k <extra[k], state_N[k]> for an optional dict of interior weights.
    Returns (J, dJ/dc1, dJ/d state_0)."""
    recs = []
    st = {k: v.copy() for k, v in st0.items()}
    J = 0.0
    navg = nsteps - avg_from + 1
    for n in range(1, nsteps + 1):
        st, rec = step(P, st, c1, n)
        recs.append(rec)
        if n >= avg_from:
            J += wall_flux(P, st["T"]) / navg
    if extra:
        J += sum(float(np.sum(extra[k] * st[k])) for k in extra)
    shape = c1.shape
    bar = {k: np.zeros(shape) for k in STATE}
    if extra:
        for k in extra:
            bar[k] = bar[k] + extra[k]
    cbar = {k: np.zeros(shape) for k in ("c1", "c2", "c3", "c4")}
    wts = wall_flux_weights(P)
    for n in range(nsteps, 0, -1):
        if n >= avg_from:
            bar["T"][:, 0, :] += wts / navg
        bar = adjoint_step(P, recs[n - 1], bar, c1, cbar)
    g1 = cbar["c1"] + face_masks_adj(cbar["c2"], cbar["c3"], cbar["c4"])
    return J, g1, bar


# ------------------------------------------------- restated adjoint.f --
def set_adj_convect(u, v, w, u_f, v_f, w_f, g, dt):
    """set_adj_convect adjoint.f:1-125 as written (including the v(i,j,k-1)
    of :45 and w_final(i,j,k+1)+w_final(i,j+1,k-1) of :79); interior outputs"""
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    uc = V(u)
    u1 = (-((V(u_f) + V(u_f, 1)) * (uc + V(u, 1)) - (V(u_f) + V(u_f, -1)) * (uc + V(u, -1))) / gx(dx12)
          - V(u_f) * (V(u, -1) - V(u, 1)) / gx(dx12) * 2.0)
    u2 = (-((V(v_f, 1) * gx(dx, 1) + V(v_f) * gx(dx)) * (V(u, 0, 1) + uc)
            - (V(v_f, 1, -1) * gx(dx, 1) + V(v_f, 0, -1) * gx(dx)) * (uc + V(u, 0, -1))) / gx(dx12) / gy(dy)
          - ((V(v_f, 1) + V(v_f, 1, -1)) * gx(dx, 1) + (V(v_f) + V(v_f, 0, -1)) * gx(dx)) / gx(dx12)
          * (-V(v, 1) - V(v, 1, -1) + V(v) + V(v, 0, -1)) / gx(dx12) / 2.0)
    u3 = (-((V(w_f, 1) * gx(dx, 1) + V(w_f) * gx(dx)) * (V(u, 0, 0, 1) + uc)
            - (V(w_f, 1, 0, -1) * gx(dx, 1) + V(w_f, 0, 0, -1) * gx(dx)) * (uc + V(u, 0, 0, -1))) / gx(dx12) / gz(dz)
          - ((V(w_f, 1) + V(w_f, 1, 0, -1)) * gx(dx, 1) + (V(w_f) + V(w_f, 0, 0, -1)) * gx(dx)) / gx(dx12)
          * (-V(w, 1) - V(w, 1, 0, -1) + V(w) + V(v, 0, 0, -1)) / gx(dx12) / 2.0)
    u_v = 0.25 * (-u1 - u2 - u3) * dt + 1.0 * dt
    vc = V(v)
    v1 = (((V(u_f, 0, 1) * gy(dy, 1) + V(u_f) * gy(dy)) * (V(v, 1) + vc)
           - (V(u_f, -1, 1) * gy(dy, 1) + V(u_f, -1) * gy(dy)) * (vc + V(v, -1))) / gy(dy12) / gx(dx)
          - ((V(u_f, 0, 1) + V(u_f, -1, 1)) * gy(dy, 1) + (V(u_f) + V(u_f, -1)) * gy(dy)) / gy(dy12)
          * (-V(u, 0, 1) - V(u, -1, 1) + uc + V(u, -1)) / gy(dy12) / 2.0)
    v2 = (((V(v_f) + V(v_f, 0, 1)) * (vc + V(v, 0, 1)) - (V(v_f) + V(v_f, 0, -1)) * (vc + V(v, 0, -1))) / gy(dy12)
          - V(v_f) * (V(v, -1) - V(v, 1)) * 2.0 / gy(dy12))
    v3 = (((V(w_f, 0, 1) * gy(dy, 1) + V(w_f) * gy(dy)) * (V(v, 0, 0, 1) + vc)
           - (V(w_f, 0, 1, -1) * gy(dy, 1) + V(w_f, 0, 0, -1) * gy(dy)) * (vc + V(v, 0, 0, -1))) / gy(dy12) / gz(dz)
          - ((V(w_f, 0, 0, 1) + V(w_f, 0, 1, -1)) * gy(dy, 1) + (V(w_f) + V(w_f, 0, 0, -1)) * gy(dy)) / gy(dy12)
          * (-V(w, 0, 1) - V(w, 0, 1, -1) + V(w) + V(w, 0, 0, -1)) / gy(dy12) / 2.0)
    v_v = 0.25 * (-v1 - v2 - v3) * dt
    wc = V(w)
    w1 = (((V(u_f, 0, 0, 1) * gz(dz, 1) + V(u_f) * gz(dz)) * (V(w, 1) + wc)
           - (V(u_f, -1, 0, 1) * gz(dz, 1) + V(u_f, -1) * gz(dz)) * (wc + V(w, -1))) / gz(dz12) / gx(dx)
          - ((V(u_f, 0, 0, 1) + V(u_f, -1, 0, 1)) * gz(dz, 1) + (V(u_f) + V(u_f, -1)) * gz(dz)) / gz(dz12)
          * (-V(u, 0, 0, 1) - V(u, -1, 0, 1) + uc + V(u, -1)) / gz(dz12) * 2.0)
    w2 = (((V(v_f, 0, 0, 1) * gz(dz, 1) + V(v_f) * gz(dz)) * (V(w, 0, 1) + wc)
           - (V(v_f, 0, -1, 1) * gz(dz, 1) + V(v_f, 0, -1) * gz(dz)) * (wc + V(w, 0, -1))) / gz(dz12) / gy(dy)
          - ((V(v_f, 0, 0, 1) + V(v_f, 0, -1, 1)) * gz(dz, 1) + (V(v_f) + V(v_f, 0, -1)) * gz(dz)) / gz(dz12)
          * (-V(v, 0, 0, 1) - V(v, 0, -1, 1) + vc + V(v, 0, -1)) / gz(dz12) * 2.0)
    w3 = (((V(w_f) + V(w_f, 0, 0, 1)) * (wc + V(w, 0, 0, 1)) - (V(w_f) + V(w_f, 0, 0, -1)) * (wc + V(w, 0, 0, -1))) / gz(dz12)
          - V(w_f) * (V(w, 0, 0, -1) - V(w, 0, 0, 1)) * 2.0 / gz(dz12))
    w_v = 0.25 * (-w1 - w2 - w3) * dt
    return u_v, v_v, w_v


def set_adj_convection_for_scalar(u_f, v_f, w_f, T, rhoCp, g, dt):
    """set_adj_convection_for_scalar adjoint.f:128-181 as written (u, v, w,
    Re are arguments the routine never reads); interior u_vT"""
    dx, dy, dz, dx12, dy12, dz12 = g.dx, g.dy, g.dz, g.dx12, g.dy12, g.dz12
    R = rhoCp
    uT = (-((V(R, -1) * V(T, -1) * gx(dx) + V(R) * V(T) * gx(dx, -1)) * V(u_f, -1)) / 2.0 / gx(dx12, -1)
          + ((V(R) * V(T) * gx(dx, 1) + V(R, 1) * V(T, 1) * gx(dx)) * V(u_f)) / 2.0 / gx(dx12)) / gx(dx)
    vT = (-((V(R, 0, -1) * V(T, 0, -1) * gy(dy) + V(R) * V(T) * gy(dy, -1)) * V(v_f, 0, -1)) / 2.0 / gy(dy12, -1)
          + ((V(R) * V(T) * gy(dy, 1) + V(R, 0, 1) * V(T, 0, 1) * gy(dy)) * V(v_f)) / 2.0 / gy(dy12)) / gy(dy)
    wT = (-((V(R, 0, 0, -1) * V(T, 0, 0, -1) * gz(dz) + V(R) * V(T) * gz(dz, -1)) * V(w_f, 0, 0, -1)) / 2.0 / gz(dz12, -1)
          + ((V(R) * V(T) * gz(dz, 1) + V(R, 0, 0, 1) * V(T, 0, 0, 1) * gz(dz)) * V(w_f)) / 2.0 / gz(dz12)) / gz(dz)
    return (uT + vT + wT) * dt / V(R) + 1.0 * dt


def set_adj_ns_scalar(T, T_final, g, dt):
    """set_adj_NS_scalar adjoint.f:185-211.  The reference reads T_final from
    an uninitialised local array (:190, :201-206); it is an argument here."""
    u_s = dt * V(T_final) * (V(T, 1) - V(T, -1)) / gx(g.dx12) / 2
    v_s = dt * V(T_final) * (V(T, 0, 1) - V(T, 0, -1)) / gy(g.dy12) / 2
    w_s = dt * V(T_final) * (V(T, 0, 0, 1) - V(T, 0, 0, -1)) / gz(g.dz12) / 2
    return u_s, v_s, w_s
