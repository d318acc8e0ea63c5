// k_adjoint.cu -- transposed kernels of the discrete adjoint of one time step
// (the step of nse_dominik.f:290-446 differentiated with respect to its
// state and to the penalisation mask), and the adjoint.f drop-ins.
//
// Every kernel here applies the transpose of one forward operation, in the
// gather form: a thread owns one input cell and sums the partial derivatives
// of every output cell that reads it, weighted by that output's adjoint, so
// nothing is scattered and no atomics are needed.  Output adjoints are read
// only where the output cell is interior (1..n in each direction); a padded
// cell that the forward SET_BC fills from an interior cell hands its adjoint
// back to that cell (the "preimage" sums of k_adj_explicit / k_adj_div).
//
// The forward formulas differentiated (reference file:line):
//   SET_CONVECT nse_dominik.f:757-831, SET_CONVECTION_FOR_SCALAR :834-884,
//   SET_CONDUCTION :888-945, SET_DIFFUSION_FOR_SCALAR :950-1004,
//   SET_IMMERSED_BOUNDARY :1011-1129, SET_EXPLICIT :1132-1341, the penalised
//   updates :387-396 and :1358-1433, implicit_uy/vy/Ty :1505-1870,
//   implicit_solver/cyclic periodic_implicit.f:1-93, MKP mkp.f:9-220.
#include "common.cuh"
#include "k_adjoint.cuh"

namespace nse {

namespace {

struct Pos {
  int c[3];
};

__device__ __forceinline__ bool inside(const Dims& D, const Pos& p) {
  return p.c[0] >= 1 && p.c[0] <= D.nx && p.c[1] >= 1 && p.c[1] <= D.ny && p.c[2] >= 1 &&
         p.c[2] <= D.nz;
}
__device__ __forceinline__ long at(const Dims& D, const Pos& p) {
  return D.P(p.c[0], p.c[1], p.c[2]);
}
__device__ __forceinline__ Pos sh(Pos p, int axis, int s) {
  p.c[axis] += s;
  return p;
}
__device__ __forceinline__ Pos sh2(Pos p, int a1, int s1, int a2, int s2) {
  p.c[a1] += s1;
  p.c[a2] += s2;
  return p;
}

// ----------------------------------------------- explicit-term transposes --
struct XArgs {
  Dims D;
  AdjGrid g;
  const double* vel[3];  // u, v, w at the start of the step, SET_BC applied
  const double* T;
  const double* A[3];    // adjoint of u_d = u_a - penalty (= a_bar), interior
  const double* B[3];    // adjoint of u_v (AB2 weight + next history), interior
  const double* At;      // adjoint of u_dT
  const double* Bt;      // adjoint of u_vT
  double dt, Re, Sc, R, L;
  double cfac, dfac, qfac;  // dt/Re/2, dt/(2 Re Sc R), -dt/R
};

__device__ __forceinline__ double val(const XArgs& a, const double* f, const Pos& p) {
  return f[at(a.D, p)];
}
// momentum convection output of component AC at o: -0.25 dt * adjoint
__device__ __forceinline__ double qmom(const XArgs& a, int AC, const Pos& o) {
  return -0.25 * a.dt * a.B[AC][at(a.D, o)];
}

// square term ((f + f+)^2 - (f + f-)^2) / d12 of output AC; adjoint w.r.t. f = vel[AC] at q
template <int AC>
__device__ double sq_f(const XArgs& a, const Pos& q) {
  const double* f = a.vel[AC];
  const double* d12 = a.g.d12[AC];
  double s = 0.0;
  if (inside(a.D, q)) {
    const double m = qmom(a, AC, q) * a.g.r12[AC][q.c[AC]];
    s += 2.0 * m * ((val(a, f, q) + val(a, f, sh(q, AC, 1))) - (val(a, f, q) + val(a, f, sh(q, AC, -1))));
  }
  Pos o = sh(q, AC, -1);
  if (inside(a.D, o)) s += 2.0 * qmom(a, AC, o) * a.g.r12[AC][o.c[AC]] * (val(a, f, o) + val(a, f, q));
  o = sh(q, AC, 1);
  if (inside(a.D, o)) s -= 2.0 * qmom(a, AC, o) * a.g.r12[AC][o.c[AC]] * (val(a, f, o) + val(a, f, q));
  return s;
}

// cross term of output AC along AF: scale (Gp (f(o+eF) + f(o)) - Gm (f(o) + f(o-eF)))
// with f = vel[AC], g = vel[AF], scale = 1/(d12_AC(o) d_AF(o)),
// Gp = g(o+eC) dC(o+1) + g(o) dC(o), Gm = g(o+eC-eF) dC(o+1) + g(o-eF) dC(o)
template <int AC, int AF>
__device__ __forceinline__ double cross_m(const XArgs& a, const Pos& o) {
  return qmom(a, AC, o) * a.g.r12[AC][o.c[AC]] * a.g.r[AF][o.c[AF]];
}
template <int AC, int AF>
__device__ __forceinline__ double cross_gp(const XArgs& a, const Pos& o) {
  const double* gg = a.vel[AF];
  const double* dC = a.g.d[AC];
  return val(a, gg, sh(o, AC, 1)) * dC[o.c[AC] + 1] + val(a, gg, o) * dC[o.c[AC]];
}
template <int AC, int AF>
__device__ __forceinline__ double cross_gm(const XArgs& a, const Pos& o) {
  const double* gg = a.vel[AF];
  const double* dC = a.g.d[AC];
  return val(a, gg, sh2(o, AC, 1, AF, -1)) * dC[o.c[AC] + 1] +
         val(a, gg, sh(o, AF, -1)) * dC[o.c[AC]];
}
// adjoint w.r.t. f = vel[AC] at q
template <int AC, int AF>
__device__ double cross_f(const XArgs& a, const Pos& q) {
  double s = 0.0;
  Pos o = sh(q, AF, -1);
  if (inside(a.D, o)) s += cross_m<AC, AF>(a, o) * cross_gp<AC, AF>(a, o);
  if (inside(a.D, q))
    s += cross_m<AC, AF>(a, q) * (cross_gp<AC, AF>(a, q) - cross_gm<AC, AF>(a, q));
  o = sh(q, AF, 1);
  if (inside(a.D, o)) s -= cross_m<AC, AF>(a, o) * cross_gm<AC, AF>(a, o);
  return s;
}
// adjoint w.r.t. g = vel[AF] at q
template <int AC, int AF>
__device__ double cross_g(const XArgs& a, const Pos& q) {
  const double* f = a.vel[AC];
  const double* dC = a.g.d[AC];
  double s = 0.0;
  Pos o = sh(q, AC, -1);  // q = o + eC: weight dC(o+1)
  if (inside(a.D, o))
    s += cross_m<AC, AF>(a, o) * dC[o.c[AC] + 1] * (val(a, f, sh(o, AF, 1)) + val(a, f, o));
  if (inside(a.D, q))  // q = o: weight dC(o)
    s += cross_m<AC, AF>(a, q) * dC[q.c[AC]] * (val(a, f, sh(q, AF, 1)) + val(a, f, q));
  o = sh2(q, AC, -1, AF, 1);  // q = o + eC - eF: weight dC(o+1)
  if (inside(a.D, o))
    s -= cross_m<AC, AF>(a, o) * dC[o.c[AC] + 1] * (val(a, f, o) + val(a, f, sh(o, AF, -1)));
  o = sh(q, AF, 1);  // q = o - eF: weight dC(o)
  if (inside(a.D, o))
    s -= cross_m<AC, AF>(a, o) * dC[o.c[AC]] * (val(a, f, o) + val(a, f, sh(o, AF, -1)));
  return s;
}

template <int X>
__device__ double conv_adj(const XArgs& a, const Pos& q) {
  constexpr int Y1 = (X + 1) % 3, Y2 = (X + 2) % 3;
  return sq_f<X>(a, q) + cross_f<X, Y1>(a, q) + cross_f<X, Y2>(a, q) + cross_g<Y1, X>(a, q) +
         cross_g<Y2, X>(a, q);
}

// SET_CONDUCTION second differences: along the component's own axis
// cp = 1/(d(o+1) d12(o)), cm = 1/(d(o) d12(o)); along the others
// cp = 1/(d12(o) d(o)), cm = 1/(d12(o-1) d(o))
__device__ __forceinline__ void lap_coef(const AdjGrid& g, int comp, int ax, int o, double& cp,
                                         double& cm) {
  const double* r = g.r[ax];
  const double* r12 = g.r12[ax];
  if (ax == comp) {
    cp = r[o + 1] * r12[o];
    cm = r[o] * r12[o];
  } else {
    cp = r12[o] * r[o];
    cm = r12[o - 1] * r[o];
  }
}

template <int C>
__device__ double cond_adj(const XArgs& a, const Pos& q) {
  const double* A = a.A[C];
  double s = 0.0;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    double cp, cm;
    if (inside(a.D, q)) {
      lap_coef(a.g, C, ax, q.c[ax], cp, cm);
      s -= (cp + cm) * val(a, A, q);
    }
    Pos o = sh(q, ax, -1);
    if (inside(a.D, o)) {
      lap_coef(a.g, C, ax, o.c[ax], cp, cm);
      s += cp * val(a, A, o);
    }
    o = sh(q, ax, 1);
    if (inside(a.D, o)) {
      lap_coef(a.g, C, ax, o.c[ax], cp, cm);
      s += cm * val(a, A, o);
    }
  }
  return a.cfac * s;
}

// with uniform conductivity the harmonic mean is L itself
__device__ __forceinline__ void diffT_coef(const AdjGrid& g, int ax, int o, double L, double& cp,
                                           double& cm) {
  const double* r = g.r[ax];
  const double* r12 = g.r12[ax];
  cp = L * r12[o] * r[o];
  cm = L * r12[o - 1] * r[o];
}

__device__ double diffT_adj(const XArgs& a, const Pos& q) {
  double s = 0.0;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    double cp, cm;
    if (inside(a.D, q)) {
      diffT_coef(a.g, ax, q.c[ax], a.L, cp, cm);
      s -= (cp + cm) * val(a, a.At, q);
    }
    Pos o = sh(q, ax, -1);
    if (inside(a.D, o)) {
      diffT_coef(a.g, ax, o.c[ax], a.L, cp, cm);
      s += cp * val(a, a.At, o);
    }
    o = sh(q, ax, 1);
    if (inside(a.D, o)) {
      diffT_coef(a.g, ax, o.c[ax], a.L, cp, cm);
      s += cm * val(a, a.At, o);
    }
  }
  return s * a.dfac;
}

// scalar convection: per axis a, with f = vel[a], d = d_a, d12 = d12_a,
//   term1(o) = -(R T(o-e) d(o) + R T(o) d(o-1)) f(o-e) m1(o),
//   m1(o) = qT(o) / (2 d12(o-1) d(o));
//   term2(o) = (R T(o) d(o+1) + R T(o+e) d(o)) f(o) m2(o),
//   m2(o) = qT(o) / (2 d12(o) d(o)),  qT = -dt/R * adjoint of u_vT
__device__ __forceinline__ double m1T(const XArgs& a, int ax, const Pos& o) {
  const double qT = a.qfac * val(a, a.Bt, o);
  return 0.5 * qT * a.g.r12[ax][o.c[ax] - 1] * a.g.r[ax][o.c[ax]];
}
__device__ __forceinline__ double m2T(const XArgs& a, int ax, const Pos& o) {
  const double qT = a.qfac * val(a, a.Bt, o);
  return 0.5 * qT * a.g.r12[ax][o.c[ax]] * a.g.r[ax][o.c[ax]];
}
// adjoint w.r.t. vel[AX] at q
template <int AX>
__device__ double cscal_vel_adj(const XArgs& a, const Pos& q) {
  const double* d = a.g.d[AX];
  const double R = a.R;
  double s = 0.0;
  Pos o = sh(q, AX, 1);
  if (inside(a.D, o))
    s -= m1T(a, AX, o) * (R * val(a, a.T, q) * d[o.c[AX]] + R * val(a, a.T, o) * d[q.c[AX]]);
  if (inside(a.D, q))
    s += m2T(a, AX, q) *
         (R * val(a, a.T, q) * d[q.c[AX] + 1] + R * val(a, a.T, sh(q, AX, 1)) * d[q.c[AX]]);
  return s;
}
// adjoint w.r.t. T at q
__device__ double cscal_T_adj(const XArgs& a, const Pos& q) {
  const double R = a.R;
  double s = 0.0;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    const double* d = a.g.d[ax];
    const double* f = a.vel[ax];
    Pos o = sh(q, ax, 1);
    if (inside(a.D, o)) s -= m1T(a, ax, o) * R * d[o.c[ax]] * val(a, f, q);
    if (inside(a.D, q)) {
      s -= m1T(a, ax, q) * R * d[q.c[ax] - 1] * val(a, f, sh(q, ax, -1));
      s += m2T(a, ax, q) * R * d[q.c[ax] + 1] * val(a, f, q);
    }
    o = sh(q, ax, -1);
    if (inside(a.D, o)) s += m2T(a, ax, o) * R * d[o.c[ax]] * val(a, f, o);
  }
  return s;
}

template <int F>
__device__ double raw_adj(const XArgs& a, const Pos& q) {
  if constexpr (F < 3) {
    double s = inside(a.D, q) ? val(a, a.A[F], q) : 0.0;
    return s + cond_adj<F>(a, q) + conv_adj<F>(a, q) + cscal_vel_adj<F>(a, q);
  } else {
    double s = inside(a.D, q) ? val(a, a.At, q) : 0.0;
    return s + diffT_adj(a, q) + cscal_T_adj(a, q);
  }
}

// padded cells whose SET_BC value is a copy of interior index p along an
// axis of length n: p itself, 0 (copy of n) and n+1 (copy of 1)
__device__ __forceinline__ int periodic_pre(int p, int n, int* q) {
  int m = 0;
  q[m++] = p;
  if (p == n) q[m++] = 0;
  if (p == 1) q[m++] = n + 1;
  return m;
}

// adjoint of the state field F (0 u, 1 v, 2 w, 3 T) at the start of the
// step, interior cells: the explicit terms transposed and SET_BC folded.
// A CTA covers an (x, y) tile of one plane, so the y neighbours every cell
// gathers are mostly the tile's own rows (L1 hits).
template <int F>
__global__ void k_adj_explicit(XArgs a, double* __restrict__ out) {
  const Dims& D = a.D;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx || j > D.ny) return;
  const long c = D.P(i, j, k);
  if (F == 1 && j == D.ny) {  // v(ny) is set to zero by SET_BC
    out[c] = 0.0;
    return;
  }
  int qi[3], qk[3], qj[3];
  double sj[3];
  const int ni = periodic_pre(i, D.nx, qi);
  const int nk = periodic_pre(k, D.nz, qk);
  int nj = 0;
  qj[nj] = j; sj[nj++] = 1.0;
  if (F != 1) {  // u, w, T: wall ghosts are minus the first interior row
    if (j == 1) { qj[nj] = 0; sj[nj++] = -1.0; }
    if (j == D.ny) { qj[nj] = D.ny + 1; sj[nj++] = -1.0; }
  }
  double s = 0.0;
  for (int b = 0; b < nj; ++b)
    for (int e = 0; e < nk; ++e)
      for (int t = 0; t < ni; ++t) {
        Pos q;
        q.c[0] = qi[t]; q.c[1] = qj[b]; q.c[2] = qk[e];
        s += sj[b] * raw_adj<F>(a, q);
      }
  out[c] = s;
}

// ------------------------------------------------- pointwise transposes --
// penalised updates, AB2 and immersed-boundary forcing (interior cells):
//   A[X]: adjoint of the penalised u_a (in) -> adjoint of the explicit u_a (out)
//   B[X] = a1 A[X] + adjoint of the new history u_pre
//   bar_pre[X] <- a2 A[X], bar_ta[X] <- eta c dt A[X]
//   cbar_X += -a0 u_a0 eta dt / den + eta dt u_ta A[X]
struct PArgs {
  Dims D;
  double* A[4];          // u, v, w, T
  double* B[4];
  double* bar_pre[4];
  double* bar_ta[3];
  const double* ta[3];   // u_ta, v_ta, w_ta at the start of the step
  const double* rin[4];  // penalised u_a, v_a, w_a, u_T (input of the y pass)
  const double* c1;
  double* cbar[4];       // c1, c2, c3, c4 (nx*ny*nz each)
  double eta, dt, tsolid, a1, a2;
};

__device__ __forceinline__ double face_mask(const Dims& D, const double* c1, int comp, int i,
                                            int j, int k) {
  const double cc = c1[D.C(i, j, k)];
  if (comp == 0) return i < D.nx ? (cc + c1[D.C(i + 1, j, k)]) * 0.5 : cc;
  if (comp == 1) return j < D.ny ? (cc + c1[D.C(i, j + 1, k)]) * 0.5 : cc;
  if (comp == 2) return k < D.nz ? (cc + c1[D.C(i, j, k + 1)]) * 0.5 : cc;
  return cc;
}

__global__ void k_adj_point(PArgs a) {
  const Dims& D = a.D;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx) return;
  const long c = D.P(i, j, k);
  const long m = D.C(i, j, k);
#pragma unroll
  for (int X = 0; X < 3; ++X) {
    const double cm = face_mask(D, a.c1, X, i, j, k);
    const double den = 1.0 + a.eta * cm * a.dt;
    const double a0 = a.A[X][c];
    const double ab = a0 / den;
    a.cbar[X + 1][m] += -a0 * a.rin[X][c] * a.eta * a.dt / den + a.eta * a.dt * a.ta[X][c] * ab;
    a.B[X][c] = a.a1 * ab + a.bar_pre[X][c];
    a.bar_pre[X][c] = a.a2 * ab;
    a.bar_ta[X][c] = a.eta * cm * a.dt * ab;
    a.A[X][c] = ab;
  }
  const double c1 = a.c1[m];
  const double den = 1.0 + a.eta * c1 * a.dt;
  const double t0 = a.A[3][c];
  const double tb = t0 / den;
  a.cbar[0][m] += t0 * a.eta * a.dt * (a.tsolid - a.rin[3][c]) / den;
  a.B[3][c] = a.a1 * tb + a.bar_pre[3][c];
  a.bar_pre[3][c] = a.a2 * tb;
  a.A[3][c] = tb;
}

// ------------------------------------- line transposes by diagonal scaling --
// Every line system of the step has rows A(j,j+-1) = -(beta/alpha_j) s(j,j+-1)/w_j
// with s symmetric (also through the wall folds, which change diagonals
// only, and the periodic corners, where the ghost spacing equals the
// opposite interior one): w_j = dy (u, w, T along y), dy12 (v along y),
// dx12 / dz12 (velocity along x / z), dx / dz (T along x / z).  So
// A = D^-1 (D + S) with D = diag(alpha_j w_j), A^T = D A D^-1 and
// A^-T = D A^-1 D^-1: the transposed solve is the step's own line solve
// between two diagonal scalings.  `out` = 0: xb /= alpha w (before the
// solve); 1: rbar = alpha w y, c_bar += rbar dt eta / alpha (r - x), and
// when the pass has a predecessor (next >= 0, its direction) the result is
// scaled at once for that pass's solve: xb = rbar / (alpha w_next).
struct SArgs {
  Dims D;
  AdjGrid g;
  double* xb;
  const double* rin;
  const double* xout;
  const double* c1;
  double* cbar;
  int dir, comp, out, next;
  double dte;  // dt * eta
};

// 1 / w of line direction `dir` for component `comp` at index idx
__device__ __forceinline__ double line_rw(const AdjGrid& g, int dir, int comp, int idx) {
  const bool wd = comp == 3 || (dir == 1 && comp != 1);
  return wd ? g.r[dir][idx] : g.r12[dir][idx];
}

__global__ void k_adj_line_scale(SArgs a) {
  const Dims& D = a.D;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx || (a.comp == 1 && j == D.ny)) return;
  const int ijk[3] = {i, j, k};
  const double rw = line_rw(a.g, a.dir, a.comp, ijk[a.dir]);  // 1 / w
  const double cm = face_mask(D, a.c1, a.comp, i, j, k);
  const double alpha = a.dte * cm + 1.0;
  const long c = D.P(i, j, k);
  if (!a.out) {
    a.xb[c] = cm == 0.0 ? a.xb[c] * rw : a.xb[c] * rw / alpha;
    return;
  }
  const double rb = cm == 0.0 ? a.xb[c] / rw : alpha * a.xb[c] / rw;
  a.cbar[D.C(i, j, k)] += rb * (cm == 0.0 ? a.dte : a.dte / alpha) * (a.rin[c] - a.xout[c]);
  if (a.next < 0) {
    a.xb[c] = rb;
    return;
  }
  const double rn = line_rw(a.g, a.next, a.comp, ijk[a.next]);
  a.xb[c] = cm == 0.0 ? rb * rn : rb * rn / alpha;
}

// -------------------------------------------------------- MKP transposes --
// adjoint of phi at the P2S sample positions (i = 0..nx-1, J = 1..ny,
// k = 0..nz-1): the correction u = u* - dt G, u_ta = dt G transposed
// (G_bar = dt (u_ta_bar - u_bar) on interior cells), then every padded
// cell that S2P's wrap fill and PHIBC copy from this sample folded back
struct GArgs {
  Dims D;
  AdjGrid g;
  const double* ub[3];
  const double* tab[3];
  double dt;
  double* xs;
};

__device__ __forceinline__ double gbar(const GArgs& a, int ax, const Pos& q) {
  if (!inside(a.D, q)) return 0.0;
  const long c = at(a.D, q);
  return a.dt * (a.tab[ax][c] - a.ub[ax][c]) * a.g.r12[ax][q.c[ax]];
}

__global__ void k_adj_phibar(GArgs a) {
  const Dims& D = a.D;
  const int si = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = 1 + blockIdx.y;
  const int sk = blockIdx.z;
  if (si >= D.nx) return;
  int qi[2], qk[2], qj[3];
  int ni = 0, nk = 0, nj = 0;
  qi[ni++] = si;
  if (si == 0) qi[ni++] = D.nx;
  if (si == 1) qi[ni++] = D.nx + 1;
  qk[nk++] = sk;
  if (sk == 0) qk[nk++] = D.nz;
  if (sk == 1) qk[nk++] = D.nz + 1;
  qj[nj++] = J;
  if (J == 1) qj[nj++] = 0;
  if (J == D.ny) qj[nj++] = D.ny + 1;
  double s = 0.0;
  for (int b = 0; b < nj; ++b)
    for (int e = 0; e < nk; ++e)
      for (int t = 0; t < ni; ++t) {
        Pos q;
        q.c[0] = qi[t]; q.c[1] = qj[b]; q.c[2] = qk[e];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) s += gbar(a, ax, sh(q, ax, -1)) - gbar(a, ax, q);
      }
  a.xs[D.P(si, J, sk)] = s;
}

// transposed SPN (per wavenumber, transposed Neumann-folded tridiagonal)
// and transposed SP0B (reverse marching) on the spectrum, in place
__global__ void k_adj_spn(int H, int ny, int nz, double* spec, long svj, long svk, double* sc,
                          long scj, long sck, const double* __restrict__ AC,
                          const double* __restrict__ KXZ) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int kx = t >> 1, comp = t & 1;
  const int kz = blockIdx.y;
  if (kx >= H || kz >= nz) return;
  const double* AC1 = AC;
  const double* AC2 = AC + ny;
  const double* AC3 = AC + 2 * ny;
  double* B = spec + 2 * (kx + svk * kz) + comp;
  const long sj = 2 * svj;
  if (kx == 0 && kz == 0) {
    // forward: phi(1) = 0, phi(J+1) = (D(J) - AC1 phi(J-1) - AC2 phi(J)) / AC3,
    // J = 1..ny-1.  Reverse: t(J) = (phibar(J+1) - AC2(J+1) t(J+1)
    // - AC1(J+2) t(J+2)) / AC3(J), Dbar(J) = t(J), Dbar(ny) = 0
    double t1 = 0.0, t2 = 0.0;
    double nxt = (double)B[sj * (ny - 1)];  // phibar(ny)
    B[sj * (ny - 1)] = 0.0;
    for (int J = ny - 1; J >= 1; --J) {
      const double pb = nxt;                   // phibar(J+1)
      nxt = (double)B[sj * (J - 1)];           // phibar(J), read before it is replaced
      double v = pb - AC2[J] * t1;
      if (J + 1 <= ny - 1) v -= AC1[J + 1] * t2;
      const double tj = v / AC3[J - 1];
      B[sj * (J - 1)] = tj;
      t2 = t1;
      t1 = tj;
    }
    return;
  }
  const double kxz = KXZ[kx + (long)H * kz];
  double* s3 = sc + kx + sck * kz;
  const int N = ny;
  // forward row r (1-based): a = AC1(r) (0 for r = 1), b = AC2(r) - kxz
  // (+AC1(1) for r = 1, +AC3(N) for r = N), c = AC3(r) (0 for r = N).
  // Transposed: sub'(r) = c(r-1), sup'(r) = a(r+1)
  auto diag = [&](int r) {
    double b = AC2[r - 1] - kxz;
    if (r == 1) b = b + AC1[0];
    if (r == N) b = b + AC3[N - 1];
    return b;
  };
  double cp_prev = 0.0, y_prev = 0.0;
  for (int r = 1; r <= N; ++r) {
    const double sub = r > 1 ? AC3[r - 2] : 0.0;
    const double sup = r < N ? AC1[r] : 0.0;
    const double mm = diag(r) - sub * cp_prev;
    const double cp = sup / mm;
    const double y = ((double)B[sj * (r - 1)] - sub * y_prev) / mm;
    s3[scj * (r - 1)] = cp;
    B[sj * (r - 1)] = y;
    cp_prev = cp;
    y_prev = y;
  }
  double ynext = y_prev;
  for (int r = N - 1; r >= 1; --r) {
    const double y = (double)B[sj * (r - 1)] - s3[scj * (r - 1)] * ynext;
    B[sj * (r - 1)] = y;
    ynext = y;
  }
}

// adjoint of u*, v*, w* after the transposed Poisson solve: the identity part
// of the correction plus the transposed divergence (rb holds the adjoint of
// the right-hand side at cell (i, J, k) = sample (i mod nx, J, k mod nz)),
// with the periodic ghost u*(0) folded onto u*(nx) and the wall rows of v*
// dropped (SET_BC sets them)
struct DArgs {
  Dims D;
  AdjGrid g;
  double* ub[3];  // in: adjoint of the corrected u, v, w; out: adjoint of u*, v*, w*
  const double* rb;
  double rdt;     // 1 / dt
};

__global__ void k_adj_div(DArgs a) {
  const Dims& D = a.D;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx) return;
  const long c = D.P(i, j, k);
  const double r0 = a.rb[c];
  {
    const int ip = i == D.nx ? 1 : i + 1;
    a.ub[0][c] += (r0 * a.g.r[0][i] - a.rb[D.P(ip, j, k)] * a.g.r[0][ip]) * a.rdt;
  }
  if (j < D.ny)
    a.ub[1][c] += (r0 * a.g.r[1][j] - a.rb[D.P(i, j + 1, k)] * a.g.r[1][j + 1]) * a.rdt;
  else
    a.ub[1][c] = 0.0;
  {
    const int kp = k == D.nz ? 1 : k + 1;
    a.ub[2][c] += (r0 * a.g.r[2][k] - a.rb[D.P(i, j, kp)] * a.g.r[2][kp]) * a.rdt;
  }
}

// ---------------------------------------------------------- objective --
// J += w * sum_ik a_ik thc (T(i,1,k) - (2 tb - T(i,1,k))) / dy12(0),
// a_ik = dx_i dz_k / (xl zl); one CTA, fixed summation order
__global__ void k_wall_flux(Dims D, AdjGrid g, const double* T, double tb, double thc,
                            double xl, double zl, double w, double* J) {
  __shared__ double red[1024];
  double s = 0.0;
  const long n = (long)D.nx * D.nz;
  for (long t = threadIdx.x; t < n; t += blockDim.x) {
    const int i = 1 + (int)(t % D.nx), k = 1 + (int)(t / D.nx);
    const double a = g.d[0][i] * g.d[2][k] / (xl * zl);
    const double T1 = T[D.P(i, 1, k)];
    s += a * thc * (T1 - (2.0 * tb - T1)) / g.d12[1][0];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *J += w * red[0];
}

__global__ void k_adj_wall_flux(Dims D, AdjGrid g, double* Tb, double thc, double xl,
                                double zl, double w) {
  const long n = (long)D.nx * D.nz;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = 1 + (int)(t % D.nx), k = 1 + (int)(t / D.nx);
  const double a = g.d[0][i] * g.d[2][k] / (xl * zl);
  Tb[D.P(i, 1, k)] += w * 2.0 * a * thc / g.d12[1][0];
}

// sum of W f over interior cells (W padded like f), one CTA
__global__ void k_weighted_sum(Dims D, const double* W, const double* f, double* J) {
  __shared__ double red[1024];
  double s = 0.0;
  for (long t = threadIdx.x; t < D.ncell; t += blockDim.x) {
    const int i = 1 + (int)(t % D.nx);
    const int j = 1 + (int)((t / D.nx) % D.ny);
    const int k = 1 + (int)(t / ((long)D.nx * D.ny));
    const long c = D.P(i, j, k);
    s += W[c] * f[c];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *J += red[0];
}

__global__ void k_add_weights(Dims D, const double* W, double* fb) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= D.ncell) return;
  const int i = 1 + (int)(t % D.nx);
  const int j = 1 + (int)((t / D.nx) % D.ny);
  const int k = 1 + (int)(t / ((long)D.nx * D.ny));
  const long c = D.P(i, j, k);
  fb[c] += W[c];
}

// c1_bar += transposed face averages of SET_IMMERSED_BOUNDARY (the last face
// of each direction copies its cell)
__global__ void k_adj_face_fold(Dims D, double* c1b, const double* c2b, const double* c3b,
                                const double* c4b) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= D.ncell) return;
  const int i = 1 + (int)(t % D.nx);
  const int j = 1 + (int)((t / D.nx) % D.ny);
  const int k = 1 + (int)(t / ((long)D.nx * D.ny));
  double s = c1b[t];
  s += i < D.nx ? 0.5 * c2b[t] : c2b[t];
  if (i > 1) s += 0.5 * c2b[D.C(i - 1, j, k)];
  s += j < D.ny ? 0.5 * c3b[t] : c3b[t];
  if (j > 1) s += 0.5 * c3b[D.C(i, j - 1, k)];
  s += k < D.nz ? 0.5 * c4b[t] : c4b[t];
  if (k > 1) s += 0.5 * c4b[D.C(i, j, k - 1)];
  c1b[t] = s;
}

// ------------------------------------------------- adjoint.f drop-ins --
// set_adj_convect adjoint.f:1-125, written as the reference writes it
// (including v(i,j,k-1) at :45 and w_final(i,j,k+1)+w_final(i,j+1,k-1) at
// :79); interior cells
__global__ void k_set_adj_convect(Dims D, AdjGrid g, const double* u, const double* v,
                                  const double* w, const double* uf, const double* vf,
                                  const double* wf, double* u_v, double* v_v, double* w_v,
                                  double dt) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx) return;
  const double *dx = g.d[0], *dy = g.d[1], *dz = g.d[2];
  const double *dx12 = g.d12[0], *dy12 = g.d12[1], *dz12 = g.d12[2];
#define F_(a, di, dj, dk) a[D.P(i + (di), j + (dj), k + (dk))]
  {
    const double u1 = -((F_(uf, 0, 0, 0) + F_(uf, 1, 0, 0)) * (F_(u, 0, 0, 0) + F_(u, 1, 0, 0)) -
                        (F_(uf, 0, 0, 0) + F_(uf, -1, 0, 0)) * (F_(u, 0, 0, 0) + F_(u, -1, 0, 0))) /
                          dx12[i] -
                      F_(uf, 0, 0, 0) * (F_(u, -1, 0, 0) - F_(u, 1, 0, 0)) / dx12[i] * 2.0;
    const double u2 =
        -((F_(vf, 1, 0, 0) * dx[i + 1] + F_(vf, 0, 0, 0) * dx[i]) * (F_(u, 0, 1, 0) + F_(u, 0, 0, 0)) -
          (F_(vf, 1, -1, 0) * dx[i + 1] + F_(vf, 0, -1, 0) * dx[i]) * (F_(u, 0, 0, 0) + F_(u, 0, -1, 0))) /
            dx12[i] / dy[j] -
        ((F_(vf, 1, 0, 0) + F_(vf, 1, -1, 0)) * dx[i + 1] + (F_(vf, 0, 0, 0) + F_(vf, 0, -1, 0)) * dx[i]) /
            dx12[i] *
            (-F_(v, 1, 0, 0) - F_(v, 1, -1, 0) + F_(v, 0, 0, 0) + F_(v, 0, -1, 0)) / dx12[i] / 2.0;
    const double u3 =
        -((F_(wf, 1, 0, 0) * dx[i + 1] + F_(wf, 0, 0, 0) * dx[i]) * (F_(u, 0, 0, 1) + F_(u, 0, 0, 0)) -
          (F_(wf, 1, 0, -1) * dx[i + 1] + F_(wf, 0, 0, -1) * dx[i]) * (F_(u, 0, 0, 0) + F_(u, 0, 0, -1))) /
            dx12[i] / dz[k] -
        ((F_(wf, 1, 0, 0) + F_(wf, 1, 0, -1)) * dx[i + 1] + (F_(wf, 0, 0, 0) + F_(wf, 0, 0, -1)) * dx[i]) /
            dx12[i] *
            (-F_(w, 1, 0, 0) - F_(w, 1, 0, -1) + F_(w, 0, 0, 0) + F_(v, 0, 0, -1)) / dx12[i] / 2.0;
    F_(u_v, 0, 0, 0) = 0.25 * (-u1 - u2 - u3) * dt + 1.0 * dt;
  }
  {
    const double v1 =
        ((F_(uf, 0, 1, 0) * dy[j + 1] + F_(uf, 0, 0, 0) * dy[j]) * (F_(v, 1, 0, 0) + F_(v, 0, 0, 0)) -
         (F_(uf, -1, 1, 0) * dy[j + 1] + F_(uf, -1, 0, 0) * dy[j]) * (F_(v, 0, 0, 0) + F_(v, -1, 0, 0))) /
            dy12[j] / dx[i] -
        ((F_(uf, 0, 1, 0) + F_(uf, -1, 1, 0)) * dy[j + 1] + (F_(uf, 0, 0, 0) + F_(uf, -1, 0, 0)) * dy[j]) /
            dy12[j] *
            (-F_(u, 0, 1, 0) - F_(u, -1, 1, 0) + F_(u, 0, 0, 0) + F_(u, -1, 0, 0)) / dy12[j] / 2.0;
    const double v2 = ((F_(vf, 0, 0, 0) + F_(vf, 0, 1, 0)) * (F_(v, 0, 0, 0) + F_(v, 0, 1, 0)) -
                       (F_(vf, 0, 0, 0) + F_(vf, 0, -1, 0)) * (F_(v, 0, 0, 0) + F_(v, 0, -1, 0))) /
                          dy12[j] -
                      F_(vf, 0, 0, 0) * (F_(v, -1, 0, 0) - F_(v, 1, 0, 0)) * 2.0 / dy12[j];
    const double v3 =
        ((F_(wf, 0, 1, 0) * dy[j + 1] + F_(wf, 0, 0, 0) * dy[j]) * (F_(v, 0, 0, 1) + F_(v, 0, 0, 0)) -
         (F_(wf, 0, 1, -1) * dy[j + 1] + F_(wf, 0, 0, -1) * dy[j]) * (F_(v, 0, 0, 0) + F_(v, 0, 0, -1))) /
            dy12[j] / dz[k] -
        ((F_(wf, 0, 0, 1) + F_(wf, 0, 1, -1)) * dy[j + 1] + (F_(wf, 0, 0, 0) + F_(wf, 0, 0, -1)) * dy[j]) /
            dy12[j] *
            (-F_(w, 0, 1, 0) - F_(w, 0, 1, -1) + F_(w, 0, 0, 0) + F_(w, 0, 0, -1)) / dy12[j] / 2.0;
    F_(v_v, 0, 0, 0) = 0.25 * (-v1 - v2 - v3) * dt;
  }
  {
    const double w1 =
        ((F_(uf, 0, 0, 1) * dz[k + 1] + F_(uf, 0, 0, 0) * dz[k]) * (F_(w, 1, 0, 0) + F_(w, 0, 0, 0)) -
         (F_(uf, -1, 0, 1) * dz[k + 1] + F_(uf, -1, 0, 0) * dz[k]) * (F_(w, 0, 0, 0) + F_(w, -1, 0, 0))) /
            dz12[k] / dx[i] -
        ((F_(uf, 0, 0, 1) + F_(uf, -1, 0, 1)) * dz[k + 1] + (F_(uf, 0, 0, 0) + F_(uf, -1, 0, 0)) * dz[k]) /
            dz12[k] *
            (-F_(u, 0, 0, 1) - F_(u, -1, 0, 1) + F_(u, 0, 0, 0) + F_(u, -1, 0, 0)) / dz12[k] * 2.0;
    const double w2 =
        ((F_(vf, 0, 0, 1) * dz[k + 1] + F_(vf, 0, 0, 0) * dz[k]) * (F_(w, 0, 1, 0) + F_(w, 0, 0, 0)) -
         (F_(vf, 0, -1, 1) * dz[k + 1] + F_(vf, 0, -1, 0) * dz[k]) * (F_(w, 0, 0, 0) + F_(w, 0, -1, 0))) /
            dz12[k] / dy[j] -
        ((F_(vf, 0, 0, 1) + F_(vf, 0, -1, 1)) * dz[k + 1] + (F_(vf, 0, 0, 0) + F_(vf, 0, -1, 0)) * dz[k]) /
            dz12[k] *
            (-F_(v, 0, 0, 1) - F_(v, 0, -1, 1) + F_(v, 0, 0, 0) + F_(v, 0, -1, 0)) / dz12[k] * 2.0;
    const double w3 = ((F_(wf, 0, 0, 0) + F_(wf, 0, 0, 1)) * (F_(w, 0, 0, 0) + F_(w, 0, 0, 1)) -
                       (F_(wf, 0, 0, 0) + F_(wf, 0, 0, -1)) * (F_(w, 0, 0, 0) + F_(w, 0, 0, -1))) /
                          dz12[k] -
                      F_(wf, 0, 0, 0) * (F_(w, 0, 0, -1) - F_(w, 0, 0, 1)) * 2.0 / dz12[k];
    F_(w_v, 0, 0, 0) = 0.25 * (-w1 - w2 - w3) * dt;
  }
}

// set_adj_convection_for_scalar adjoint.f:128-181 (u, v, w, Re are unused
// arguments of the reference routine)
__global__ void k_set_adj_cscalar(Dims D, AdjGrid g, const double* T, const double* R,
                                  const double* uf, const double* vf, const double* wf,
                                  double* u_vT, double dt) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx) return;
  const double *dx = g.d[0], *dy = g.d[1], *dz = g.d[2];
  const double *dx12 = g.d12[0], *dy12 = g.d12[1], *dz12 = g.d12[2];
  const double uT =
      (-((F_(R, -1, 0, 0) * F_(T, -1, 0, 0) * dx[i] + F_(R, 0, 0, 0) * F_(T, 0, 0, 0) * dx[i - 1]) *
         F_(uf, -1, 0, 0)) / 2.0 / dx12[i - 1] +
       ((F_(R, 0, 0, 0) * F_(T, 0, 0, 0) * dx[i + 1] + F_(R, 1, 0, 0) * F_(T, 1, 0, 0) * dx[i]) *
        F_(uf, 0, 0, 0)) / 2.0 / dx12[i]) /
      dx[i];
  const double vT =
      (-((F_(R, 0, -1, 0) * F_(T, 0, -1, 0) * dy[j] + F_(R, 0, 0, 0) * F_(T, 0, 0, 0) * dy[j - 1]) *
         F_(vf, 0, -1, 0)) / 2.0 / dy12[j - 1] +
       ((F_(R, 0, 0, 0) * F_(T, 0, 0, 0) * dy[j + 1] + F_(R, 0, 1, 0) * F_(T, 0, 1, 0) * dy[j]) *
        F_(vf, 0, 0, 0)) / 2.0 / dy12[j]) /
      dy[j];
  const double wT =
      (-((F_(R, 0, 0, -1) * F_(T, 0, 0, -1) * dz[k] + F_(R, 0, 0, 0) * F_(T, 0, 0, 0) * dz[k - 1]) *
         F_(wf, 0, 0, -1)) / 2.0 / dz12[k - 1] +
       ((F_(R, 0, 0, 0) * F_(T, 0, 0, 0) * dz[k + 1] + F_(R, 0, 0, 1) * F_(T, 0, 0, 1) * dz[k]) *
        F_(wf, 0, 0, 0)) / 2.0 / dz12[k]) /
      dz[k];
  F_(u_vT, 0, 0, 0) = (uT + vT + wT) * dt / F_(R, 0, 0, 0) + 1.0 * dt;
}

// set_adj_NS_scalar adjoint.f:185-211 with the adjoint temperature given
__global__ void k_set_adj_ns_scalar(Dims D, AdjGrid g, const double* T, const double* Tf,
                                    double* u_s, double* v_s, double* w_s, double dt) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > D.nx) return;
  F_(u_s, 0, 0, 0) = dt * F_(Tf, 0, 0, 0) * (F_(T, 1, 0, 0) - F_(T, -1, 0, 0)) / g.d12[0][i] / 2;
  F_(v_s, 0, 0, 0) = dt * F_(Tf, 0, 0, 0) * (F_(T, 0, 1, 0) - F_(T, 0, -1, 0)) / g.d12[1][j] / 2;
  F_(w_s, 0, 0, 0) = dt * F_(Tf, 0, 0, 0) * (F_(T, 0, 0, 1) - F_(T, 0, 0, -1)) / g.d12[2][k] / 2;
#undef F_
}

dim3 cell_grid(const Dims& D, int bx) {
  return dim3((D.nx + bx - 1) / bx, D.ny, D.nz);
}

}  // namespace

// ============================================================== launchers ==
void launch_adj_explicit(const Dims& D, const AdjGrid& g, const double* const vel[3],
                         const double* T, double* const A[4], double* const B[4], double dt,
                         double Re, double Sc, double R, double L, double* const out[4],
                         cudaStream_t s, const cudaStream_t* side) {
  XArgs a;
  a.D = D; a.g = g;
  for (int c = 0; c < 3; ++c) { a.vel[c] = vel[c]; a.A[c] = A[c]; a.B[c] = B[c]; }
  a.T = T; a.At = A[3]; a.Bt = B[3];
  a.dt = dt; a.Re = Re; a.Sc = Sc; a.R = R; a.L = L;
  a.cfac = dt / Re / 2.0;
  a.dfac = dt / (2.0 * Re * Sc * R);
  a.qfac = -dt / R;
  const dim3 block(32, 8, 1);
  const dim3 grid((D.nx + 31) / 32, (D.ny + 7) / 8, D.nz);
  const cudaStream_t* ss = side ? side : nullptr;
  count_launch();
  k_adj_explicit<0><<<grid, block, 0, s>>>(a, out[0]);
  count_launch();
  k_adj_explicit<1><<<grid, block, 0, ss ? ss[0] : s>>>(a, out[1]);
  count_launch();
  k_adj_explicit<2><<<grid, block, 0, ss ? ss[1] : s>>>(a, out[2]);
  count_launch();
  k_adj_explicit<3><<<grid, block, 0, ss ? ss[2] : s>>>(a, out[3]);
}

void launch_adj_point(const Dims& D, double* const A[4], double* const B[4],
                      double* const bar_pre[4], double* const bar_ta[3],
                      const double* const ta[3], const double* const rin[4], const double* c1,
                      double* const cbar[4], double eta, double dt, double tsolid, int l,
                      cudaStream_t s) {
  PArgs a;
  a.D = D;
  for (int c = 0; c < 4; ++c) {
    a.A[c] = A[c]; a.B[c] = B[c]; a.bar_pre[c] = bar_pre[c]; a.rin[c] = rin[c];
    a.cbar[c] = cbar[c];
  }
  for (int c = 0; c < 3; ++c) { a.bar_ta[c] = bar_ta[c]; a.ta[c] = ta[c]; }
  a.c1 = c1; a.eta = eta; a.dt = dt; a.tsolid = tsolid;
  a.a1 = l == 1 ? 1.0 : 1.5;
  a.a2 = l == 1 ? 0.0 : -0.5;
  count_launch();
  k_adj_point<<<cell_grid(D, 128), 128, 0, s>>>(a);
}

void launch_adj_line_scale(const Dims& D, const AdjGrid& g, int dir, int comp, bool out,
                           double* xb, const double* rin, const double* xout, const double* c1,
                           double* cbar, double dt, double eta, cudaStream_t s, int next) {
  SArgs a;
  a.D = D; a.g = g; a.xb = xb; a.rin = rin; a.xout = xout; a.c1 = c1; a.cbar = cbar;
  a.dir = dir; a.comp = comp; a.out = out ? 1 : 0; a.next = out ? next : -1;
  a.dte = dt * eta;
  count_launch();
  k_adj_line_scale<<<cell_grid(D, 128), 128, 0, s>>>(a);
}

void launch_adj_phibar(const Dims& D, const AdjGrid& g, const double* const ub[3],
                       const double* const tab[3], double dt, double* xs, cudaStream_t s) {
  GArgs a;
  a.D = D; a.g = g; a.dt = dt; a.xs = xs;
  for (int c = 0; c < 3; ++c) { a.ub[c] = ub[c]; a.tab[c] = tab[c]; }
  const int bx = 64;
  count_launch();
  k_adj_phibar<<<dim3((D.nx + bx - 1) / bx, D.ny, D.nz), bx, 0, s>>>(a);
}

void launch_adj_spn(const PoissonPlan& pp, cudaStream_t s) {
  dim3 grid((2 * pp.H + 63) / 64, pp.nz);
  count_launch();
  k_adj_spn<<<grid, 64, 0, s>>>(pp.H, pp.ny, pp.nz, pp.spec, pp.Hp, (long)pp.Hp * pp.ny, pp.scr,
                                pp.Hp, (long)pp.Hp * pp.ny, pp.AC, pp.KXZ);
}

void launch_adj_div(const Dims& D, const AdjGrid& g, double* const ub[3], const double* rb,
                    double dt, cudaStream_t s) {
  DArgs a;
  a.D = D; a.g = g; a.rb = rb; a.rdt = 1.0 / dt;
  for (int c = 0; c < 3; ++c) a.ub[c] = ub[c];
  count_launch();
  k_adj_div<<<cell_grid(D, 128), 128, 0, s>>>(a);
}

void launch_wall_flux(const Dims& D, const AdjGrid& g, const double* T, double tb, double thc,
                      double xl, double zl, double w, double* J, cudaStream_t s) {
  count_launch();
  k_wall_flux<<<1, 1024, 0, s>>>(D, g, T, tb, thc, xl, zl, w, J);
}

void launch_adj_wall_flux(const Dims& D, const AdjGrid& g, double* Tb, double thc, double xl,
                          double zl, double w, cudaStream_t s) {
  long n = (long)D.nx * D.nz;
  count_launch();
  k_adj_wall_flux<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(D, g, Tb, thc, xl, zl, w);
}

void launch_weighted_sum(const Dims& D, const double* W, const double* f, double* J,
                         cudaStream_t s) {
  count_launch();
  k_weighted_sum<<<1, 1024, 0, s>>>(D, W, f, J);
}

void launch_add_weights(const Dims& D, const double* W, double* fb, cudaStream_t s) {
  count_launch();
  k_add_weights<<<(unsigned)((D.ncell + 255) / 256), 256, 0, s>>>(D, W, fb);
}

void launch_adj_face_fold(const Dims& D, double* c1b, const double* c2b, const double* c3b,
                          const double* c4b, cudaStream_t s) {
  count_launch();
  k_adj_face_fold<<<(unsigned)((D.ncell + 255) / 256), 256, 0, s>>>(D, c1b, c2b, c3b, c4b);
}

void launch_set_adj_convect(const Dims& D, const AdjGrid& g, const double* u, const double* v,
                            const double* w, const double* uf, const double* vf,
                            const double* wf, double* u_v, double* v_v, double* w_v, double dt,
                            cudaStream_t s) {
  count_launch();
  k_set_adj_convect<<<cell_grid(D, 64), 64, 0, s>>>(D, g, u, v, w, uf, vf, wf, u_v, v_v, w_v,
                                                     dt);
}

void launch_set_adj_cscalar(const Dims& D, const AdjGrid& g, const double* T, const double* R,
                            const double* uf, const double* vf, const double* wf,
                            double* u_vT, double dt, cudaStream_t s) {
  count_launch();
  k_set_adj_cscalar<<<cell_grid(D, 64), 64, 0, s>>>(D, g, T, R, uf, vf, wf, u_vT, dt);
}

void launch_set_adj_ns_scalar(const Dims& D, const AdjGrid& g, const double* T,
                              const double* Tf, double* u_s, double* v_s, double* w_s,
                              double dt, cudaStream_t s) {
  count_launch();
  k_set_adj_ns_scalar<<<cell_grid(D, 64), 64, 0, s>>>(D, g, T, Tf, u_s, v_s, w_s, dt);
}

}  // namespace nse
