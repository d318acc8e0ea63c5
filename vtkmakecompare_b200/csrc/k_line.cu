// k_line.cu -- penalised ADI line solves (nse_dominik.f:1344-1501,
// :1505-1870, :2893-3045; periodic_implicit.f:1-93).
//
// One thread owns one grid line and runs the reference's own elimination on
// it, so the arithmetic (and, with --fmad=false, the rounding) is that of the
// reference:
//  * y lines: implicit_uy / implicit_vy / implicit_Ty build a dense
//    (n+2)^2 matrix per line and eliminate "from lower" (a UL factorisation).
//    Only three diagonals are ever non-zero, so the thread streams them:
//    pass 1 walks j = m..1, normalising row j and folding it into row j-1,
//    pass 2 walks j = 0..m forward.  Between the passes the normalised
//    sub-diagonal lives in a scratch field and the half-solved value in the
//    field itself.
//  * x and z lines: implicit_solver / implicit_Tx augment the periodic line
//    with two ghost rows and call cyclic (Sherman-Morrison, gamma = 1) which
//    runs TDMA twice with the same matrix; both right-hand sides share the
//    gam/bet recurrence so one forward and one backward sweep solve both,
//    and a third sweep applies x - fact*z.
// Consecutive threads own lines that are adjacent in x (y and z lines) so
// loads are coalesced; x lines are contiguous per thread and rely on L1.
#include "k_lines.cuh"

namespace nse {

#define LD(p, i) __ldg((p) + (i))

struct LineGeom {
  long base;  // padded index of element 0 of the line
  long es;    // element stride
  int i, j, k;
};

// mask value of row r on a line: either a given column of cellvalue
// (derive = false, m points at that column) or a face mask built from c1
struct MaskSrc {
  const double* m;
  int comp;  // 0 x-face (c2), 1 y-face (c3), 2 z-face (c4), 3 cell (c1)
  bool derive;
  __device__ double at(const Dims& d, int i, int j, int k) const {
    long c = d.C(i, j, k);
    if (!derive || comp == 3) return LD(m, c);
    double a = LD(m, c);
    if (comp == 0) return (i < d.nx) ? (a + LD(m, c + 1)) * 0.50 : a;
    if (comp == 1) return (j < d.ny) ? (a + LD(m, c + d.nx)) * 0.50 : a;
    return (k < d.nz) ? (a + LD(m, c + (long)d.nx * d.ny)) * 0.50 : a;
  }
};

// --------------------------------------------------------- UL (y) solver --
// Rows 0..m; interior rows 1..m-1 come from rowfn(r); boundary rows:
//   row 0: di = 1, up = up0 ;  row m: lo = lom, di = 1.
// rhs: row 0 = ft, row m = fb, row r = f[base + r*es].
template <class RowFn>
__device__ __forceinline__ void ul_line(double* __restrict__ f, double* __restrict__ lsc,
                                        long base, long es, int m, double up0, double lom,
                                        double ft, double fb, const RowFn& rowfn) {
  double aa = 1.0;  // current (modified) diagonal of row j
  double ut = fb;   // current (modified) rhs of row j
  double lo = lom;  // sub-diagonal of row j
  for (int j = m; j >= 1; --j) {
    double l = lo / aa;
    double up_j = ut / aa;
    long o = base + (long)j * es;
    f[o] = up_j;
    lsc[o] = l;
    Row rp;
    double rhs;
    if (j - 1 == 0) {
      rp.lo = 0.0; rp.di = 1.0; rp.up = up0;
      rhs = ft;
    } else {
      rp = rowfn(j - 1);
      rhs = f[base + (long)(j - 1) * es];
    }
    double bb = rp.up;
    aa = rp.di - bb * l;
    ut = rhs - bb * up_j;
    lo = rp.lo;
  }
  double x = ut / aa;
  f[base] = x;
  for (int j = 1; j <= m; ++j) {
    long o = base + (long)j * es;
    x = f[o] - lsc[o] * x;
    f[o] = x;
  }
}

// ------------------------------------------------------ cyclic (x,z) line --
// periodic_implicit.f:67-93 with a(0)=0,b(0)=0,c(0)=1, a(n+1)=1,b(n+1)=0,
// c(n+1)=0 and corners alpha = beta = -1 (:93-100, nse_dominik.f:1771-1778).
template <class RowFn>
__device__ __forceinline__ void cyc_line(double* __restrict__ f, double* __restrict__ gsc,
                                         double* __restrict__ zsc, long base, long es, int n,
                                         double ft, double fb, const RowFn& rowfn) {
  const double gamma = 1.0, alpha = -1.0, beta = -1.0;
  double bet = 0.0 - gamma;                     // bb(0) = b(0) - gamma
  double x = ft / bet;                          // TDMA(a,bb,c,r,x)
  double z = gamma / bet;                       // TDMA(a,bb,c,u,z), u(0)=gamma
  f[base] = x;
  zsc[base] = z;
  double cprev = 1.0;                           // c(0)
  for (int j = 1; j <= n + 1; ++j) {
    long o = base + (long)j * es;
    double a, b, c, r, uv;
    if (j == n + 1) {
      a = 1.0; b = 0.0 - alpha * beta / gamma; c = 0.0; r = fb; uv = alpha;
    } else {
      Row rw = rowfn(j);
      a = rw.lo; b = rw.di; c = rw.up; r = f[o]; uv = 0.0;
    }
    double gam = cprev / bet;
    bet = b - a * gam;
    x = (r - a * x) / bet;
    z = (uv - a * z) / bet;
    gsc[o] = gam;
    f[o] = x;
    zsc[o] = z;
    cprev = c;
  }
  double xn1 = x, zn1 = z;
  for (int j = n; j >= 0; --j) {
    long o = base + (long)j * es;
    double g1 = gsc[o + es];
    x = f[o] - g1 * x;
    z = zsc[o] - g1 * z;
    f[o] = x;
    zsc[o] = z;
  }
  double fact = (x + beta * xn1 / gamma) / (1.0 + z + beta * zn1 / gamma);
  for (int j = 0; j <= n + 1; ++j) {
    long o = base + (long)j * es;
    f[o] = f[o] - fact * zsc[o];
  }
}

// --------------------------------------------------------- velocity lines --
// dir: 0 x lines (j,k), 1 y lines (i,k), 2 z lines (i,j); comp 0 u,1 v,2 w
__device__ __forceinline__ bool line_of(const Dims& d, int dir, int jtop, long t,
                                        LineGeom& L) {
  if (dir == 1) {  // (i,k): i fastest
    if (t >= (long)d.nx * d.nz) return false;
    L.i = 1 + (int)(t % d.nx); L.k = 1 + (int)(t / d.nx); L.j = 0;
    L.base = d.P(L.i, 0, L.k); L.es = d.sx;
  } else if (dir == 2) {  // (i,j): i fastest
    if (t >= (long)d.nx * jtop) return false;
    L.i = 1 + (int)(t % d.nx); L.j = 1 + (int)(t / d.nx); L.k = 0;
    L.base = d.P(L.i, L.j, 0); L.es = d.sy;
  } else {  // (j,k): j fastest
    if (t >= (long)jtop * d.nz) return false;
    L.j = 1 + (int)(t % jtop); L.k = 1 + (int)(t / jtop); L.i = 0;
    L.base = d.P(0, L.j, L.k); L.es = 1;
  }
  return true;
}

__global__ void k_vel_line(Dims d, GridDev g, double* f, MaskSrc ms, int dir, int comp,
                           double Re, double dt, double eta, double* sa, double* sb) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int jtop = (comp == 1) ? d.ny - 1 : d.ny;
  LineGeom L;
  if (!line_of(d, dir, jtop, t, L)) return;
  const double beta = dt / Re / 2.0;
  if (dir == 1) {
    if (comp == 1) {  // implicit_vy over rows 0..ny
      auto rowfn = [&](int r) {
        double alpha = dt * eta * ms.at(d, L.i, r, L.k) + 1.0;
        return row_vy(beta, alpha, LD(g.dy, r), LD(g.dy, r + 1), LD(g.dy12, r));
      };
      ul_line(f, sa, L.base, L.es, d.ny, 0.0, 0.0, 0.0, 0.0, rowfn);
    } else {  // implicit_uy over rows 0..ny+1
      auto rowfn = [&](int r) {
        double alpha = dt * eta * ms.at(d, L.i, r, L.k) + 1.0;
        return row_uy(beta, alpha, LD(g.dy12, r - 1), LD(g.dy12, r), LD(g.dy, r));
      };
      ul_line(f, sa, L.base, L.es, d.ny + 1, 1.0, 1.0, 0.0, 0.0, rowfn);
    }
  } else if (dir == 2) {
    auto rowfn = [&](int r) {
      double alpha = dt * eta * ms.at(d, L.i, L.j, r) + 1.0;
      return row_cyc(beta, alpha, LD(g.dz, r), LD(g.dz, r + 1), LD(g.dz12, r));
    };
    cyc_line(f, sa, sb, L.base, L.es, d.nz, 0.0, 0.0, rowfn);
  } else {
    auto rowfn = [&](int r) {
      double alpha = dt * eta * ms.at(d, r, L.j, L.k) + 1.0;
      return row_cyc(beta, alpha, LD(g.dx, r), LD(g.dx, r + 1), LD(g.dx12, r));
    };
    cyc_line(f, sa, sb, L.base, L.es, d.nx, 0.0, 0.0, rowfn);
  }
}

static void launch_vel(const Dims& d, const GridDev& g, double* f, const double* mask,
                       bool derive, int dir, int comp, double Re, double dt, double eta,
                       double* sa, double* sb, cudaStream_t s) {
  int jtop = (comp == 1) ? d.ny - 1 : d.ny;
  long n = (dir == 1) ? (long)d.nx * d.nz : (dir == 2 ? (long)d.nx * jtop : (long)jtop * d.nz);
  MaskSrc ms{mask, comp, derive};
  int bs = 128;
  count_launch();
  k_vel_line<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(d, g, f, ms, dir, comp, Re, dt,
                                                          eta, sa, sb);
}

// derive: the mask pointer is c1 and face masks are built on the fly;
// otherwise it points at the cellvalue column of this component
void launch_ysolve_vel(const Dims& d, const GridDev& g, double* f, const double* c1,
                       int comp, double Re, double dt, double eta, const LineScratch& sc,
                       cudaStream_t s) {
  launch_vel(d, g, f, c1, true, 1, comp, Re, dt, eta, sc.a, sc.b, s);
}
void launch_zsolve_vel(const Dims& d, const GridDev& g, double* f, const double* c1,
                       int comp, double Re, double dt, double eta, const LineScratch& sc,
                       cudaStream_t s) {
  launch_vel(d, g, f, c1, true, 2, comp, Re, dt, eta, sc.a, sc.b, s);
}
void launch_xsolve_vel(const Dims& d, const GridDev& g, double* f, const double* c1,
                       int comp, double Re, double dt, double eta, const LineScratch& sc,
                       cudaStream_t s) {
  launch_vel(d, g, f, c1, true, 0, comp, Re, dt, eta, sc.a, sc.b, s);
}
void launch_vel_line_col(const Dims& d, const GridDev& g, double* f, const double* column,
                         int dir, int comp, double Re, double dt, double eta,
                         const LineScratch& sc, cudaStream_t s) {
  launch_vel(d, g, f, column, false, dir, comp, Re, dt, eta, sc.a, sc.b, s);
}

// ------------------------------------------------------ temperature lines --
struct Props {
  const double* rcp;  // padded or null
  const double* thc;  // padded or null
  double r0, l0;
  __device__ double r(long o) const { return rcp ? LD(rcp, o) : r0; }
  __device__ double l(long o) const { return thc ? LD(thc, o) : l0; }
};

__global__ void k_T_line(Dims d, GridDev g, double* f, const double* c1, Props pr, int dir,
                         double Re, double Sc, double dt, double eta, double ft, double fb,
                         double* sa, double* sb) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  LineGeom L;
  if (!line_of(d, dir, d.ny, t, L)) return;
  const double beta = dt / Re / Sc / 2.0;
  if (dir == 1) {
    auto rowfn = [&](int r) {
      long o = L.base + (long)r * L.es;
      double alpha = dt * eta * LD(c1, d.C(L.i, r, L.k)) + 1.0;
      return row_T(beta, alpha, LD(g.dy, r - 1), LD(g.dy, r), LD(g.dy, r + 1), LD(g.dy12, r - 1),
                   LD(g.dy12, r), pr.l(o - L.es), pr.l(o), pr.l(o + L.es), pr.r(o));
    };
    ul_line(f, sa, L.base, L.es, d.ny + 1, 1.0, 1.0, ft, fb, rowfn);
  } else if (dir == 2) {
    auto rowfn = [&](int r) {
      long o = L.base + (long)r * L.es;
      double alpha = dt * eta * LD(c1, d.C(L.i, L.j, r)) + 1.0;
      return row_T(beta, alpha, LD(g.dz, r - 1), LD(g.dz, r), LD(g.dz, r + 1), LD(g.dz12, r - 1),
                   LD(g.dz12, r), pr.l(o - L.es), pr.l(o), pr.l(o + L.es), pr.r(o));
    };
    cyc_line(f, sa, sb, L.base, L.es, d.nz, 0.0, 0.0, rowfn);
  } else {
    auto rowfn = [&](int r) {
      long o = L.base + (long)r * L.es;
      double alpha = dt * eta * LD(c1, d.C(r, L.j, L.k)) + 1.0;
      return row_T(beta, alpha, LD(g.dx, r - 1), LD(g.dx, r), LD(g.dx, r + 1), LD(g.dx12, r - 1),
                   LD(g.dx12, r), pr.l(o - L.es), pr.l(o), pr.l(o + L.es), pr.r(o));
    };
    cyc_line(f, sa, sb, L.base, L.es, d.nx, 0.0, 0.0, rowfn);
  }
}

static void launch_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0, int dir,
                     double Re, double Sc, double dt, double eta, double ft, double fb,
                     double* sa, double* sb, cudaStream_t s) {
  long n = (dir == 1) ? (long)d.nx * d.nz : (dir == 2 ? (long)d.nx * d.ny : (long)d.ny * d.nz);
  Props pr{rcp, thc, rcp0, thc0};
  int bs = 128;
  count_launch();
  k_T_line<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(d, g, f, c1, pr, dir, Re, Sc, dt,
                                                        eta, ft, fb, sa, sb);
}

void launch_ysolve_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0,
                     double Re, double Sc, double dt, double eta, double ft, double fb,
                     const LineScratch& sc, cudaStream_t s) {
  launch_T(d, g, f, c1, rcp, thc, rcp0, thc0, 1, Re, Sc, dt, eta, ft, fb, sc.a, sc.b, s);
}
void launch_zsolve_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0,
                     double Re, double Sc, double dt, double eta, const LineScratch& sc,
                     cudaStream_t s) {
  launch_T(d, g, f, c1, rcp, thc, rcp0, thc0, 2, Re, Sc, dt, eta, 0.0, 0.0, sc.a, sc.b, s);
}
void launch_xsolve_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0,
                     double Re, double Sc, double dt, double eta, const LineScratch& sc,
                     cudaStream_t s) {
  launch_T(d, g, f, c1, rcp, thc, rcp0, thc0, 0, Re, Sc, dt, eta, 0.0, 0.0, sc.a, sc.b, s);
}

// ----------------------------------------------- single-line entry points --
// tier-1/2 single-line routines run one system on one GPU thread
__global__ void k_single_ul(double* f, double* lsc, int kind, int n, GridDev g, double Re,
                            double Sc, double dt, double eta, double ft, double fb,
                            const double* cu, const double* ll, const double* rr) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (kind == 0) {  // implicit_uy: cu indexed 1..n at cu[r-1]
    double beta = dt / Re / 2.0;
    auto rowfn = [&](int r) {
      double alpha = dt * eta * cu[r - 1] + 1.0;
      return row_uy(beta, alpha, g.dy12[r - 1], g.dy12[r], g.dy[r]);
    };
    ul_line(f, lsc, 0, 1, n + 1, 1.0, 1.0, ft, fb, rowfn);
  } else if (kind == 1) {  // implicit_vy
    double beta = dt / Re / 2.0;
    auto rowfn = [&](int r) {
      double alpha = dt * eta * cu[r - 1] + 1.0;
      return row_vy(beta, alpha, g.dy[r], g.dy[r + 1], g.dy12[r]);
    };
    ul_line(f, lsc, 0, 1, n, 0.0, 0.0, ft, fb, rowfn);
  } else {  // implicit_Ty: cu, ll, rr indexed 0..n+1
    double beta = dt / Re / Sc / 2.0;
    auto rowfn = [&](int r) {
      double alpha = dt * eta * cu[r] + 1.0;
      return row_T(beta, alpha, g.dy[r - 1], g.dy[r], g.dy[r + 1], g.dy12[r - 1], g.dy12[r],
                   ll[r - 1], ll[r], ll[r + 1], rr[r]);
    };
    ul_line(f, lsc, 0, 1, n + 1, 1.0, 1.0, ft, fb, rowfn);
  }
}

__global__ void k_single_cyc(double* f, double* gsc, double* zsc, int kind, int n, GridDev g,
                             double Re, double Sc, double dt, double eta, double ft,
                             double fb, const double* cu, const double* ll,
                             const double* rr) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (kind == 0) {  // implicit_solver with dx=g.dx, dx12=g.dx12, CUX(1..n) at cu[r-1]
    double beta = dt / Re / 2.0;
    auto rowfn = [&](int r) {
      double alpha = dt * eta * cu[r - 1] + 1.0;
      return row_cyc(beta, alpha, g.dx[r], g.dx[r + 1], g.dx12[r]);
    };
    cyc_line(f, gsc, zsc, 0, 1, n, ft, fb, rowfn);
  } else {  // implicit_Tx: cu, ll, rr indexed 0..n+1
    double beta = dt / Re / Sc / 2.0;
    auto rowfn = [&](int r) {
      double alpha = dt * eta * cu[r] + 1.0;
      return row_T(beta, alpha, g.dx[r - 1], g.dx[r], g.dx[r + 1], g.dx12[r - 1], g.dx12[r],
                   ll[r - 1], ll[r], ll[r + 1], rr[r]);
    };
    cyc_line(f, gsc, zsc, 0, 1, n, ft, fb, rowfn);
  }
}

// general cyclic system of periodic_implicit.f:67 (given a,b,c,alpha,beta,r)
__global__ void k_single_cyclic_general(const double* a, const double* b, const double* c,
                                        double alpha, double beta, const double* r, double* x,
                                        double* bb, double* gam, double* z, int n) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double gamma = 1.0;
  bb[0] = b[0] - gamma;
  bb[n + 1] = b[n + 1] - alpha * beta / gamma;
  for (int i = 1; i <= n; ++i) bb[i] = b[i];
  // TDMA(a,bb,c,r,x) and TDMA(a,bb,c,u,z) (periodic_implicit.f:47-64)
  double bet = bb[0];
  x[0] = r[0] / bet;
  z[0] = gamma / bet;
  for (int j = 1; j <= n + 1; ++j) {
    gam[j] = c[j - 1] / bet;
    bet = bb[j] - a[j] * gam[j];
    double uj = (j == n + 1) ? alpha : 0.0;
    x[j] = (r[j] - a[j] * x[j - 1]) / bet;
    z[j] = (uj - a[j] * z[j - 1]) / bet;
  }
  for (int j = n; j >= 0; --j) {
    x[j] = x[j] - gam[j + 1] * x[j + 1];
    z[j] = z[j] - gam[j + 1] * z[j + 1];
  }
  double fact = (x[0] + beta * x[n + 1] / gamma) / (1.0 + z[0] + beta * z[n + 1] / gamma);
  for (int i = 0; i <= n + 1; ++i) x[i] = x[i] - fact * z[i];
}

__global__ void k_single_tdma(const double* a, const double* b, const double* c,
                              const double* r, double* u, double* gam, int n) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double bet = b[0];
  u[0] = r[0] / bet;
  for (int j = 1; j <= n + 1; ++j) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n; j >= 0; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
}

// TRIDIAG / CTRIDIAG / TRID2 (tridiag.f): A(NN,3) column-major, one thread
// per right-hand side column of TRID2 (the coefficient update is identical
// in every thread, so each keeps its own copy of the modified diagonal)
__global__ void k_tridiag(double* A, double* B, int NN, int ncomp, int ldb) {
  // ncomp = 1: real B(NN); 2: complex B(NN) interleaved.  One system.
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double* A1 = A; double* A2 = A + NN; double* A3 = A + 2 * NN;
  (void)ldb;
  for (int I = 0; I < NN - 1; ++I) {
    A3[I] = A3[I] / A2[I];
    for (int q = 0; q < ncomp; ++q) B[ncomp * I + q] = B[ncomp * I + q] / A2[I];
    A2[I + 1] = A2[I + 1] - A1[I + 1] * A3[I];
    for (int q = 0; q < ncomp; ++q)
      B[ncomp * (I + 1) + q] = B[ncomp * (I + 1) + q] - A1[I + 1] * B[ncomp * I + q];
  }
  for (int q = 0; q < ncomp; ++q) B[ncomp * (NN - 1) + q] = B[ncomp * (NN - 1) + q] / A2[NN - 1];
  for (int I = NN - 2; I >= 0; --I)
    for (int q = 0; q < ncomp; ++q)
      B[ncomp * I + q] = B[ncomp * I + q] - A3[I] * B[ncomp * (I + 1) + q];
}

__global__ void k_trid2(const double* A0, double* Amod, double* B, int M, int N) {
  // TRID2 tridiag.f:21-41; thread J owns column J of B(M,N).  The coefficient
  // recurrence is the same in every thread; thread 0 also stores the
  // overwritten A (column 3 and the modified diagonal) into Amod.
  int J = blockIdx.x * blockDim.x + threadIdx.x;
  if (J >= M) return;
  const double* A1 = A0; const double* A2i = A0 + N; const double* A3i = A0 + 2 * N;
  double a2 = A2i[0];
  for (int I = 0; I < N - 1; ++I) {
    double a3 = A3i[I] / a2;
    B[J + (long)M * I] = B[J + (long)M * I] / a2;
    double a2n = A2i[I + 1] - A1[I + 1] * a3;
    B[J + (long)M * (I + 1)] = B[J + (long)M * (I + 1)] - A1[I + 1] * B[J + (long)M * I];
    if (J == 0) { Amod[2 * N + I] = a3; Amod[N + I + 1] = a2n; }
    a2 = a2n;
  }
  B[J + (long)M * (N - 1)] = B[J + (long)M * (N - 1)] / a2;
}
__global__ void k_trid2_back(const double* Amod, double* B, int M, int N) {
  int J = blockIdx.x * blockDim.x + threadIdx.x;
  if (J >= M) return;
  for (int I = N - 2; I >= 0; --I)
    B[J + (long)M * I] = B[J + (long)M * I] - Amod[2 * N + I] * B[J + (long)M * (I + 1)];
}

}  // namespace nse

// launchers used by the legacy glue (declared here to keep common.cuh small)
namespace nse {
void launch_single_ul(double* f, double* lsc, int kind, int n, const GridDev& g, double Re,
                      double Sc, double dt, double eta, double ft, double fb, const double* cu,
                      const double* ll, const double* rr, cudaStream_t s) {
  count_launch();
  k_single_ul<<<1, 32, 0, s>>>(f, lsc, kind, n, g, Re, Sc, dt, eta, ft, fb, cu, ll, rr);
}
void launch_single_cyc(double* f, double* gsc, double* zsc, int kind, int n, const GridDev& g,
                       double Re, double Sc, double dt, double eta, double ft, double fb,
                       const double* cu, const double* ll, const double* rr, cudaStream_t s) {
  count_launch();
  k_single_cyc<<<1, 32, 0, s>>>(f, gsc, zsc, kind, n, g, Re, Sc, dt, eta, ft, fb, cu, ll, rr);
}
void launch_cyclic_general(const double* a, const double* b, const double* c, double alpha,
                           double beta, const double* r, double* x, double* bb, double* gam,
                           double* z, int n, cudaStream_t s) {
  count_launch();
  k_single_cyclic_general<<<1, 32, 0, s>>>(a, b, c, alpha, beta, r, x, bb, gam, z, n);
}
void launch_tdma(const double* a, const double* b, const double* c, const double* r, double* u,
                 double* gam, int n, cudaStream_t s) {
  count_launch();
  k_single_tdma<<<1, 32, 0, s>>>(a, b, c, r, u, gam, n);
}
void launch_tridiag(double* A, double* B, int NN, int ncomp, cudaStream_t s) {
  count_launch();
  k_tridiag<<<1, 32, 0, s>>>(A, B, NN, ncomp, 0);
}
void launch_trid2(const double* A0, double* Amod, double* B, int M, int N, cudaStream_t s) {
  int bs = 128;
  count_launch();
  k_trid2<<<(M + bs - 1) / bs, bs, 0, s>>>(A0, Amod, B, M, N);
  count_launch();
  k_trid2_back<<<(M + bs - 1) / bs, bs, 0, s>>>(Amod, B, M, N);
}
}  // namespace nse
