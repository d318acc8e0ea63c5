// k_stencil.cu -- boundary conditions and right-hand-side stencils of the
// fractional step (nse_dominik.f:611-1341 and the driver loop :387-396).
//
// Every per-cell expression keeps the reference's evaluation order and this
// file is built with --fmad=false, so each value rounds exactly like the
// reference's Fortran (x86-64, no FMA) build of the same expression.
#include "common.cuh"

namespace nse {

#define LD(p, i) __ldg((p) + (i))

// ---------------------------------------------------------------- SET_BC --
// nse_dominik.f:611-753 applies, per field, an x pass (all j,k), a y pass
// (all i,k) and a z pass (all i,j), each copying from an interior plane of
// its own direction.  The composition is closed-form: the final ghost value
// at (i,j,k) is s * f(mx(i), my(j), mz(k)) with the periodic maps mx, mz and
// the y rule of the field; the kernel evaluates that directly for every cell
// of the ghost shell (and the v wall plane j=ny), reading only cells that
// are never written, so one launch replaces the 15 sequential passes.
// VT: storage type of u, v, w (float for the FP32 intermediates of the
// mixed-precision form)
template <class VT>
__device__ __forceinline__ void bc_cell(const Dims& d, VT* u, VT* v, VT* w, double* p,
                                        double* T, double tbot, double ttop, int which, int i,
                                        int j, int k) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  int mx = (i == 0) ? nx : (i == nx + 1 ? 1 : i);
  int mz = (k == 0) ? nz : (k == nz + 1 ? 1 : k);
  bool jlo = (j == 0), jhi = (j == ny + 1);
  int my = jlo ? 1 : (jhi ? ny : j);
  long dst = d.P(i, j, k);
  long src = d.P(mx, my, mz);
  if (which & 1) {  // u: y ghosts = -interior
    VT val = u[src];
    if (jlo || jhi) val = VT(-1.0) * val;
    if (dst != src) u[dst] = val;
  }
  if (which & 4) {  // w
    VT val = w[src];
    if (jlo || jhi) val = VT(-1.0) * val;
    if (dst != src) w[dst] = val;
  }
  if (which & 8) {  // p: Neumann copy
    if (dst != src) p[dst] = p[src];
  }
  if (which & 16) {  // T: -interior, or 2*T_wall - interior
    double val = T[src];
    if (jlo) val = (tbot == 0.0) ? -1.0 * val : 2.0 * tbot - val;
    if (jhi) val = (ttop == 0.0) ? -1.0 * val : 2.0 * ttop - val;
    if (dst != src) T[dst] = val;
  }
  if (which & 2) {  // v: v(.,0,.)=v(.,ny,.)=0; v(.,ny+1,.) only wrapped in x,z
    if (j == 0 || j == ny) {
      v[dst] = VT(0.0);
    } else {
      long s2 = d.P(mx, j, mz);
      if (s2 != dst) v[dst] = v[s2];
    }
  }
}

template <class VT>
__global__ void k_set_bc(Dims d, VT* u, VT* v, VT* w, double* p, double* T, double tbot,
                         double ttop, int which) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  long nA = 2L * (ny + 2) * (nz + 2);  // x faces
  long nB = 3L * nx * (nz + 2);        // y faces j = 0, ny, ny+1
  long nC = 2L * nx * ny;              // z faces
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (t < nA) {
    i = (t & 1) ? nx + 1 : 0;
    long r = t >> 1;
    j = (int)(r % (ny + 2));
    k = (int)(r / (ny + 2));
  } else if (t < nA + nB) {
    long r = t - nA;
    i = 1 + (int)(r % nx);
    r /= nx;
    int sel = (int)(r % 3);
    k = (int)(r / 3);
    j = sel == 0 ? 0 : (sel == 1 ? ny : ny + 1);
    if (sel == 1 && !(which & 2)) return;  // j=ny is only a v plane
    if (sel == 1) {
      // only v changes on the wall plane
      bc_cell(d, u, v, w, p, T, tbot, ttop, which & 2, i, j, k);
      return;
    }
  } else if (t < nA + nB + nC) {
    long r = t - nA - nB;
    i = 1 + (int)(r % nx);
    r /= nx;
    j = 1 + (int)(r % ny);
    k = (r / ny) ? nz + 1 : 0;
  } else {
    return;
  }
  bc_cell(d, u, v, w, p, T, tbot, ttop, which, i, j, k);
}

void launch_set_bc(const Dims& d, double* u, double* v, double* w, double* p, double* T,
                   double tbot, double ttop, int which, cudaStream_t s) {
  long n = 2L * (d.ny + 2) * (d.nz + 2) + 3L * d.nx * (d.nz + 2) + 2L * d.nx * d.ny;
  int bs = 256;
  count_launch();
  k_set_bc<double><<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(d, u, v, w, p, T, tbot, ttop,
                                                                which);
}
void launch_set_bc_f32(const Dims& d, float* u, float* v, float* w, double* p, double* T,
                       double tbot, double ttop, int which, cudaStream_t s) {
  long n = 2L * (d.ny + 2) * (d.nz + 2) + 3L * d.nx * (d.nz + 2) + 2L * d.nx * d.ny;
  int bs = 256;
  count_launch();
  k_set_bc<float><<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(d, u, v, w, p, T, tbot, ttop,
                                                               which);
}

// ------------------------------------------------------------ cell terms --
struct Cell3 {
  long c, xp, xm, yp, ym, zp, zm;
};
__device__ __forceinline__ Cell3 nbr(const Dims& d, int I, int J, int K) {
  Cell3 n;
  n.c = d.P(I, J, K);
  n.xp = n.c + 1; n.xm = n.c - 1;
  n.yp = n.c + d.sx; n.ym = n.c - d.sx;
  n.zp = n.c + d.sy; n.zm = n.c - d.sy;
  return n;
}

// SET_CONVECT nse_dominik.f:774-785 (without the force term)
__device__ __forceinline__ double conv_u(const Dims& d, const GridDev& g, const double* U,
                                         const double* V, const double* W, int I, int J,
                                         int K) {
  Cell3 n = nbr(d, I, J, K);
  double uc = LD(U, n.c);
  double U1 = ((uc + LD(U, n.xp)) * (uc + LD(U, n.xp)) - (uc + LD(U, n.xm)) * (uc + LD(U, n.xm))) /
              LD(g.dx12, I);
  double dxp = LD(g.dx, I + 1), dxc = LD(g.dx, I);
  double U2 = ((LD(V, n.xp) * dxp + LD(V, n.c) * dxc) * (LD(U, n.yp) + uc) -
               (LD(V, n.xp - d.sx) * dxp + LD(V, n.ym) * dxc) * (uc + LD(U, n.ym))) /
              LD(g.dx12, I) / LD(g.dy, J);
  double U3 = ((LD(W, n.xp) * dxp + LD(W, n.c) * dxc) * (LD(U, n.zp) + uc) -
               (LD(W, n.xp - d.sy) * dxp + LD(W, n.zm) * dxc) * (uc + LD(U, n.zm))) /
              LD(g.dx12, I) / LD(g.dz, K);
  return 0.25 * (-U1 - U2 - U3);
}
// :794-805
__device__ __forceinline__ double conv_v(const Dims& d, const GridDev& g, const double* U,
                                         const double* V, const double* W, int I, int J,
                                         int K) {
  Cell3 n = nbr(d, I, J, K);
  double vc = LD(V, n.c);
  double dyp = LD(g.dy, J + 1), dyc = LD(g.dy, J);
  double V1 = ((LD(U, n.yp) * dyp + LD(U, n.c) * dyc) * (LD(V, n.xp) + vc) -
               (LD(U, n.yp - 1) * dyp + LD(U, n.xm) * dyc) * (vc + LD(V, n.xm))) /
              LD(g.dy12, J) / LD(g.dx, I);
  double V2 = ((vc + LD(V, n.yp)) * (vc + LD(V, n.yp)) - (vc + LD(V, n.ym)) * (vc + LD(V, n.ym))) /
              LD(g.dy12, J);
  double V3 = ((LD(W, n.yp) * dyp + LD(W, n.c) * dyc) * (LD(V, n.zp) + vc) -
               (LD(W, n.yp - d.sy) * dyp + LD(W, n.zm) * dyc) * (vc + LD(V, n.zm))) /
              LD(g.dy12, J) / LD(g.dz, K);
  return 0.25 * (-V1 - V2 - V3);
}
// :814-825
__device__ __forceinline__ double conv_w(const Dims& d, const GridDev& g, const double* U,
                                         const double* V, const double* W, int I, int J,
                                         int K) {
  Cell3 n = nbr(d, I, J, K);
  double wc = LD(W, n.c);
  double dzp = LD(g.dz, K + 1), dzc = LD(g.dz, K);
  double W1 = ((LD(U, n.zp) * dzp + LD(U, n.c) * dzc) * (LD(W, n.xp) + wc) -
               (LD(U, n.zp - 1) * dzp + LD(U, n.xm) * dzc) * (wc + LD(W, n.xm))) /
              LD(g.dz12, K) / LD(g.dx, I);
  double W2 = ((LD(V, n.zp) * dzp + LD(V, n.c) * dzc) * (LD(W, n.yp) + wc) -
               (LD(V, n.zp - d.sx) * dzp + LD(V, n.ym) * dzc) * (wc + LD(W, n.ym))) /
              LD(g.dz12, K) / LD(g.dy, J);
  double W3 = ((wc + LD(W, n.zp)) * (wc + LD(W, n.zp)) - (wc + LD(W, n.zm)) * (wc + LD(W, n.zm))) /
              LD(g.dz12, K);
  return 0.25 * (-W1 - W2 - W3);
}

// SET_CONVECTION_FOR_SCALAR :852-879 -> (-UT-VT-WT)*DT/RHOCP (source added by caller)
// rcp == nullptr means uniform rhoCp = r0
__device__ __forceinline__ double conv_T(const Dims& d, const GridDev& g, const double* U,
                                         const double* V, const double* W, const double* T,
                                         const double* R, double r0, double DT, int I, int J,
                                         int K) {
  Cell3 n = nbr(d, I, J, K);
#define RR(x) (R ? LD(R, (x)) : r0)
  double rc = RR(n.c), tc = LD(T, n.c);
  double UT = (-((RR(n.xm) * LD(T, n.xm) * LD(g.dx, I) + rc * tc * LD(g.dx, I - 1)) * LD(U, n.xm)) /
                   2.0 / LD(g.dx12, I - 1) +
               ((rc * tc * LD(g.dx, I + 1) + RR(n.xp) * LD(T, n.xp) * LD(g.dx, I)) * LD(U, n.c)) /
                   2.0 / LD(g.dx12, I)) /
              LD(g.dx, I);
  double VT = (-((RR(n.ym) * LD(T, n.ym) * LD(g.dy, J) + rc * tc * LD(g.dy, J - 1)) * LD(V, n.ym)) /
                   2.0 / LD(g.dy12, J - 1) +
               ((rc * tc * LD(g.dy, J + 1) + RR(n.yp) * LD(T, n.yp) * LD(g.dy, J)) * LD(V, n.c)) /
                   2.0 / LD(g.dy12, J)) /
              LD(g.dy, J);
  double WT = (-((RR(n.zm) * LD(T, n.zm) * LD(g.dz, K) + rc * tc * LD(g.dz, K - 1)) * LD(W, n.zm)) /
                   2.0 / LD(g.dz12, K - 1) +
               ((rc * tc * LD(g.dz, K + 1) + RR(n.zp) * LD(T, n.zp) * LD(g.dz, K)) * LD(W, n.c)) /
                   2.0 / LD(g.dz12, K)) /
              LD(g.dz, K);
#undef RR
  return (-UT - VT - WT) * DT / rc;
}

// SET_CONDUCTION :903-909 ; returns U1+U2+U3 (scaled by caller)
__device__ __forceinline__ double lap_u(const Dims& d, const GridDev& g, const double* U,
                                        int I, int J, int K) {
  Cell3 n = nbr(d, I, J, K);
  double c = LD(U, n.c);
  double U1 = ((LD(U, n.xp) - c) / LD(g.dx, I + 1) - (c - LD(U, n.xm)) / LD(g.dx, I)) / LD(g.dx12, I);
  double U2 = ((LD(U, n.yp) - c) / LD(g.dy12, J) - (c - LD(U, n.ym)) / LD(g.dy12, J - 1)) / LD(g.dy, J);
  double U3 = ((LD(U, n.zp) - c) / LD(g.dz12, K) - (c - LD(U, n.zm)) / LD(g.dz12, K - 1)) / LD(g.dz, K);
  return U1 + U2 + U3;
}
__device__ __forceinline__ double lap_v(const Dims& d, const GridDev& g, const double* V,
                                        int I, int J, int K) {
  Cell3 n = nbr(d, I, J, K);
  double c = LD(V, n.c);
  double V1 = ((LD(V, n.xp) - c) / LD(g.dx12, I) - (c - LD(V, n.xm)) / LD(g.dx12, I - 1)) / LD(g.dx, I);
  double V2 = ((LD(V, n.yp) - c) / LD(g.dy, J + 1) - (c - LD(V, n.ym)) / LD(g.dy, J)) / LD(g.dy12, J);
  double V3 = ((LD(V, n.zp) - c) / LD(g.dz12, K) - (c - LD(V, n.zm)) / LD(g.dz12, K - 1)) / LD(g.dz, K);
  return V1 + V2 + V3;
}
__device__ __forceinline__ double lap_w(const Dims& d, const GridDev& g, const double* W,
                                        int I, int J, int K) {
  Cell3 n = nbr(d, I, J, K);
  double c = LD(W, n.c);
  double W1 = ((LD(W, n.xp) - c) / LD(g.dx12, I) - (c - LD(W, n.xm)) / LD(g.dx12, I - 1)) / LD(g.dx, I);
  double W2 = ((LD(W, n.yp) - c) / LD(g.dy12, J) - (c - LD(W, n.ym)) / LD(g.dy12, J - 1)) / LD(g.dy, J);
  double W3 = ((LD(W, n.zp) - c) / LD(g.dz, K + 1) - (c - LD(W, n.zm)) / LD(g.dz, K)) / LD(g.dz12, K);
  return W1 + W2 + W3;
}

// SET_DIFFUSION_FOR_SCALAR :969-999 -> (UT1+UT2+UT3)/2/RE/SC/RHOCP*DT
__device__ __forceinline__ double diff_T(const Dims& d, const GridDev& g, const double* T,
                                         const double* L, const double* R, double l0,
                                         double r0, double RE, double SC, double DT, int I,
                                         int J, int K) {
  Cell3 n = nbr(d, I, J, K);
#define LL(x) (L ? LD(L, (x)) : l0)
  double tc = LD(T, n.c), lc = LL(n.c);
  double UT1 = ((LD(g.dx, I + 1) + LD(g.dx, I)) / (LD(g.dx, I + 1) / LL(n.xp) + LD(g.dx, I) / lc) *
                    (LD(T, n.xp) - tc) / LD(g.dx12, I) -
                (LD(g.dx, I - 1) + LD(g.dx, I)) / (LD(g.dx, I - 1) / LL(n.xm) + LD(g.dx, I) / lc) *
                    (tc - LD(T, n.xm)) / LD(g.dx12, I - 1)) /
               LD(g.dx, I);
  double UT2 = ((LD(g.dy, J + 1) + LD(g.dy, J)) / (LD(g.dy, J + 1) / LL(n.yp) + LD(g.dy, J) / lc) *
                    (LD(T, n.yp) - tc) / LD(g.dy12, J) -
                (LD(g.dy, J - 1) + LD(g.dy, J)) / (LD(g.dy, J - 1) / LL(n.ym) + LD(g.dy, J) / lc) *
                    (tc - LD(T, n.ym)) / LD(g.dy12, J - 1)) /
               LD(g.dy, J);
  double UT3 = ((LD(g.dz, K + 1) + LD(g.dz, K)) / (LD(g.dz, K + 1) / LL(n.zp) + LD(g.dz, K) / lc) *
                    (LD(T, n.zp) - tc) / LD(g.dz12, K) -
                (LD(g.dz, K - 1) + LD(g.dz, K)) / (LD(g.dz, K - 1) / LL(n.zm) + LD(g.dz, K) / lc) *
                    (tc - LD(T, n.zm)) / LD(g.dz12, K - 1)) /
               LD(g.dz, K);
#undef LL
  double rc = R ? LD(R, n.c) : r0;
  return (UT1 + UT2 + UT3) / 2.0 / RE / SC / rc * DT;
}

// face masks of SET_IMMERSED_BOUNDARY :1037-1080 from c1 (nx,ny,nz)
__device__ __forceinline__ double face_mask(const Dims& d, const double* c1, int comp, int i,
                                            int j, int k) {
  long c = d.C(i, j, k);
  double a = LD(c1, c);
  if (comp == 0) return (i < d.nx) ? (a + LD(c1, c + 1)) * 0.50 : a;
  if (comp == 1) return (j < d.ny) ? (a + LD(c1, c + d.nx)) * 0.50 : a;
  if (comp == 2) return (k < d.nz) ? (a + LD(c1, c + (long)d.nx * d.ny)) * 0.50 : a;
  return a;
}

// ------------------------------------------------------ interior launcher --
struct Interior {
  dim3 grid, block;
};
static Interior interior_shape(const Dims& d) {
  Interior r;
  r.block = dim3(64, 4, 1);
  r.grid = dim3((d.nx + 63) / 64, (d.ny + 3) / 4, d.nz);
  return r;
}
#define INTERIOR_IJK                                  \
  int I = 1 + blockIdx.x * blockDim.x + threadIdx.x; \
  int J = 1 + blockIdx.y * blockDim.y + threadIdx.y; \
  int K = 1 + blockIdx.z;                            \
  if (I > d.nx || J > d.ny) return;

__global__ void k_convect(Dims d, GridDev g, const double* U, const double* V, const double* W,
                          double* U_V, double* V_V, double* W_V, double DT, double force) {
  INTERIOR_IJK
  long c = d.P(I, J, K);
  U_V[c] = conv_u(d, g, U, V, W, I, J, K) * DT + force * DT;
  V_V[c] = conv_v(d, g, U, V, W, I, J, K) * DT;
  W_V[c] = conv_w(d, g, U, V, W, I, J, K) * DT;
}
void launch_convect(const Dims& d, const GridDev& g, const double* u, const double* v,
                    const double* w, double* u_v, double* v_v, double* w_v, double dt,
                    double force, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_convect<<<sh.grid, sh.block, 0, s>>>(d, g, u, v, w, u_v, v_v, w_v, dt, force);
}

__global__ void k_convect_scalar(Dims d, GridDev g, const double* U, const double* V,
                                 const double* W, const double* T, const double* R,
                                 double* U_VT, double DT, double source) {
  INTERIOR_IJK
  U_VT[d.P(I, J, K)] = conv_T(d, g, U, V, W, T, R, 1.0, DT, I, J, K) + source * DT;
}
void launch_convect_scalar(const Dims& d, const GridDev& g, const double* u,
                           const double* v, const double* w, const double* T,
                           const double* rcp, double* u_vT, double dt, double source,
                           cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_convect_scalar<<<sh.grid, sh.block, 0, s>>>(d, g, u, v, w, T, rcp, u_vT, dt, source);
}

__global__ void k_conduction(Dims d, GridDev g, const double* U, const double* V,
                             const double* W, double* U_D, double* V_D, double* W_D,
                             double RE, double DT) {
  INTERIOR_IJK
  long c = d.P(I, J, K);
  U_D[c] = DT / RE / 2.0 * lap_u(d, g, U, I, J, K);
  V_D[c] = DT / RE / 2.0 * lap_v(d, g, V, I, J, K);
  W_D[c] = DT / RE / 2.0 * lap_w(d, g, W, I, J, K);
}
void launch_conduction(const Dims& d, const GridDev& g, const double* u, const double* v,
                       const double* w, double* u_d, double* v_d, double* w_d, double Re,
                       double dt, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_conduction<<<sh.grid, sh.block, 0, s>>>(d, g, u, v, w, u_d, v_d, w_d, Re, dt);
}

__global__ void k_diffusion_scalar(Dims d, GridDev g, const double* T, const double* L,
                                   const double* R, double* U_DT, double RE, double SC,
                                   double DT) {
  INTERIOR_IJK
  U_DT[d.P(I, J, K)] = diff_T(d, g, T, L, R, 1.0, 1.0, RE, SC, DT, I, J, K);
}
void launch_diffusion_scalar(const Dims& d, const GridDev& g, const double* T,
                             const double* thc, const double* rcp, double* u_dT, double Re,
                             double Sc, double dt, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_diffusion_scalar<<<sh.grid, sh.block, 0, s>>>(d, g, T, thc, rcp, u_dT, Re, Sc, dt);
}

// cellvalue(:,:,:,2..4) from column 1 (SET_IMMERSED_BOUNDARY at l == 1)
__global__ void k_face_masks(Dims d, double* cv) {
  INTERIOR_IJK
  long c = d.C(I, J, K);
  long col = d.ncell;
  cv[c + col] = face_mask(d, cv, 0, I, J, K);
  cv[c + 2 * col] = face_mask(d, cv, 1, I, J, K);
  cv[c + 3 * col] = face_mask(d, cv, 2, I, J, K);
}
void launch_build_face_masks(const Dims& d, double* cellvalue4, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_face_masks<<<sh.grid, sh.block, 0, s>>>(d, cellvalue4);
}

// SET_IMMERSED_BOUNDARY :1086-1126
__global__ void k_ib_forcing(Dims d, const double* cv, const double* U_TA, const double* V_TA,
                             const double* W_TA, double* U_L, double* V_L, double* W_L,
                             double* T_L, double ETA, double DT) {
  INTERIOR_IJK
  long c = d.P(I, J, K);
  long m = d.C(I, J, K);
  U_L[c] = ETA * LD(cv, m + d.ncell) * LD(U_TA, c) * DT;
  V_L[c] = ETA * LD(cv, m + 2 * d.ncell) * LD(V_TA, c) * DT;
  W_L[c] = ETA * LD(cv, m + 3 * d.ncell) * LD(W_TA, c) * DT;
  T_L[c] = 0.0;
}
void launch_ib_forcing(const Dims& d, const double* cellvalue4, const double* u_ta,
                       const double* v_ta, const double* w_ta, double* u_l, double* v_l,
                       double* w_l, double* T_l, double eta, double dt, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_ib_forcing<<<sh.grid, sh.block, 0, s>>>(d, cellvalue4, u_ta, v_ta, w_ta, u_l, v_l, w_l,
                                            T_l, eta, dt);
}

// SET_EXPLICIT :1162-1171 (+ pre update :1275-1283); the ghost copies of
// :1176-1272 are applied by k_explicit_ghosts afterwards
__global__ void k_explicit(Dims d, const double* u_v, double* u_pre, const double* u_d,
                           double* u_a, const double* v_v, double* v_pre, const double* v_d,
                           double* v_a, const double* w_v, double* w_pre, const double* w_d,
                           double* w_a, const double* u_l, const double* v_l,
                           const double* w_l, double a1, double a2, double b1) {
  INTERIOR_IJK
  long c = d.P(I, J, K);
  double uv = u_v[c], vv = v_v[c], wv = w_v[c];
  u_a[c] = a1 * uv + a2 * u_pre[c] + b1 * u_d[c] + b1 * u_l[c];
  v_a[c] = a1 * vv + a2 * v_pre[c] + b1 * v_d[c] + b1 * v_l[c];
  w_a[c] = a1 * wv + a2 * w_pre[c] + b1 * w_d[c] + b1 * w_l[c];
  u_pre[c] = uv;
  v_pre[c] = vv;
  w_pre[c] = wv;
}
// ghost copies of SET_EXPLICIT: x (j,k interior), y (i,k interior, sign -1),
// z (i,j interior); these regions are disjoint and read interior cells only
__global__ void k_explicit_ghosts(Dims d, double* a) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  long nA = 2L * ny * nz, nB = 2L * nx * nz, nC = 2L * nx * ny;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nA) {
    int side = (int)(t & 1);
    long r = t >> 1;
    int j = 1 + (int)(r % ny), k = 1 + (int)(r / ny);
    if (side == 0) a[d.P(0, j, k)] = a[d.P(nx, j, k)];
    else a[d.P(nx + 1, j, k)] = a[d.P(1, j, k)];
  } else if (t < nA + nB) {
    long r = t - nA;
    int side = (int)(r & 1);
    r >>= 1;
    int i = 1 + (int)(r % nx), k = 1 + (int)(r / nx);
    if (side == 0) a[d.P(i, 0, k)] = -1.0 * a[d.P(i, 1, k)];
    else a[d.P(i, ny + 1, k)] = -1.0 * a[d.P(i, ny, k)];
  } else if (t < nA + nB + nC) {
    long r = t - nA - nB;
    int side = (int)(r & 1);
    r >>= 1;
    int i = 1 + (int)(r % nx), j = 1 + (int)(r / nx);
    if (side == 0) a[d.P(i, j, 0)] = a[d.P(i, j, nz)];
    else a[d.P(i, j, nz + 1)] = a[d.P(i, j, 1)];
  }
}
void launch_explicit(const Dims& d, const double* u_v, double* u_pre, const double* u_d,
                     double* u_a, const double* v_v, double* v_pre, const double* v_d,
                     double* v_a, const double* w_v, double* w_pre, const double* w_d,
                     double* w_a, const double* u_l, const double* v_l, const double* w_l,
                     int l, cudaStream_t s) {
  double a1 = (l == 1) ? 1.0 : 1.5, a2 = (l == 1) ? 0.0 : -0.5, b1 = 1.0;
  Interior sh = interior_shape(d);
  count_launch();
  k_explicit<<<sh.grid, sh.block, 0, s>>>(d, u_v, u_pre, u_d, u_a, v_v, v_pre, v_d, v_a, w_v,
                                          w_pre, w_d, w_a, u_l, v_l, w_l, a1, a2, b1);
  long n = 2L * d.ny * d.nz + 2L * d.nx * d.nz + 2L * d.nx * d.ny;
  unsigned nb = (unsigned)((n + 255) / 256);
  count_launch();
  k_explicit_ghosts<<<nb, 256, 0, s>>>(d, u_a);
  count_launch();
  k_explicit_ghosts<<<nb, 256, 0, s>>>(d, v_a);
  count_launch();
  k_explicit_ghosts<<<nb, 256, 0, s>>>(d, w_a);
}

// set_explicit_for_tempreture :1310-1339
__global__ void k_explicit_T(Dims d, const double* u_vT, const double* u_dT, double* u_T,
                             double* T_pre, const double* T_l, double a1, double a2,
                             double b1) {
  INTERIOR_IJK
  long c = d.P(I, J, K);
  double vt = u_vT[c];
  u_T[c] = a1 * vt + a2 * T_pre[c] + b1 * u_dT[c] + b1 * T_l[c];
  T_pre[c] = vt;
}
// periodic ghosts :1319-1330: x over all (j,k), then z over all (i,j) where
// u_T(i,j,nz+1) = u_T(i,j,0) = u_T(i,j,nz) after the first of the two copies
__global__ void k_explicit_T_ghosts_x(Dims d, double* a) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long n = (long)(d.ny + 2) * (d.nz + 2);
  if (t >= n) return;
  int j = (int)(t % (d.ny + 2)), k = (int)(t / (d.ny + 2));
  a[d.P(0, j, k)] = a[d.P(d.nx, j, k)];
  a[d.P(d.nx + 1, j, k)] = a[d.P(1, j, k)];
}
__global__ void k_explicit_T_ghosts_z(Dims d, double* a) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long n = (long)(d.nx + 2) * (d.ny + 2);
  if (t >= n) return;
  int i = (int)(t % (d.nx + 2)), j = (int)(t / (d.nx + 2));
  double v = a[d.P(i, j, d.nz)];
  a[d.P(i, j, 0)] = v;
  a[d.P(i, j, d.nz + 1)] = v;
}
void launch_explicit_T(const Dims& d, const double* u_vT, const double* u_dT, double* u_T,
                       double* T_pre, const double* T_l, int l, cudaStream_t s) {
  double a1 = (l == 1) ? 1.0 : 1.5, a2 = (l == 1) ? 0.0 : -0.5, b1 = 1.0;
  Interior sh = interior_shape(d);
  count_launch();
  k_explicit_T<<<sh.grid, sh.block, 0, s>>>(d, u_vT, u_dT, u_T, T_pre, T_l, a1, a2, b1);
  long nx_ = (long)(d.ny + 2) * (d.nz + 2), nz_ = (long)(d.nx + 2) * (d.ny + 2);
  count_launch();
  k_explicit_T_ghosts_x<<<(unsigned)((nx_ + 255) / 256), 256, 0, s>>>(d, u_T);
  count_launch();
  k_explicit_T_ghosts_z<<<(unsigned)((nz_ + 255) / 256), 256, 0, s>>>(d, u_T);
}

// a = (base + a)/(1 + eta*mask*dt) on interior cells (nse_dominik.f:387-396,
// :1358-1365); mask indexed (nx,ny,nz); tsolid != 0 adds eta*mask*dt*tsolid
__global__ void k_penalize(Dims d, const double* base, double* a, const double* mask,
                           double eta, double dt, double tsolid) {
  INTERIOR_IJK
  long c = d.P(I, J, K);
  double m = LD(mask, d.C(I, J, K));
  if (tsolid == 0.0) a[c] = (base[c] + a[c]) / (1.0 + eta * m * dt);
  else a[c] = (base[c] + a[c] + eta * m * dt * tsolid) / (1.0 + eta * m * dt);
}
void launch_penalize(const Dims& d, const double* base, double* a, const double* mask,
                     double eta, double dt, double tsolid, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_penalize<<<sh.grid, sh.block, 0, s>>>(d, base, a, mask, eta, dt, tsolid);
}

// ------------------------------------------------------------ fused RHS --
// One thread per interior cell computes every explicit term of the step
// (set_convect, set_convection_for_scalar, set_conduction,
// set_diffusion_for_scalar, set_immersed_boundary, set_explicit,
// set_explicit_for_tempreture), then the penalised update of the driver loop
// and solve_u_temp (:387-396, :1358-1433).  Only the values that later stages
// read are stored: u_a, v_a, w_a, u_T (interior) and the AB2 histories.
// The v wall plane j = ny gets v_a = (v + 0)/(1+eta*c3*dt) because
// set_bc(u_a,v_a,...) zeroes v_a(:,ny,:) before the penalised update.
__global__ void __launch_bounds__(256) k_rhs_fused(
    Dims d, GridDev g, StepParams sp, const double* __restrict__ U,
    const double* __restrict__ V, const double* __restrict__ W, const double* __restrict__ T,
    const double* __restrict__ U_TA, const double* __restrict__ V_TA,
    const double* __restrict__ W_TA, double* __restrict__ U_PRE, double* __restrict__ V_PRE,
    double* __restrict__ W_PRE, double* __restrict__ T_PRE, const double* __restrict__ C1,
    double* __restrict__ U_A, double* __restrict__ V_A, double* __restrict__ W_A,
    double* __restrict__ U_T) {
  INTERIOR_IJK
  const double DT = sp.dt;
  const double a1 = (sp.l == 1) ? 1.0 : 1.5, a2 = (sp.l == 1) ? 0.0 : -0.5, b1 = 1.0;
  long c = d.P(I, J, K);
  double c2 = face_mask(d, C1, 0, I, J, K);
  double c3 = face_mask(d, C1, 1, I, J, K);
  double c4 = face_mask(d, C1, 2, I, J, K);
  double cc1 = LD(C1, d.C(I, J, K));
  double kd = DT / sp.Re / 2.0;
  // u
  {
    double uv = conv_u(d, g, U, V, W, I, J, K) * DT + sp.force * DT;
    double ud = kd * lap_u(d, g, U, I, J, K);
    double ul = sp.eta * c2 * LD(U_TA, c) * DT;
    double ua = a1 * uv + a2 * U_PRE[c] + b1 * ud + b1 * ul;
    U_PRE[c] = uv;
    U_A[c] = (LD(U, c) + ua) / (1.0 + sp.eta * c2 * DT);
  }
  // v
  {
    double vv = conv_v(d, g, U, V, W, I, J, K) * DT;
    double vd = kd * lap_v(d, g, V, I, J, K);
    double vl = sp.eta * c3 * LD(V_TA, c) * DT;
    double va = a1 * vv + a2 * V_PRE[c] + b1 * vd + b1 * vl;
    V_PRE[c] = vv;
    if (J == d.ny) va = 0.0;
    V_A[c] = (LD(V, c) + va) / (1.0 + sp.eta * c3 * DT);
  }
  // w
  {
    double wv = conv_w(d, g, U, V, W, I, J, K) * DT;
    double wd = kd * lap_w(d, g, W, I, J, K);
    double wl = sp.eta * c4 * LD(W_TA, c) * DT;
    double wa = a1 * wv + a2 * W_PRE[c] + b1 * wd + b1 * wl;
    W_PRE[c] = wv;
    W_A[c] = (LD(W, c) + wa) / (1.0 + sp.eta * c4 * DT);
  }
  // T
  {
    double r0 = sp.rho_cp, l0 = sp.thc;
    double vt = conv_T(d, g, U, V, W, T, nullptr, r0, DT, I, J, K) + sp.source * DT;
    double dtt = diff_T(d, g, T, nullptr, nullptr, l0, r0, sp.Re, sp.Sc, DT, I, J, K);
    double ut = a1 * vt + a2 * T_PRE[c] + b1 * dtt + b1 * 0.0;
    T_PRE[c] = vt;
    double tc = LD(T, c);
    double pen = sp.eta * cc1 * DT;
    if (sp.tsolid == 0.0) U_T[c] = (tc + ut) / (1.0 + pen);
    else U_T[c] = (tc + ut + pen * sp.tsolid) / (1.0 + pen);
  }
}

void launch_rhs_fused(const Dims& d, const GridDev& g, const StepParams& sp,
                      const double* u, const double* v, const double* w, const double* T,
                      const double* u_ta, const double* v_ta, const double* w_ta,
                      double* u_pre, double* v_pre, double* w_pre, double* T_pre,
                      const double* c1, double* u_a, double* v_a, double* w_a,
                      double* u_T, cudaStream_t s) {
  Interior sh = interior_shape(d);
  count_launch();
  k_rhs_fused<<<sh.grid, sh.block, 0, s>>>(d, g, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre,
                                           v_pre, w_pre, T_pre, c1, u_a, v_a, w_a, u_T);
}

// --------------------------------------------------------------- correct --
// mkp.f:141-217: gradient on 0..n, u = u* - dt G (0..n), p = PHI (1..n),
// u_ep2 = -dt grad p + u_ta (1..n, with p's old ghost at n+1), u_ta = dt G
// (0..n), divu of the corrected velocity (1..n)
__global__ void k_correct(Dims d, GridDev g, const double* __restrict__ PHI,
                          const double* __restrict__ ut, const double* __restrict__ vt,
                          const double* __restrict__ wt, double* p, double* u, double* v,
                          double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                          double* v_ep2, double* w_ep2, double* divu, double dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long c = d.P(i, j, k);
  double ph = PHI[c];
  double gx = (PHI[c + 1] - ph) / g.dx12[i];
  double gy = (PHI[c + d.sx] - ph) / g.dy12[j];
  double gz = (PHI[c + d.sy] - ph) / g.dz12[k];
  double un = ut[c] - dt * gx;
  double vn = vt[c] - dt * gy;
  double wn = wt[c] - dt * gz;
  u[c] = un;
  v[c] = vn;
  w[c] = wn;
  bool inner = (i >= 1 && j >= 1 && k >= 1);
  if (inner) {
    p[c] = ph;
    double pxp = (i < d.nx) ? PHI[c + 1] : p[c + 1];
    double pyp = (j < d.ny) ? PHI[c + d.sx] : p[c + d.sx];
    double pzp = (k < d.nz) ? PHI[c + d.sy] : p[c + d.sy];
    u_ep2[c] = -dt * (pxp - ph) / g.dx12[i] + u_ta[c];
    v_ep2[c] = -dt * (pyp - ph) / g.dy12[j] + v_ta[c];
    w_ep2[c] = -dt * (pzp - ph) / g.dz12[k] + w_ta[c];
    // corrected neighbours at i-1, j-1, k-1 (recomputed, same arithmetic)
    double um = ut[c - 1] - dt * ((ph - PHI[c - 1]) / g.dx12[i - 1]);
    double vm = vt[c - d.sx] - dt * ((ph - PHI[c - d.sx]) / g.dy12[j - 1]);
    double wm = wt[c - d.sy] - dt * ((ph - PHI[c - d.sy]) / g.dz12[k - 1]);
    divu[c] = (un - um) / g.dx[i] + (vn - vm) / g.dy[j] + (wn - wm) / g.dz[k];
  }
  u_ta[c] = dt * gx;
  v_ta[c] = dt * gy;
  w_ta[c] = dt * gz;
}

void launch_correct(const Dims& d, const GridDev& g, const double* PHI, const double* ut,
                    const double* vt, const double* wt, double* p, double* u, double* v,
                    double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                    double* v_ep2, double* w_ep2, double* divu, double dt, cudaStream_t s) {
  dim3 block(64, 4, 1);
  dim3 grid((d.nx + 1 + 63) / 64, (d.ny + 1 + 3) / 4, d.nz + 1);
  count_launch();
  k_correct<<<grid, block, 0, s>>>(d, g, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta, w_ta, u_ep2,
                                   v_ep2, w_ep2, divu, dt);
}

}  // namespace nse
