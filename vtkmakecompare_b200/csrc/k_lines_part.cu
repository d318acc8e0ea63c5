// k_lines_part.cu -- partitioned ADI line solver of the resident step (fast
// form).
//
// Every line system of the step (the UL systems of implicit_uy/vy/Ty,
// nse_dominik.f:1505-1648,1784-1870, and the augmented cyclic systems of
// implicit_solver/implicit_Tx, periodic_implicit.f:1-93, nse_dominik.f:
// 1725-1781) is, after folding its boundary rows, a tridiagonal system on
// the interior unknowns, periodic for the x and z lines:
//   UL u, w, T:  x0 = ft - x1 and x(n+1) = fb - x(n)   (rows 0 and n+1)
//   UL v:        x0 = ft, x(ny) = fb                     (Dirichlet)
//   cyclic:      x0 = x(n), x(n+1) = x(1)                (the ghost rows)
// The reference eliminates each line sequentially.  Here a line is cut into
// P partitions of m >= 3 rows.  Within a partition every interior row is
// written as x = g + F p + E q, where F and E are the partition's first and
// last unknowns, g solves the interior rows with F = E = 0 and p, q are the
// responses to unit F and E.  The first and last rows then form a reduced
// tridiagonal system of 2P unknowns (F0, E0, F1, E1, ...), periodic when the
// line is.  Everything that does not depend on the right-hand side -- the
// interior factorisation, p, q, and the factorisation of the reduced system
// -- is tabulated once per matrix: one table for all mask-free lines of a
// kind, one per line that touches the penalisation mask (the mask is fixed
// between level-set calls).  A solve then costs one read and one write of
// the line plus a few FMAs per row, with the rows held in registers.
//
//   x lines (contiguous): one warp per line, lane k = partition k (P = 32,
//     m = nx/32); the reduced system is reduced once more to the E unknowns
//     and solved by parallel cyclic reduction over warp shuffles.
//   y and z lines (strided): one CTA per 16 adjacent lines, one thread per
//     (line, partition), threads of a partition adjacent; the reduced
//     system goes through shared memory and is applied as its tabulated
//     inverse (two rows per partition).
#include <algorithm>

#include "k_lines.cuh"
#include "tma.cuh"

// launch shapes (compile-time): x lines per warp iteration, y/z lines per CTA
#ifndef NSE_XL_NL
#define NSE_XL_NL 2
#endif
#ifndef NSE_YZ_LPB
#define NSE_YZ_LPB 16
#endif
// Register caps of the line kernels, as CTAs that must fit on an SM.  Left
// to itself the compiler gives the FP64 y/z kernel 60-80 registers (3-4
// CTAs of 256 threads) and the x kernel 76 (3 CTAs).  Measured at
// 256x192x256: a cap of 64 registers (1024 threads per SM) takes the FP64 y
// lines 0.247 -> 0.222 ms, the FP32 z lines 0.169 -> 0.149 and the x lines
// 0.194 -> 0.188 (FP32 0.144 -> 0.126) per step; the FP64 kernel with 16 rows
// per thread spills at 64 (z lines 0.219 -> 0.239) and keeps 768 threads, and
// the x kernel with 16 rows per lane (nx = 512) keeps 128 registers.
template <int NT, int MM, class R>
struct YZMinB {
  static constexpr int value = ((sizeof(R) == 8 && MM > 12) ? 768 : 1024) / NT > 0
                                   ? ((sizeof(R) == 8 && MM > 12) ? 768 : 1024) / NT
                                   : 1;
};

namespace nse {

namespace {

// ------------------------------------------------ rows of a folded line --
// Unknown t (0-based) of a line is reference row jr(t): t + 1, or for the
// x kernel (which rotates the periodic unknowns so lane 0 starts at the
// 16-byte aligned ghost position) n for t = 0 and t otherwise.
template <int DIR, int KIND>
struct FoldedLine {
  Dims d;
  GridDev g;
  const double* c1;
  LineArgs a;
  bool masked;
  int i, j, k;
  int n, nu;  // reference interior length, number of unknowns
  bool rot;

  __device__ Row ref(int r) const {
    if (masked) return line_row<DIR, KIND>(d, g, c1, a, i, j, k, r);
    const double alpha = a.dt * a.eta * 0.0 + 1.0;
    const double* D = DIR == 0 ? g.dx : (DIR == 1 ? g.dy : g.dz);
    const double* D12 = DIR == 0 ? g.dx12 : (DIR == 1 ? g.dy12 : g.dz12);
    if (KIND == LK_UL_U) return row_uy(a.beta, alpha, D12[r - 1], D12[r], D[r]);
    if (KIND == LK_UL_V) return row_vy(a.beta, alpha, D[r], D[r + 1], D12[r]);
    if (KIND == LK_CYC_VEL) return row_cyc(a.beta, alpha, D[r], D[r + 1], D12[r]);
    return row_T(a.beta, alpha, D[r - 1], D[r], D[r + 1], D12[r - 1], D12[r], a.l0, a.l0, a.l0,
                 a.r0);
  }
  __device__ int jr(int t) const { return rot ? (t == 0 ? n : t) : t + 1; }
  // coefficients of unknown t: A x(t-1) + B x(t) + C x(t+1) (indices mod nu
  // for periodic lines; A of the first and C of the last unknown are zero
  // for the others)
  __device__ void coef(int t, double& A, double& B, double& C) const {
    Row rw = ref(jr(t));
    A = rw.lo; B = rw.di; C = rw.up;
    if (KIND <= LK_UL_T) {
      if (t == 0) { if (KIND != LK_UL_V) B = B - A; A = 0.0; }
      if (t == nu - 1) { if (KIND != LK_UL_V) B = B - C; C = 0.0; }
    }
  }
};

template <int DIR, int KIND>
__device__ FoldedLine<DIR, KIND> folded_line(const Dims& d, const GridDev& g, const double* c1,
                                             const LineArgs& a, long id, bool masked,
                                             bool rot) {
  FoldedLine<DIR, KIND> L;
  L.d = d; L.g = g; L.c1 = c1; L.a = a; L.masked = masked; L.rot = rot;
  L.i = L.j = L.k = 0;
  if (masked) {
    if (DIR == 1) { L.i = 1 + (int)(id % d.nx); L.k = 1 + (int)(id / d.nx); }
    else if (DIR == 2) { L.i = 1 + (int)(id % d.nx); L.j = 1 + (int)(id / d.nx); }
    else { L.j = 1 + (int)(id % a.jtop); L.k = 1 + (int)(id / a.jtop); }
  }
  L.n = DIR == 0 ? d.nx : (DIR == 1 ? d.ny : d.nz);
  L.nu = KIND == LK_UL_V ? L.n - 1 : L.n;
  return L;
}

// interior rows s+1..e-1 of one partition: forward multipliers W, reciprocal
// pivots RB, super-diagonals CC and the responses P (to x(s) = 1) and Q (to
// x(e) = 1); element t of each array is at arr[t * step]
template <class Line>
__device__ void partition_rows(const Line& L, int s, int e, double* W, double* RB, double* CC,
                               double* PP, double* QQ, long step) {
  double A, B, C, Cprev = 0.0, beta = 1.0, pp = 0.0;
  for (int t = s + 1; t <= e - 1; ++t) {
    L.coef(t, A, B, C);
    double w = (t == s + 1) ? 0.0 : A / beta;
    beta = (t == s + 1) ? B : B - w * Cprev;
    pp = (t == s + 1) ? -A : -w * pp;  // forward sweep of the P response
    W[t * step] = w;
    RB[t * step] = 1.0 / beta;
    CC[t * step] = C;
    PP[t * step] = pp;
    Cprev = C;
  }
  // back substitution of P and Q (Q's right-hand side is -C(e-1) in row e-1)
  double pn = 0.0, qn = 0.0;
  for (int t = e - 1; t >= s + 1; --t) {
    double rb = RB[t * step], c = CC[t * step];
    double pv = (PP[t * step] - c * pn) * rb;
    double qv = ((t == e - 1 ? -c : 0.0) - c * qn) * rb;
    PP[t * step] = pv;
    QQ[t * step] = qv;
    pn = pv;
    qn = qv;
  }
}

}  // namespace

// ===================================================== y and z line tables
// layout (nu unknowns, P partitions; value v of partition k at
// T[5 nu + v P + k]):
//   W, RB, CC, PP, QQ [nu] | CF, AE, MU, NU, K1 [4], K2 [4], LAM, KAP, RDF,
//   LFR, UFR (per partition) | bg, rden, fold0, foldN
// The reduced system of the partition end unknowns F(k) (first row) and E(k)
// (last row) is solved as in the x tables: F eliminated, cyclic reduction
// over the partitions on E (strides 1, 2, ..., P/4; the non-periodic lines
// have zero couplings past their ends), the pair k, k ^ P/2 solved directly,
// then F from E.
enum {
  YT_CF = 0, YT_AE, YT_MU, YT_NU, YT_K1, YT_K2 = YT_K1 + 4, YT_LAM = YT_K2 + 4, YT_KAP, YT_RDF,
  YT_LFR, YT_UFR, YT_NV
};
__host__ __device__ size_t yz_table_stride(int nu, int P) {
  return 5 * (size_t)nu + (size_t)YT_NV * P + 4;
}

template <int DIR, int KIND>
__global__ void k_build_yz(Dims d, GridDev g, const double* c1, LineArgs a, const int* ids,
                           int count, int P, double* out) {
  const int line = blockIdx.x;
  const int lane = threadIdx.x;
  if (line >= count || threadIdx.x >= 32) return;  // warp 0 builds the table (P <= 32)
  const bool masked = ids != nullptr;
  auto L = folded_line<DIR, KIND>(d, g, c1, a, masked ? ids[line] : 0, masked, false);
  const int nu = L.nu;
  double* T = out + (size_t)line * yz_table_stride(nu, P);
  double *W = T, *RB = T + nu, *CC = T + 2 * nu, *PP = T + 3 * nu, *QQ = T + 4 * nu;
  double* V = T + 5 * nu;  // V[v * P + k]
  double* cst = V + YT_NV * P;
  const bool periodic = KIND >= LK_CYC_VEL;
  // lanes past P repeat partition P-1 (every lane takes part in the
  // shuffles; only lanes < P store)
  const bool own = lane < P;
  const int k = own ? lane : P - 1;
  const int s = (int)((long)k * nu / P), e = (int)((long)(k + 1) * nu / P) - 1;
  if (own) partition_rows(L, s, e, W, RB, CC, PP, QQ, 1);
  __syncwarp();
  double As, Bs, Cs, Ae, Be, Ce;
  L.coef(s, As, Bs, Cs);
  L.coef(e, Ae, Be, Ce);
  // F row: LF E(k-1) + DF F(k) + UF E(k); E row: LE F(k) + DE E(k) + UE F(k+1)
  // (A of the first and C of the last unknown are zero on non-periodic lines)
  const double LF = As, DF = Bs + Cs * PP[s + 1], UF = Cs * QQ[s + 1];
  const double LE = Ae * PP[e - 1], DE = Be + Ae * QQ[e - 1], UE = Ce;
  const unsigned FULL = 0xffffffffu;
  const int kp = (k + 1) % P;
  const double LF1 = __shfl_sync(FULL, LF, kp), DF1 = __shfl_sync(FULL, DF, kp);
  const double UF1 = __shfl_sync(FULL, UF, kp);
  // eliminate the F unknowns: al E(k-1) + be E(k) + ga E(k+1) = rho
  double al = -LE * LF / DF;
  double be = DE - LE * UF / DF - UE * LF1 / DF1;
  double ga = -UE * UF1 / DF1;
  if (own) {
    V[YT_CF * P + k] = Cs;
    V[YT_AE * P + k] = Ae;
    V[YT_MU * P + k] = -LE / DF;
    V[YT_NU * P + k] = -UE / DF1;
  }
  for (int lv = 0; lv < 4; ++lv) {
    if ((1 << lv) >= P / 2) {
      if (own) V[(YT_K1 + lv) * P + k] = V[(YT_K2 + lv) * P + k] = 0.0;
      continue;
    }
    const int sft = 1 << lv;
    const int km = (k - sft + P) % P, kq = (k + sft) % P;
    const double alm = __shfl_sync(FULL, al, km), bem = __shfl_sync(FULL, be, km);
    const double gam = __shfl_sync(FULL, ga, km);
    const double alp = __shfl_sync(FULL, al, kq), bep = __shfl_sync(FULL, be, kq);
    const double gap = __shfl_sync(FULL, ga, kq);
    const double k1 = -al / bem, k2 = -ga / bep;
    if (own) {
      V[(YT_K1 + lv) * P + k] = k1;
      V[(YT_K2 + lv) * P + k] = k2;
    }
    const double nal = k1 * alm, nga = k2 * gap, nbe = be + k1 * gam + k2 * alp;
    al = nal;
    ga = nga;
    be = nbe;
  }
  // rows k and k ^ P/2 now couple only each other
  const int kx = k ^ (P / 2);
  const double alx = __shfl_sync(FULL, al, kx), bex = __shfl_sync(FULL, be, kx);
  const double gax = __shfl_sync(FULL, ga, kx);
  const double a2 = al + ga;
  const double det = be * bex - a2 * (alx + gax);
  if (own) {
    V[YT_LAM * P + k] = bex / det;
    V[YT_KAP * P + k] = -a2 / det;
    V[YT_RDF * P + k] = 1.0 / DF;
    V[YT_LFR * P + k] = -LF / DF;
    V[YT_UFR * P + k] = -UF / DF;
  }
  if (lane == 0) {
    // fold constants: right-hand-side corrections of the first and last rows
    Row r1 = L.ref(1), rn = L.ref(nu);
    cst[0] = 0.0;
    cst[1] = 0.0;
    cst[2] = periodic ? 0.0 : r1.lo;
    cst[3] = periodic ? 0.0 : rn.up;
  }
}

// ========================================================== x line tables
// PL partitions per line (32: one warp per line; 16: one half-warp per line),
// values v = 0..XV-1 of partition k at [v * PL + k]
enum {
  XT_CF = 0, XT_AE, XT_MU, XT_NU, XT_K1, XT_K2 = XT_K1 + 4, XT_LAM = XT_K2 + 4, XT_KAP, XT_RDF,
  XT_LFR, XT_UFR, XT_ROW  // then 5 values per interior row: W, RB, CC, PP, QQ
};
__host__ __device__ constexpr int x_table_values(int M) { return XT_ROW + 5 * (M - 2); }
__host__ __device__ size_t x_table_stride(int M, int PL) {
  return (size_t)PL * (size_t)x_table_values(M);
}

template <int KIND, int PL>
__global__ void k_build_x(Dims d, GridDev g, const double* c1, LineArgs a, const int* ids,
                          int count, double* out) {
  const int line = blockIdx.x;
  const int k = threadIdx.x;  // blockDim = PL
  if (line >= count) return;
  const bool masked = ids != nullptr;
  auto L = folded_line<0, KIND>(d, g, c1, a, masked ? ids[line] : 0, masked, true);
  const int M = L.n / PL;
  double* T = out + (size_t)line * x_table_stride(M, PL);
  const int s = k * M, e = s + M - 1;
  // interior rows: values at T[(XT_ROW + 5 (r-1) + c) * PL + k], r = t - s;
  // partition_rows indexes arr[t * step], so shift the bases by -s rows
  double* rowb = T + XT_ROW * PL + k;
  const long step = 5 * PL;
  double* base = rowb - (long)(s + 1) * step;
  partition_rows(L, s, e, base, base + PL, base + 2 * PL, base + 3 * PL, base + 4 * PL, step);
  double As, Bs, Cs, Ae, Be, Ce;
  L.coef(s, As, Bs, Cs);
  L.coef(e, Ae, Be, Ce);
  const double p1 = base[(s + 1) * step + 3 * PL], q1 = base[(s + 1) * step + 4 * PL];
  const double pm = base[(e - 1) * step + 3 * PL], qm = base[(e - 1) * step + 4 * PL];
  // F row: LF E(k-1) + DF F(k) + UF E(k); E row: LE F(k) + DE E(k) + UE F(k+1)
  const double LF = As, DF = Bs + Cs * p1, UF = Cs * q1;
  const double LE = Ae * pm, DE = Be + Ae * qm, UE = Ce;
  const unsigned MASK = PL == 32 ? 0xffffffffu : 0xffffu;
  const int kp = (k + 1) & (PL - 1);
  const double LF1 = __shfl_sync(MASK, LF, kp, PL), DF1 = __shfl_sync(MASK, DF, kp, PL);
  const double UF1 = __shfl_sync(MASK, UF, kp, PL);
  // eliminate the F unknowns: al E(k-1) + be E(k) + ga E(k+1) = rho
  double al = -LE * LF / DF;
  double be = DE - LE * UF / DF - UE * LF1 / DF1;
  double ga = -UE * UF1 / DF1;
  T[XT_CF * PL + k] = Cs;
  T[XT_AE * PL + k] = Ae;
  T[XT_MU * PL + k] = -LE / DF;
  T[XT_NU * PL + k] = -UE / DF1;
  // parallel cyclic reduction over the PL lanes, strides 1, 2, ..., PL/4
  for (int lv = 0; (1 << lv) < PL / 2; ++lv) {
    const int sft = 1 << lv;
    const int km = (k - sft) & (PL - 1), kq = (k + sft) & (PL - 1);
    double alm = __shfl_sync(MASK, al, km, PL), bem = __shfl_sync(MASK, be, km, PL);
    double gam = __shfl_sync(MASK, ga, km, PL);
    double alp = __shfl_sync(MASK, al, kq, PL), bep = __shfl_sync(MASK, be, kq, PL);
    double gap = __shfl_sync(MASK, ga, kq, PL);
    double k1 = -al / bem, k2 = -ga / bep;
    T[(XT_K1 + lv) * PL + k] = k1;
    T[(XT_K2 + lv) * PL + k] = k2;
    double nal = k1 * alm, nga = k2 * gap, nbe = be + k1 * gam + k2 * alp;
    al = nal; ga = nga; be = nbe;
  }
  // rows k and k ^ PL/2 now couple only each other
  const int kx = k ^ (PL / 2);
  double alx = __shfl_sync(MASK, al, kx, PL), bex = __shfl_sync(MASK, be, kx, PL);
  double gax = __shfl_sync(MASK, ga, kx, PL);
  double a2 = al + ga;
  double det = be * bex - a2 * (alx + gax);
  T[XT_LAM * PL + k] = bex / det;
  T[XT_KAP * PL + k] = -a2 / det;
  T[XT_RDF * PL + k] = 1.0 / DF;
  T[XT_LFR * PL + k] = -LF / DF;
  T[XT_UFR * PL + k] = -UF / DF;
}

// =============================================================== solvers ==
// The solvers are templates on the storage type S of the line data and on
// the arithmetic and table type R (both double in the FP64 form; in the
// mixed-precision form S is float and R float, or double with the FP64
// tables).
template <class T> struct Vec2T;
template <> struct Vec2T<double> { using T = double2; };
template <> struct Vec2T<float> { using T = float2; };

// Products with the table entries that are close to 1 (the reciprocal pivots
// RB and the reduced-system factors LAM and RDF: near-identity systems,
// dt/Re/dx^2 ~ 1e-3).  The FP32 tables hold
// these entries as their deviation from 1, so a * v is formed as a + a * dv:
// a table rounded to FP32 then carries a relative error of 6e-8 of the
// deviation, not of 1, and the solve has no systematic bias of that size
// (which every step would repeat).  FP64 tables hold the values themselves.
__device__ __forceinline__ double mul1(double a, double v) { return a * v; }
__device__ __forceinline__ float mul1(float a, float dv) { return a + a * dv; }
// The line solvers' arithmetic with every rounding spelled out: products and
// sums the compiler may fuse differently in each template instantiation (the
// launch shapes schedule differently) are written as explicit fused or
// separately rounded operations, so every launch shape gives the same bits.
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
// mul1 with its rounding spelled out
__device__ __forceinline__ double xmul1(double a, double v) { return __dmul_rn(a, v); }
__device__ __forceinline__ float xmul1(float a, float dv) { return __fmaf_rn(a, dv, a); }

// interior Thomas on registers: g <- solution of the interior rows with
// zero end values; rows r = 1..m-2 of the partition, table rows at tb(r).
// Returns g(m-2) (taken inside the unrolled chain: selecting x[m-2] after
// the loop would make the compiler index x dynamically, in local memory).
template <int MM, class R, class TB>
__device__ __forceinline__ R interior_solve(R (&x)[MM], int m, const TB& tb) {
  R gp = x[1];
#pragma unroll
  for (int r = 2; r < MM - 1; ++r)
    if (r <= m - 2) { gp = xfma(-tb.w(r), gp, x[r]); x[r] = gp; }
  R gn = R(0), glast = R(0);
#pragma unroll
  for (int r = MM - 2; r >= 1; --r)
    if (r <= m - 2) {
      // gn is still 0 at r = m-2, so this is x(m-2) * rb there
      R v = xmul1(xfma(-tb.cc(r), gn, x[r]), tb.rb(r));
      if (r == m - 2) glast = v;
      x[r] = v;
      gn = v;
    }
  return glast;
}

// x lines: table of lane `lane`, values at p[v * PL + lane] (shared memory
// for the mask-free lines, global memory for a masked line)
template <class R, int PL>
struct XTab {
  const R* p;
  int lane;
  __device__ R v(int i) const { return p[i * PL + lane]; }
  __device__ R w(int r) const { return v(XT_ROW + 5 * (r - 1)); }
  __device__ R rb(int r) const { return v(XT_ROW + 5 * (r - 1) + 1); }
  __device__ R cc(int r) const { return v(XT_ROW + 5 * (r - 1) + 2); }
  __device__ R pp(int r) const { return v(XT_ROW + 5 * (r - 1) + 3); }
  __device__ R qq(int r) const { return v(XT_ROW + 5 * (r - 1) + 4); }
};

// NL lines per warp iteration share every table load (the table reads, not
// the line data, dominate the L1 traffic of this kernel)
// (with PL = 16 the two half-warps work on different lines).  STG (PL = 32,
// even M <= 8): a warp reads and writes its lines with consecutive lanes on
// consecutive 16-byte pairs (512 bytes per instruction) and moves them to and
// from its lanes' partitions through shared memory, with an XOR swizzle of
// the pair index so both sides stay free of bank conflicts; unstaged, each
// lane reads its own M values (pairs at a 16 M-byte lane stride, several
// sectors per request).
template <int M, int NL, bool MASKED, class S, class R, int PL, bool STG = false>
__global__ void __launch_bounds__(256, (M >= 16 ? 2 : 4)) k_xlines(Dims d, S* __restrict__ f, int jtop,
                                                const R* __restrict__ tab,
                                                const int* __restrict__ slots,
                                                const int* __restrict__ ids, int count) {
  using V2 = typename Vec2T<S>::T;
  static_assert(!STG || (PL == 32 && M % 2 == 0 && M <= 8), "staged x lines: PL 32, even M <= 8");
  constexpr int CH = STG ? 16 * M : 1;       // pairs of one line
  constexpr int WV = 128 / (int)sizeof(V2);  // pairs per 128-byte row of banks
  __shared__ V2 xsb[STG ? 8 * NL * CH : 1];  // [warp of the CTA][line][pair]
  V2* wb = xsb + (STG ? (threadIdx.x >> 5) * NL * CH : 0);
  // swizzled pair index (M = 6 reads conflict-free without it)
  auto sw = [](int c) { return (M % 4 == 0) ? (c ^ ((c / WV) % WV)) : c; };
  constexpr int NV = x_table_values(M);
  // FP32 tables (mixed form) carry the row coefficients of the increment
  // form after the factorisation values (see line_coef_values)
  constexpr bool INC = sizeof(R) == 4;
  constexpr int NVC = NV + (INC ? 3 * M : 0);
  constexpr int HW = 32 / PL;  // lines per warp at a time
  __shared__ R stab[MASKED ? 1 : NVC * PL];
  const int lane = threadIdx.x & (PL - 1), half = (threadIdx.x & 31) / PL;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  const int n = d.nx;
  const unsigned FULL = 0xffffffffu;
  if (!MASKED) {
    for (int t = threadIdx.x; t < NVC * PL; t += blockDim.x) stab[t] = __ldg(tab + t);
    __syncthreads();
  }
  const long nlines = MASKED ? count : (long)jtop * d.nz;
  const long ngroups = (nlines + NL * HW - 1) / (NL * HW);
  for (long gi = warp; gi < ngroups; gi += nwarps) {
    XTab<R, PL> tb;
    tb.lane = lane;
    // (masked pass: NL = 1, table of line gi*HW + half)
    tb.p = MASKED ? tab + (size_t)min(gi * HW + half, (long)count - 1) * (size_t)(NVC * PL)
                  : stab;
    S* line[NL];
    bool ok[NL];
    R x[NL][M];
#pragma unroll
    for (int q = 0; q < NL; ++q) {
      const long l = (gi * NL + q) * HW + half;
      long id = 0;
      ok[q] = l < nlines;
      if (ok[q]) {
        if (MASKED) id = ids[l];
        else { id = l; ok[q] = slots[l] < 0; }  // masked lines: their own pass
      }
      const int j = 1 + (int)(id % jtop), k = 1 + (int)(id / jtop);
      line[q] = f + d.P(0, j, k);
      if constexpr (STG) continue;
      // unknowns t = lane*M + r at positions t (t = 0 stands for x(n))
      if (ok[q]) {
        if (M % 2 == 0) {
          const V2* p2 = reinterpret_cast<const V2*>(line[q] + lane * M);
#pragma unroll
          for (int u = 0; u < M / 2; ++u) {
            V2 v = p2[u];
            x[q][2 * u] = (R)v.x;
            x[q][2 * u + 1] = (R)v.y;
          }
        } else {
#pragma unroll
          for (int r = 0; r < M; ++r) x[q][r] = (R)line[q][lane * M + r];
        }
        if (lane == 0) x[q][0] = (R)line[q][n];
      } else {
#pragma unroll
        for (int r = 0; r < M; ++r) x[q][r] = R(0);
      }
    }
    if constexpr (STG) {
      // each line's pairs through shared memory
#pragma unroll
      for (int q = 0; q < NL; ++q)
        if (ok[q]) {
          const V2* g2 = reinterpret_cast<const V2*>(line[q]);
          V2 tmp[M / 2];
#pragma unroll
          for (int u = 0; u < M / 2; ++u) tmp[u] = g2[lane + 32 * u];
#pragma unroll
          for (int u = 0; u < M / 2; ++u) wb[q * CH + sw(lane + 32 * u)] = tmp[u];
        }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        if (ok[q]) {
#pragma unroll
          for (int u = 0; u < M / 2; ++u) {
            const V2 v = wb[q * CH + sw((M / 2) * lane + u)];
            x[q][2 * u] = (R)v.x;
            x[q][2 * u + 1] = (R)v.y;
          }
          if (lane == 0) x[q][0] = (R)line[q][n];
        } else {
#pragma unroll
          for (int r = 0; r < M; ++r) x[q][r] = R(0);
        }
      }
      __syncwarp();  // the buffer is rewritten with the solution below
    }
    // increment form (FP32 tables): solve A y = r - A r and return r + y,
    // so the FP32 rounding of the solve scales with |y| ~ |(A - I) r|
    R xr[INC ? NL : 1][INC ? M : 1];
    if constexpr (INC) {
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const R left = __shfl_sync(FULL, x[q][M - 1], (lane - 1) & (PL - 1), PL);
        const R right = __shfl_sync(FULL, x[q][0], (lane + 1) & (PL - 1), PL);
#pragma unroll
        for (int r = 0; r < M; ++r) xr[q][r] = x[q][r];
#pragma unroll
        for (int r = 0; r < M; ++r) {
          const R xm = r == 0 ? left : xr[q][r > 0 ? r - 1 : 0];
          const R xp = r == M - 1 ? right : xr[q][r + 1 < M ? r + 1 : M - 1];
          x[q][r] = -xfma(tb.v(NV + 3 * r + 2), xp,
                          xfma(tb.v(NV + 3 * r + 1), xr[q][r], xmul(tb.v(NV + 3 * r), xm)));
        }
      }
    }
    // interior rows (Thomas with the tabulated factorisation)
    R gp[NL];
#pragma unroll
    for (int q = 0; q < NL; ++q) gp[q] = x[q][1];
#pragma unroll
    for (int r = 2; r <= M - 2; ++r) {
      const R w = tb.w(r);
#pragma unroll
      for (int q = 0; q < NL; ++q) { gp[q] = xfma(-w, gp[q], x[q][r]); x[q][r] = gp[q]; }
    }
#pragma unroll
    for (int r = M - 2; r >= 1; --r) {
      const R rb = tb.rb(r), cc = tb.cc(r);
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        R v = xmul1((r == M - 2) ? x[q][r] : xfma(-cc, gp[q], x[q][r]), rb);
        x[q][r] = v;
        gp[q] = v;
      }
    }
    // reduced system: eliminate F, cyclic reduction over the lanes on E
    R rhsF[NL], rho[NL];
    {
      const R cf = tb.v(XT_CF), ae = tb.v(XT_AE), mu = tb.v(XT_MU), nu = tb.v(XT_NU);
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        rhsF[q] = xfma(-cf, x[q][1], x[q][0]);
        const R rhsE = xfma(-ae, x[q][M - 2], x[q][M - 1]);
        rho[q] = xfma(nu, __shfl_sync(FULL, rhsF[q], (lane + 1) & (PL - 1), PL),
                      xfma(mu, rhsF[q], rhsE));
      }
    }
#pragma unroll
    for (int lv = 0; (1 << lv) < PL / 2; ++lv) {
      const int sft = 1 << lv;
      const R k1 = tb.v(XT_K1 + lv), k2 = tb.v(XT_K2 + lv);
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const R rm = __shfl_sync(FULL, rho[q], (lane - sft) & (PL - 1), PL);
        const R rp = __shfl_sync(FULL, rho[q], (lane + sft) & (PL - 1), PL);
        rho[q] = xfma(k2, rp, xfma(k1, rm, rho[q]));
      }
    }
    {
      const R lam = tb.v(XT_LAM), kap = tb.v(XT_KAP), rdf = tb.v(XT_RDF);
      const R lfr = tb.v(XT_LFR), ufr = tb.v(XT_UFR);
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const R E = xfma(kap, __shfl_sync(FULL, rho[q], lane ^ (PL / 2), PL),
                         xmul1(rho[q], lam));
        const R Em = __shfl_sync(FULL, E, (lane - 1) & (PL - 1), PL);
        const R F = xfma(ufr, E, xfma(lfr, Em, xmul1(rhsF[q], rdf)));
        rhsF[q] = F;
        rho[q] = E;
      }
    }
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
      const R pp = tb.pp(r), qq = tb.qq(r);
#pragma unroll
      for (int q = 0; q < NL; ++q) x[q][r] = xfma(qq, rho[q], xfma(pp, rhsF[q], x[q][r]));
    }
#pragma unroll
    for (int q = 0; q < NL; ++q) {
      x[q][0] = rhsF[q];
      x[q][M - 1] = rho[q];
      if constexpr (INC) {
#pragma unroll
        for (int r = 0; r < M; ++r) x[q][r] = xadd(xr[q][r], x[q][r]);
      }
      if (STG || !ok[q]) continue;
      if (M % 2 == 0) {
        V2* p2 = reinterpret_cast<V2*>(line[q] + lane * M);
#pragma unroll
        for (int u = 0; u < M / 2; ++u) {
          V2 v;
          v.x = (S)x[q][2 * u];
          v.y = (S)x[q][2 * u + 1];
          p2[u] = v;
        }
      } else {
#pragma unroll
        for (int r = 0; r < M; ++r) line[q][lane * M + r] = (S)x[q][r];
      }
      // position 0 received x(n), the value of the periodic ghost x(0)
      if (lane == 0) line[q][n] = (S)x[q][0];
    }
    if constexpr (STG) {
#pragma unroll
      for (int q = 0; q < NL; ++q)
        if (ok[q]) {
#pragma unroll
          for (int u = 0; u < M / 2; ++u) {
            V2 v;
            v.x = (S)x[q][2 * u];
            v.y = (S)x[q][2 * u + 1];
            wb[q * CH + sw((M / 2) * lane + u)] = v;
          }
        }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < NL; ++q)
        if (ok[q]) {
          V2* g2 = reinterpret_cast<V2*>(line[q]);
#pragma unroll
          for (int u = 0; u < M / 2; ++u) g2[lane + 32 * u] = wb[q * CH + sw(lane + 32 * u)];
          // position 0 received x(n), the value of the periodic ghost x(0)
          if (lane == 0) line[q][n] = (S)x[q][0];
        }
      __syncwarp();  // the next group's loads rewrite the buffer
    }
  }
}

// y / z lines: table values read through the cache (one table for all the
// mask-free lanes, so the loads broadcast)
template <class R>
struct YZTab {
  const R* T;
  int nu, s;
  __device__ R w(int r) const { return __ldg(T + s + r); }
  __device__ R rb(int r) const { return __ldg(T + nu + s + r); }
  __device__ R cc(int r) const { return __ldg(T + 2 * nu + s + r); }
  __device__ R pp(int r) const { return __ldg(T + 3 * nu + s + r); }
  __device__ R qq(int r) const { return __ldg(T + 4 * nu + s + r); }
};
// the same table through generic loads, for a table that may sit in shared
// memory (__ldg is a global-memory load: on a shared-memory address it fails
// with "operation not supported on global/shared address space")
template <class R>
struct YZTabAny {
  const R* T;
  int nu, s;
  __device__ R w(int r) const { return T[s + r]; }
  __device__ R rb(int r) const { return T[nu + s + r]; }
  __device__ R cc(int r) const { return T[2 * nu + s + r]; }
  __device__ R pp(int r) const { return T[3 * nu + s + r]; }
  __device__ R qq(int r) const { return T[4 * nu + s + r]; }
};
// the reduced-system values of partition k (YT_* of the table layout)
template <class R, bool LDG>
struct YZRed {
  const R* V;  // T + 5 nu
  int P, k;
  __device__ R v(int q) const { return LDG ? __ldg(V + q * P + k) : V[q * P + k]; }
};

// F and E of partition k for the LPB lines of a CTA (lane = line), from the
// partition's reduced right-hand sides rhsF (first row) and rhsE (last row):
// cyclic reduction over the P partitions through shared memory, xs two
// buffers of P x LPB values.  Every thread of the CTA calls it (it holds the
// CTA's barriers); lanes of invalid lines carry values nothing reads.
template <int P, int LPB, class R, class RV>
__device__ __forceinline__ void yz_reduced(R* xs, const RV& rv, int k, int lane, R rhsF, R rhsE,
                                           R& F, R& E) {
  R* b0 = xs;
  R* b1 = xs + P * LPB;
  b0[k * LPB + lane] = rhsF;
  __syncthreads();
  const R rhsF1 = b0[((k + 1) % P) * LPB + lane];
  R rho = xfma(rv.v(YT_NU), rhsF1, xfma(rv.v(YT_MU), rhsF, rhsE));
  R* cur = b1;
#pragma unroll
  for (int lv = 0; (1 << lv) < P / 2; ++lv) {
    const int sft = 1 << lv;
    cur[k * LPB + lane] = rho;
    __syncthreads();
    const R rm = cur[((k - sft + P) % P) * LPB + lane];
    const R rp = cur[((k + sft) % P) * LPB + lane];
    rho = xfma(rv.v(YT_K2 + lv), rp, xfma(rv.v(YT_K1 + lv), rm, rho));
    cur = (cur == b0) ? b1 : b0;
  }
  cur[k * LPB + lane] = rho;
  __syncthreads();
  const R rx = cur[(k ^ (P / 2)) * LPB + lane];
  E = xfma(rv.v(YT_KAP), rx, xmul1(rho, rv.v(YT_LAM)));
  cur = (cur == b0) ? b1 : b0;
  cur[k * LPB + lane] = E;
  __syncthreads();
  const R Em = cur[((k - 1 + P) % P) * LPB + lane];
  F = xfma(rv.v(YT_UFR), E, xfma(rv.v(YT_LFR), Em, xmul1(rhsF, rv.v(YT_RDF))));
}

// LPB lines per CTA (adjacent in x; 16 lines keep two CTAs resident per SM).
// The solution goes to `out` (type RO) when given, else back into f.
template <int DIR, int MM, int P, int LPB, class S, class R, class RO>
__global__ void __launch_bounds__(LPB * P, (YZMinB<LPB * P, MM, R>::value)) k_yzlines(Dims d, S* __restrict__ f,
                                                      RO* __restrict__ out, int nu, int nother,
                                                      const R* __restrict__ tab,
                                                      const int* __restrict__ slots,
                                                      const R* __restrict__ mtab, R ft, R fb,
                                                      int periodic) {
  // FP32 tables (mixed form): increment form, row coefficients after the
  // factorisation values (see line_coef_values)
  constexpr bool INC = sizeof(R) == 4;
  __shared__ R xs[2 * P * LPB];
  const int lane = threadIdx.x % LPB, k = threadIdx.x / LPB;
  const int i = 1 + blockIdx.x * LPB + lane;
  const int o = 1 + blockIdx.y;  // k of a y line, j of a z line
  const bool valid = i <= d.nx && o <= nother;
  const size_t stride = yz_table_stride(nu, P) + (INC ? 3 * (size_t)nu : 0);
  const R* T = tab;
  if (valid) {
    long lineid = (long)(i - 1) + (long)d.nx * (o - 1);
    int slot = slots[lineid];
    if (slot >= 0) T = mtab + (size_t)slot * stride;
  }
  const int s = (int)((long)k * nu / P), e = (int)((long)(k + 1) * nu / P) - 1;
  const int m = e - s + 1;
  const long es = DIR == 1 ? d.sx : d.sy;
  const long off = (DIR == 1 ? d.P(i, 0, o) : d.P(i, o, 0)) + (long)(s + 1) * es;
  const S* line = f + off;
  R x[MM];
  R xr[INC ? MM : 1];
  R xe = R(0), xer = R(0);
  YZTab<R> tb{T, nu, s};
  if (valid) {
    // right-hand-side folds of the boundary rows (zero for periodic lines)
    const R c0 = (!periodic && k == 0) ? __ldg(T + 5 * nu + YT_NV * P + 2) * ft : R(0);
    const R cN = (!periodic && k == P - 1) ? __ldg(T + 5 * nu + YT_NV * P + 3) * fb : R(0);
    // every load is issued up front (rows past m re-read row m-1); the
    // right-hand side of row m-1 is loaded once more on its own, so no
    // register is selected by the run-time m
#pragma unroll
    for (int r = 0; r < MM; ++r) x[r] = (R)line[(long)min(r, m - 1) * es];
    x[0] = x[0] - c0;
    xe = (R)line[(long)(m - 1) * es] - cN;
  }
  if constexpr (INC) {
    if (valid) {
      // right-hand side of A y = r - A r on this partition's rows s..e; the
      // neighbouring unknowns s-1 and e+1 are read from the line (they are
      // never folded: the folds touch unknowns 0 and nu-1 only, and every
      // partition has at least 3 rows)
      const R* CA = T + yz_table_stride(nu, P) + s;
      const R* CB = CA + nu;
      const R* CC = CB + nu;
      R left = R(0), right = R(0);
      if (k > 0) left = (R)line[-es];
      else if (periodic) left = (R)line[(long)(nu - 1) * es];
      if (k < P - 1) right = (R)line[(long)m * es];
      else if (periodic) right = (R)line[-(long)s * es];
#pragma unroll
      for (int r = 0; r < MM; ++r) xr[r] = (r == m - 1) ? xe : x[r];
      xer = xe;
#pragma unroll
      for (int r = 0; r < MM; ++r) {
        if (r < m) {
          const R xm = r == 0 ? left : xr[r > 0 ? r - 1 : 0];
          const R xc = r == m - 1 ? xe : xr[r];
          const R xp = r == m - 1 ? right : xr[r + 1 < MM ? r + 1 : MM - 1];
          const R sv = -xfma(__ldg(CC + r), xp, xfma(__ldg(CB + r), xc, xmul(__ldg(CA + r), xm)));
          if (r == m - 1) xe = sv;
          else x[r] = sv;
        }
      }
    }
  }
  const YZRed<R, true> rv{T + 5 * nu, P, k};
  R rhsF = R(0), rhsE = R(0);
  if (valid) {
    const R xe1 = interior_solve<MM>(x, m, tb);
    rhsF = xfma(-rv.v(YT_CF), x[1], x[0]);
    rhsE = xfma(-rv.v(YT_AE), xe1, xe);
  }
  R F, E;
  yz_reduced<P, LPB>(xs, rv, k, lane, rhsF, rhsE, F, E);
  if (!valid) return;
#pragma unroll
  for (int r = 1; r < MM; ++r) {
    if (r < m - 1) x[r] = xfma(tb.qq(r), E, xfma(tb.pp(r), F, x[r]));
    if (r == m - 1) x[r] = E;
  }
  x[0] = F;
  if constexpr (INC) {
#pragma unroll
    for (int r = 0; r < MM; ++r) x[r] = xadd(r == m - 1 ? xer : xr[r], x[r]);
  }
  RO* dst = out ? out + off : reinterpret_cast<RO*>(f + off);
#pragma unroll
  for (int r = 0; r < MM; ++r)
    if (r < m) dst[r * es] = (RO)x[r];
}

// ------------------------------------------ y / z lines through TMA tiles
// FP64 form.  A persistent CTA (16 lines x P partitions) walks tiles of 16
// x-adjacent lines: the tile's nu rows (16 x nu doubles) come into shared
// memory by one TMA copy (tensor map over the padded field, box 16 x nu at
// x = 16 t, so the box starts 16-byte aligned: tile t covers i = 16t..16t+15,
// the ghost columns i = 0 and nx+1 are carried along unchanged and columns
// past nx+1 fall outside the map), the solution is written back into the
// tile and leaves by one TMA store.  Two tile buffers: the next tile's load
// is in flight while this one is solved.  The mask-free table sits in shared
// memory; a line that touches the mask reads its own table from global
// memory.  The arithmetic is k_yzlines' (same values).
__host__ __device__ __forceinline__ size_t yzt_tile_bytes(int nu) {
  return (((size_t)nu * 16 * 8) + 127) & ~(size_t)127;
}
// set when a wait on a tile copy gave up (read by the host: line_wait_error)
__device__ int g_line_wait_err = 0;

template <int DIR, int MM, int P>
__global__ void __launch_bounds__(16 * P, 2)
    k_yzlines_tma(const __grid_constant__ CUtensorMap tm, Dims d, int nu, int nother, int ntx,
                  const double* __restrict__ tab, const int* __restrict__ slots,
                  const double* __restrict__ mtab, double ft, double fb, int periodic) {
  constexpr int LPB = 16;
  extern __shared__ __align__(128) unsigned char ysm[];
  const size_t tb_bytes = yzt_tile_bytes(nu);
  double* buf0 = reinterpret_cast<double*>(ysm);
  double* buf1 = reinterpret_cast<double*>(ysm + tb_bytes);
  double* xs = reinterpret_cast<double*>(ysm + 2 * tb_bytes);  // [2][P][LPB]
  const size_t stride = yz_table_stride(nu, P);
  double* stab = xs + 2 * P * LPB;  // mask-free table
  uint64_t* bar = reinterpret_cast<uint64_t*>(stab + ((stride + 1) & ~(size_t)1));
  const int lane = threadIdx.x % LPB, k = threadIdx.x / LPB;
  const long ntiles = (long)ntx * nother;
  const unsigned tile_tx = (unsigned)nu * LPB * 8;
  for (size_t t = threadIdx.x; t < stride; t += blockDim.x) stab[t] = __ldg(tab + t);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  // the copies need the tensor map 64-byte aligned and the tile buffers
  // 128-byte aligned in shared memory; a launch that finds otherwise records
  // the error and copies nothing (its tiles are then left as they are)
  const bool aligned = ((reinterpret_cast<uintptr_t>(&tm) & 63) == 0) &&
                       ((smem_u32(buf0) & 127) == 0) && ((smem_u32(buf1) & 127) == 0) &&
                       ((smem_u32(bar) & 7) == 0);
  if (!aligned) {
    if (threadIdx.x == 0) atomicExch(&g_line_wait_err, 2);
    return;
  }
  __syncthreads();
  long q = blockIdx.x;
  if (threadIdx.x == 0 && q < ntiles) {
    mbar_expect_tx(&bar[0], tile_tx);
    const int x0 = (int)(q % ntx) * LPB, o = 1 + (int)(q / ntx);
    if (DIR == 1) tma_load_3d(buf0, &tm, x0, 1, o, &bar[0]);
    else tma_load_3d(buf0, &tm, x0, o, 1, &bar[0]);
  }
  const int s = (int)((long)k * nu / P), e = (int)((long)(k + 1) * nu / P) - 1;
  const int m = e - s + 1;
  for (int it = 0; q < ntiles; q += gridDim.x, ++it) {
    double* cur = (it & 1) ? buf1 : buf0;
    double* nxt = (it & 1) ? buf0 : buf1;
    const long qn = q + gridDim.x;
    if (threadIdx.x == 0 && qn < ntiles) {
      tma_store_wait_read();  // the previous tile's store has read its buffer
      uint64_t* nb = &bar[(it + 1) & 1];
      mbar_expect_tx(nb, tile_tx);
      const int x0 = (int)(qn % ntx) * LPB, o = 1 + (int)(qn / ntx);
      if (DIR == 1) tma_load_3d(nxt, &tm, x0, 1, o, nb);
      else tma_load_3d(nxt, &tm, x0, o, 1, nb);
    }
    if (!tma_wait(&bar[it & 1], (unsigned)((it >> 1) & 1)) && threadIdx.x == 0)
      atomicExch(&g_line_wait_err, 1);
    const int i = (int)(q % ntx) * LPB + lane;
    const int o = 1 + (int)(q / ntx);
    const bool valid = i >= 1 && i <= d.nx;
    const double* T = stab;
    if (valid) {
      const long lineid = (long)(i - 1) + (long)d.nx * (o - 1);
      const int slot = slots[lineid];
      if (slot >= 0) T = mtab + (size_t)slot * stride;
    }
    YZTabAny<double> tb{T, nu, s};
    double x[MM];
    const double* col = cur + (size_t)s * LPB + lane;
    const double c0 = (!periodic && k == 0) ? T[5 * nu + YT_NV * P + 2] * ft : 0.0;
    const double cN = (!periodic && k == P - 1) ? T[5 * nu + YT_NV * P + 3] * fb : 0.0;
#pragma unroll
    for (int r = 0; r < MM; ++r) x[r] = col[(size_t)min(r, m - 1) * LPB];
    x[0] = x[0] - c0;
    const double xe = col[(size_t)(m - 1) * LPB] - cN;
    const double xe1 = interior_solve<MM>(x, m, tb);
    const YZRed<double, false> rv{T + 5 * nu, P, k};
    const double rhsF = xfma(-rv.v(YT_CF), x[1], x[0]);
    const double rhsE = xfma(-rv.v(YT_AE), xe1, xe);
    double F, E;
    yz_reduced<P, LPB>(xs, rv, k, lane, rhsF, rhsE, F, E);
#pragma unroll
    for (int r = 1; r < MM; ++r) {
      if (r < m - 1) x[r] = xfma(tb.qq(r), E, xfma(tb.pp(r), F, x[r]));
      if (r == m - 1) x[r] = E;
    }
    x[0] = F;
    double* dst = cur + (size_t)s * LPB + lane;
    if (valid) {
#pragma unroll
      for (int r = 0; r < MM; ++r)
        if (r < m) dst[(size_t)r * LPB] = x[r];
    }
    fence_async_smem();
    __syncthreads();  // the tile is complete; the exchange buffers may be rewritten
    if (threadIdx.x == 0) {
      const int x0 = (int)(q % ntx) * LPB;
      if (DIR == 1) tma_store_3d(&tm, x0, 1, o, cur);
      else tma_store_3d(&tm, x0, o, 1, cur);
      tma_store_commit();
    }
  }
  if (threadIdx.x == 0) tma_store_wait_all();
}

// ============================================================== launchers
// partitions of a y/z line of nu unknowns: the fewest of 4, 8, 16 that
// leave at most 16 rows each (rows per thread are registers)
int yz_partitions(int nu) { return nu <= 64 ? 4 : (nu <= 128 ? 8 : (nu <= 256 ? 16 : 32)); }
static int yz_rows(int nu) {
  int P = yz_partitions(nu);
  int m = (nu + P - 1) / P;
  return m <= 8 ? 8 : (m <= 12 ? 12 : 16);
}
// partitions per line (PL) and rows per partition (M) of the x kernel;
// M = 0 when the x kernel does not apply
static void x_shape(int nx, int& M, int& PL) {
  M = 0;
  PL = 32;
  if (nx % 32 == 0) {
    const int m = nx / 32;
    if (m == 3 || m == 4 || m == 5 || m == 6 || m == 8 || m == 16) { M = m; return; }
  }
  if (nx % 16 == 0) {
    const int m = nx / 16;
    if (m == 3 || m == 4 || m == 5) { M = m; PL = 16; }
  }
}
int x_rows_per_lane(int nx) {
  int M, PL;
  x_shape(nx, M, PL);
  return M;
}
// the y/z kernel needs at least 3 and at most 16 rows per partition
static bool yz_ok(int nu) {
  return nu / yz_partitions(nu) >= 3 && (nu + yz_partitions(nu) - 1) / yz_partitions(nu) <= 16;
}
bool part_lines_supported(const Dims& d) {
  return x_rows_per_lane(d.nx) > 0 && yz_ok(d.ny - 1) && yz_ok(d.ny) && yz_ok(d.nz);
}
size_t part_table_stride(int dir, int kind, const Dims& d) {
  if (dir == 0) {
    int M, PL;
    x_shape(d.nx, M, PL);
    return x_table_stride(M, PL);
  }
  int nu = dir == 1 ? (kind == LK_UL_V ? d.ny - 1 : d.ny) : d.nz;
  return yz_table_stride(nu, yz_partitions(nu));
}

// tables of the lines `ids` (count of them), or with ids == nullptr the one
// table of the mask-free lines
void launch_part_tables(int dir, int kind, const Dims& d, const GridDev& g, const double* c1,
                        const LineArgs& a, const int* ids, int count, double* out,
                        cudaStream_t s) {
  if (count <= 0) return;
  count_launch();
  if (dir == 0) {
    int M, PL;
    x_shape(d.nx, M, PL);
    if (PL == 32) {
      if (kind == LK_CYC_VEL) k_build_x<LK_CYC_VEL, 32><<<count, 32, 0, s>>>(d, g, c1, a, ids, count, out);
      else k_build_x<LK_CYC_T, 32><<<count, 32, 0, s>>>(d, g, c1, a, ids, count, out);
    } else {
      if (kind == LK_CYC_VEL) k_build_x<LK_CYC_VEL, 16><<<count, 16, 0, s>>>(d, g, c1, a, ids, count, out);
      else k_build_x<LK_CYC_T, 16><<<count, 16, 0, s>>>(d, g, c1, a, ids, count, out);
    }
    return;
  }
  int nu = dir == 1 ? (kind == LK_UL_V ? d.ny - 1 : d.ny) : d.nz;
  int P = yz_partitions(nu);
  const int nt = P <= 16 ? 32 : 2 * P;  // one thread per partition and per inverse column
  if (dir == 1) {
    if (kind == LK_UL_U) k_build_yz<1, LK_UL_U><<<count, nt, 0, s>>>(d, g, c1, a, ids, count, P, out);
    else if (kind == LK_UL_V) k_build_yz<1, LK_UL_V><<<count, nt, 0, s>>>(d, g, c1, a, ids, count, P, out);
    else k_build_yz<1, LK_UL_T><<<count, nt, 0, s>>>(d, g, c1, a, ids, count, P, out);
  } else {
    if (kind == LK_CYC_VEL) k_build_yz<2, LK_CYC_VEL><<<count, nt, 0, s>>>(d, g, c1, a, ids, count, P, out);
    else k_build_yz<2, LK_CYC_T><<<count, nt, 0, s>>>(d, g, c1, a, ids, count, P, out);
  }
}

static int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
    if (cached <= 0) cached = 148;
  }
  return cached;
}

template <int M, class S, class R, int PL = 32, int NLW = 0, bool STG = false>
static void go_x(const Dims& d, S* f, int jtop, const R* tab, const int* slots, const int* ids,
                 int nmasked, const R* mtab, cudaStream_t s) {
  const int sms = sm_count();
  constexpr int NL = NLW > 0 ? NLW : (M <= 8 ? NSE_XL_NL : 2);
  constexpr int HW = 32 / PL;
  long nlines = (long)jtop * d.nz;
  long per_blk = 8L * NL * HW;
  long blocks = std::min<long>((long)sms * 8, (nlines + per_blk - 1) / per_blk);
  count_launch();
  k_xlines<M, NL, false, S, R, PL, STG><<<(unsigned)blocks, 256, 0, s>>>(d, f, jtop, tab, slots,
                                                                          nullptr, 0);
  if (nmasked > 0) {
    long mb = std::min<long>((long)sms * 8, (nmasked + 8 * HW - 1) / (8 * HW));
    count_launch();
    // (the pass over the few masked lines keeps the direct loads: staged, its
    // per-line table pointer pushes it past the 64-register cap)
    k_xlines<M, 1, true, S, R, PL><<<(unsigned)mb, 256, 0, s>>>(d, f, jtop, mtab, slots, ids,
                                                                nmasked);
  }
}

// the TMA tile path of the FP64 y/z lines; false when it does not apply or
// the tensor map cannot be made (the caller then launches k_yzlines)
static bool yz_tma_lines(int dir, const Dims& d, double* f, int nu, int P, int MM, int nother,
                         const double* tab, const int* slots, const double* mtab, double ft,
                         double fb, bool periodic, cudaStream_t s) {
  CUtensorMap tm;
  const long p1 = (long)(d.nx + 2) * 8, p2 = p1 * (d.ny + 2);
  if (p1 % 16 != 0 || ((uintptr_t)f & 15) != 0) return false;
  const bool ok = dir == 1 ? tma_encode_3d(&tm, f, true, d.nx + 2, d.ny + 2, d.nz + 2, p1, p2, 16,
                                           nu, 1)
                           : tma_encode_3d(&tm, f, true, d.nx + 2, d.ny + 2, d.nz + 2, p1, p2, 16,
                                           1, nu);
  if (!ok) return false;
  const int ntx = (d.nx + 2 + 15) / 16;
  const long ntiles = (long)ntx * nother;
  const size_t stride = yz_table_stride(nu, P);
  const size_t smem = 2 * yzt_tile_bytes(nu) + (size_t)2 * P * 16 * 8 +
                      ((stride + 1) & ~(size_t)1) * 8 + 16;
  const int grid = (int)std::min<long>(ntiles, 2L * sm_count());
  const int per = periodic ? 1 : 0;
#define NSE_YZT(DIR_, MM_, P_)                                                                \
  {                                                                                           \
    auto kern = k_yzlines_tma<DIR_, MM_, P_>;                                                 \
    cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                         (int)smem);                                                          \
    count_launch();                                                                           \
    kern<<<grid, 16 * P_, smem, s>>>(tm, d, nu, nother, ntx, tab, slots, mtab, ft, fb, per);  \
  }
#define NSE_YZT_MM(DIR_, P_)                 \
  if (MM == 8) NSE_YZT(DIR_, 8, P_)          \
  else if (MM == 12) NSE_YZT(DIR_, 12, P_)   \
  else NSE_YZT(DIR_, 16, P_)
  if (dir == 1) {
    if (P == 16) { NSE_YZT_MM(1, 16) } else if (P == 8) { NSE_YZT_MM(1, 8) } else { NSE_YZT_MM(1, 4) }
  } else {
    if (P == 16) { NSE_YZT_MM(2, 16) } else if (P == 8) { NSE_YZT_MM(2, 8) } else { NSE_YZT_MM(2, 4) }
  }
#undef NSE_YZT_MM
#undef NSE_YZT
  return true;
}

int line_wait_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_line_wait_err, sizeof(int)) != cudaSuccess) return 0;
  if (v) {
    const int z = 0;
    cudaMemcpyToSymbol(g_line_wait_err, &z, sizeof(int));
  }
  return v;
}

template <int LPB, class S, class R, class RO>
static void yz_launch(int dir, const Dims& d, S* f, RO* out, int nu, int P, int MM, int nother,
                      const R* tab, const int* slots, const R* mtab, R ft, R fb, bool per,
                      cudaStream_t s) {
  dim3 grid((d.nx + LPB - 1) / LPB, nother);
  const int periodic = per ? 1 : 0;
  count_launch();
#define NSE_YZ(DIR_, MM_, P_)                                                               \
  k_yzlines<DIR_, MM_, P_, LPB, S, R, RO><<<grid, LPB * P_, 0, s>>>(                        \
      d, f, out, nu, nother, tab, slots, mtab, ft, fb, periodic)
#define NSE_YZ_MM(DIR_, P_)                \
  if (MM == 8) NSE_YZ(DIR_, 8, P_);        \
  else if (MM == 12) NSE_YZ(DIR_, 12, P_); \
  else NSE_YZ(DIR_, 16, P_);
  if (dir == 1) {
    if (P == 32) { NSE_YZ_MM(1, 32) } else if (P == 16) { NSE_YZ_MM(1, 16) }
    else if (P == 8) { NSE_YZ_MM(1, 8) } else { NSE_YZ_MM(1, 4) }
  } else {
    if (P == 32) { NSE_YZ_MM(2, 32) } else if (P == 16) { NSE_YZ_MM(2, 16) }
    else if (P == 8) { NSE_YZ_MM(2, 8) } else { NSE_YZ_MM(2, 4) }
  }
#undef NSE_YZ_MM
#undef NSE_YZ
}

template <class S, class R, class RO>
static void lines_part(int dir, int kind, const Dims& d, S* f, RO* out, const LineArgs& a,
                       const R* tab, const int* slots, const int* ids, int nmasked,
                       const R* mtab, cudaStream_t s) {
  if (dir == 0) {
    int M, PL;
    x_shape(d.nx, M, PL);
    if (PL == 16) {
      if (M == 3) go_x<3, S, R, 16>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
      else if (M == 4) go_x<4, S, R, 16>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
      else go_x<5, S, R, 16>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
      return;
    }
    // one line per warp iteration is the autotuner's alternative to two, and
    // the staged loads (3: two lines, 4: one line) for even M <= 8 (same values)
    if constexpr (sizeof(S) == sizeof(R)) {
      if (a.xnl == 3 || a.xnl == 4) {
        const bool two = a.xnl == 3;
        switch (M) {
          case 4:
            if (two) go_x<4, S, R, 32, 2, true>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
            else go_x<4, S, R, 32, 1, true>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
            return;
          case 6:
            if (two) go_x<6, S, R, 32, 2, true>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
            else go_x<6, S, R, 32, 1, true>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
            return;
          case 8:
            if (two) go_x<8, S, R, 32, 2, true>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
            else go_x<8, S, R, 32, 1, true>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s);
            return;
          default: break;
        }
      }
      if (a.xnl == 1) {
        switch (M) {
          case 3: go_x<3, S, R, 32, 1>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); return;
          case 4: go_x<4, S, R, 32, 1>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); return;
          case 5: go_x<5, S, R, 32, 1>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); return;
          case 6: go_x<6, S, R, 32, 1>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); return;
          case 8: go_x<8, S, R, 32, 1>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); return;
          default: break;
        }
      }
    }
    switch (M) {
      case 3: go_x<3>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); break;
      case 4: go_x<4>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); break;
      case 5: go_x<5>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); break;
      case 6: go_x<6>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); break;
      case 8: go_x<8>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); break;
      default: go_x<16>(d, f, a.jtop, tab, slots, ids, nmasked, mtab, s); break;
    }
    return;
  }
  int nu = dir == 1 ? (kind == LK_UL_V ? d.ny - 1 : d.ny) : d.nz;
  int P = yz_partitions(nu);
  int MM = yz_rows(nu);
  int nother = dir == 1 ? d.nz : a.jtop;
  if constexpr (sizeof(S) == 8 && sizeof(R) == 8 && sizeof(RO) == 8) {
    if (a.yzshape == 2 && !out && P <= 16 &&
        yz_tma_lines(dir, d, reinterpret_cast<double*>(f), nu, P, MM, nother,
                     reinterpret_cast<const double*>(tab), slots,
                     reinterpret_cast<const double*>(mtab), a.ft, a.fb, kind >= LK_CYC_VEL, s))
      return;
  }
  // lines per CTA: 16, or the autotuner's alternatives 8 and 32 (same values)
  // for the uniform storage/arithmetic types
  constexpr bool uni = sizeof(S) == sizeof(R) && sizeof(R) == sizeof(RO);
  if constexpr (uni) {
    if (a.yzshape == 1 && !out) {
      yz_launch<8>(dir, d, f, out, nu, P, MM, nother, tab, slots, mtab, (R)a.ft, (R)a.fb,
                   kind >= LK_CYC_VEL, s);
      return;
    }
    if (a.yzshape == 3 && !out) {
      yz_launch<32>(dir, d, f, out, nu, P, MM, nother, tab, slots, mtab, (R)a.ft, (R)a.fb,
                    kind >= LK_CYC_VEL, s);
      return;
    }
  }
  yz_launch<NSE_YZ_LPB>(dir, d, f, out, nu, P, MM, nother, tab, slots, mtab, (R)a.ft, (R)a.fb,
                        kind >= LK_CYC_VEL, s);
}

void launch_lines_part(int dir, int kind, const Dims& d, double* f, const LineArgs& a,
                       const double* tab, const int* slots, const int* ids, int nmasked,
                       const double* mtab, cudaStream_t s) {
  lines_part<double, double, double>(dir, kind, d, f, nullptr, a, tab, slots, ids, nmasked,
                                     mtab, s);
}

// mixed-precision form: FP32 line data with FP32 arithmetic and tables, or
// (tab64/mtab64 given) FP64 arithmetic and tables; a y or z solve may write
// its result to a separate FP64 array (`out`, the temperature's last sweep)
void launch_lines_part_f32(int dir, int kind, const Dims& d, float* f, double* out,
                           const LineArgs& a, const float* tab, const int* slots,
                           const int* ids, int nmasked, const float* mtab,
                           const double* tab64, const double* mtab64, cudaStream_t s) {
  const bool to64 = out && dir != 0;
  if (tab64) {
    if (to64)
      lines_part<float, double, double>(dir, kind, d, f, out, a, tab64, slots, ids, nmasked,
                                        mtab64, s);
    else
      lines_part<float, double, float>(dir, kind, d, f, nullptr, a, tab64, slots, ids, nmasked,
                                       mtab64, s);
  } else if (to64) {
    lines_part<float, float, double>(dir, kind, d, f, out, a, tab, slots, ids, nmasked, mtab, s);
  } else {
    lines_part<float, float, float>(dir, kind, d, f, nullptr, a, tab, slots, ids, nmasked, mtab,
                                    s);
  }
}

// the FP64 tables rounded to FP32 for the mixed-precision form
__global__ void k_round_table(const double* __restrict__ in, float* __restrict__ out, long n) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x)
    out[t] = (float)in[t];
}
void launch_round_table(const double* in, float* out, long n, cudaStream_t s) {
  if (n <= 0) return;
  count_launch();
  k_round_table<<<(unsigned)std::min<long>((n + 255) / 256, 4096), 256, 0, s>>>(in, out, n);
}

// FP32 line tables of the mixed form.  Each FP32 table is the FP64 table
// rounded, with the entries close to 1 stored as their deviation from 1 (see
// mul1: x tables RB of every row, LAM, RDF; y/z tables RB of every unknown,
// LAM and RDF of every partition), followed by the row coefficients of the
// increment form: A (to the previous unknown), B - 1, C (to the next) of
// every unknown, FP64 values rounded once.  x tables: value NV + 3r + c of
// lane k (unknown k*M + r) at [(NV + 3r + c) * PL + k]; y/z tables:
// [stride64 + c*nu + t].
size_t part_table_stride32(int dir, int kind, const Dims& d) {
  int nu = dir == 0 ? d.nx : (dir == 1 ? (kind == LK_UL_V ? d.ny - 1 : d.ny) : d.nz);
  return part_table_stride(dir, kind, d) + 3 * (size_t)nu;
}

__global__ void k_round_line_table(const double* __restrict__ in, float* __restrict__ out,
                                   long n, long stride64, long stride32, int PL, int nu, int P) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const long o = t % stride64, line = t / stride64;
    bool near1;
    if (PL > 0) {
      const int v = (int)(o / PL);
      near1 = v == XT_LAM || v == XT_RDF || (v >= XT_ROW && (v - XT_ROW) % 5 == 1);
    } else {
      const long vl = 5L * nu + (long)YT_LAM * P, vr = 5L * nu + (long)YT_RDF * P;
      near1 = (o >= nu && o < 2L * nu) || (o >= vl && o < vl + P) || (o >= vr && o < vr + P);
    }
    out[line * stride32 + o] = near1 ? (float)(in[t] - 1.0) : (float)in[t];
  }
}

template <int DIR, int KIND>
__global__ void k_build_coef(Dims d, GridDev g, const double* c1, LineArgs a, const int* ids,
                             int count, float* out, long stride32, long off, int PL, int M,
                             int NV) {
  const int line = blockIdx.x;
  if (line >= count) return;
  const bool masked = ids != nullptr;
  auto L = folded_line<DIR, KIND>(d, g, c1, a, masked ? ids[line] : 0, masked, DIR == 0);
  float* T = out + (size_t)line * stride32;
  for (int t = threadIdx.x; t < L.nu; t += blockDim.x) {
    double A, B, C;
    L.coef(t, A, B, C);
    const double v[3] = {A, B - 1.0, C};
    for (int c = 0; c < 3; ++c) {
      if (DIR == 0) T[(NV + 3 * (t % M) + c) * PL + t / M] = (float)v[c];
      else T[off + (long)c * L.nu + t] = (float)v[c];
    }
  }
}

void launch_round_line_table(int dir, int kind, const Dims& d, const GridDev& g,
                             const double* c1, const LineArgs& a, const int* ids,
                             const double* in, float* out, long ntables, cudaStream_t s) {
  if (ntables <= 0) return;
  const long stride64 = (long)part_table_stride(dir, kind, d);
  const long stride32 = (long)part_table_stride32(dir, kind, d);
  int PL = 0, M = 0, nu = 0, P = 0;
  if (dir == 0) {
    x_shape(d.nx, M, PL);
  } else {
    nu = dir == 1 ? (kind == LK_UL_V ? d.ny - 1 : d.ny) : d.nz;
    P = yz_partitions(nu);
  }
  const long n = stride64 * ntables;
  count_launch();
  k_round_line_table<<<(unsigned)std::min<long>((n + 255) / 256, 4096), 256, 0, s>>>(
      in, out, n, stride64, stride32, PL, nu, P);
  const int NV = dir == 0 ? x_table_values(M) : 0;
  count_launch();
#define NSE_COEF(DIR_, KIND_)                                                              \
  k_build_coef<DIR_, KIND_><<<(unsigned)ntables, 128, 0, s>>>(d, g, c1, a, ids, (int)ntables, \
                                                              out, stride32, stride64, PL, M, NV)
  if (dir == 0) {
    if (kind == LK_CYC_VEL) NSE_COEF(0, LK_CYC_VEL);
    else NSE_COEF(0, LK_CYC_T);
  } else if (dir == 1) {
    if (kind == LK_UL_U) NSE_COEF(1, LK_UL_U);
    else if (kind == LK_UL_V) NSE_COEF(1, LK_UL_V);
    else NSE_COEF(1, LK_UL_T);
  } else {
    if (kind == LK_CYC_VEL) NSE_COEF(2, LK_CYC_VEL);
    else NSE_COEF(2, LK_CYC_T);
  }
#undef NSE_COEF
}

}  // namespace nse
