// k_lines.cuh -- tiled ADI line solver of the resident step.
//
// A CTA is one warp and owns 32 parallel grid lines.  The 32 lines are
// loaded into shared memory with coalesced accesses (for y and z lines the
// 32 lines are adjacent in x; x lines are contiguous and are loaded row by
// row), each thread then runs the reference's sequential elimination on its
// own line out of shared memory, and the tile is stored back.  The only
// global traffic is one read and one write of the field.
//
// Lines on which the penalisation mask is zero (almost all of them) have
// the same matrix, so their recurrence coefficients come from per-row
// tables built once per configuration (k_line_tables) with the same
// arithmetic as the per-line path; lines that touch the mask compute their
// rows on the fly and keep the coefficient sweep in a global scratch field.
//
// EXACT = true keeps every division of the reference (bit-identical to the
// per-line kernels and the oracle when built without FMA contraction);
// EXACT = false multiplies by tabulated reciprocals on mask-free lines.
#pragma once
#include "common.cuh"

namespace nse {

enum LineKind { LK_UL_U = 0, LK_UL_V = 1, LK_UL_T = 2, LK_CYC_VEL = 3, LK_CYC_T = 4 };

struct Row {
  double lo, di, up;
};

// implicit_uy rows (nse_dominik.f:1524-1529)
__device__ __forceinline__ Row row_uy(double beta, double alpha, double dy12m, double dy12c,
                                      double dyc) {
  Row r;
  r.lo = -beta / alpha / dy12m / dyc;
  r.di = 1.0 + beta / alpha * (1.0 / dy12c + 1.0 / dy12m) / dyc;
  r.up = -beta / alpha / dy12c / dyc;
  return r;
}
// implicit_vy rows (:1605-1610)
__device__ __forceinline__ Row row_vy(double beta, double alpha, double dyc, double dyp,
                                      double dy12c) {
  Row r;
  r.lo = -beta / alpha / dyc / dy12c;
  r.di = 1.0 + beta / alpha * (1.0 / dyp + 1.0 / dyc) / dy12c;
  r.up = -beta / alpha / dyp / dy12c;
  return r;
}
// implicit_solver rows (periodic_implicit.f:28-33)
__device__ __forceinline__ Row row_cyc(double beta, double alpha, double dc, double dp,
                                       double d12c) {
  Row r;
  r.lo = -beta / alpha / dc / d12c;
  r.di = 1.0 + beta / alpha * (1.0 / dp + 1.0 / dc) / d12c;
  r.up = -beta / alpha / dp / d12c;
  return r;
}
// implicit_Ty / implicit_Tx harmonic-conductance rows (:1752-1770, :1811-1829)
__device__ __forceinline__ Row row_T(double beta, double alpha, double dm, double dc,
                                     double dp, double d12m, double d12c, double llm,
                                     double llc, double llp, double rrc) {
  double Hm = (dc + dm) / (dc / llc + dm / llm);
  double Hp = (dp + dc) / (dp / llp + dc / llc);
  Row r;
  r.lo = -beta / alpha * Hm / d12m / dc / rrc;
  r.di = 1.0 + beta / alpha * (Hp / d12c / dc + Hm / d12m / dc) / rrc;
  r.up = -beta / alpha * Hp / d12c / dc / rrc;
  return r;
}

// asynchronous 8-byte global -> shared copy (cp.async, sm_80+): the whole
// tile is put in flight before the warp waits once
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// per-row tables of a mask-free line, all indexed by row r = 0..n+1
struct LineTab {
  // UL (y lines): normalised sub-diagonal l, modified diagonal dm and its
  // reciprocal, super-diagonal up
  const double *l, *dm, *rdm, *up;
  // cyclic (x, z lines): sub-diagonal a, TDMA gam/bet (+ reciprocal), the
  // back-substituted second solution z of cyclic, and its denominator
  const double *a, *gam, *bet, *rbet, *z;
  double den;
};

struct LineArgs {
  double beta, dt, eta, ft, fb, r0, l0;
  int comp;  // 0 c2, 1 c3, 2 c4, 3 c1
  int jtop;  // lines along j for z and x tiles (ny, or ny-1 for v)
  // launch shape of the partitioned solver (chosen by the context's autotuner;
  // every shape gives the same values): y/z lines 0 = 16 lines per CTA, 1 = 8,
  // 3 = 32, 2 = TMA tiles of 16 lines (FP64); x lines per warp iteration 1 or
  // 2 (0: the default, 2), or 3 / 4: two / one with the staged loads
  int yzshape = 0;
  int xnl = 0;
};

__device__ __forceinline__ double mask_at(const Dims& d, const double* c1, int comp, int i,
                                          int j, int k) {
  long c = d.C(i, j, k);
  double a = __ldg(c1 + c);
  if (comp == 0) return (i < d.nx) ? (a + __ldg(c1 + c + 1)) * 0.50 : a;
  if (comp == 1) return (j < d.ny) ? (a + __ldg(c1 + c + d.nx)) * 0.50 : a;
  if (comp == 2) return (k < d.nz) ? (a + __ldg(c1 + c + (long)d.nx * d.ny)) * 0.50 : a;
  return a;
}

// row r of the line through (i,j,k) along DIR, computed from the mask
template <int DIR, int KIND>
__device__ __forceinline__ Row line_row(const Dims& d, const GridDev& g, const double* c1,
                                        const LineArgs& a, int i, int j, int k, int r) {
  int ii = DIR == 0 ? r : i, jj = DIR == 1 ? r : j, kk = DIR == 2 ? r : k;
  double alpha = a.dt * a.eta * mask_at(d, c1, a.comp, ii, jj, kk) + 1.0;
  const double* D = DIR == 0 ? g.dx : (DIR == 1 ? g.dy : g.dz);
  const double* D12 = DIR == 0 ? g.dx12 : (DIR == 1 ? g.dy12 : g.dz12);
  if (KIND == LK_UL_U) return row_uy(a.beta, alpha, __ldg(D12 + r - 1), __ldg(D12 + r), __ldg(D + r));
  if (KIND == LK_UL_V) return row_vy(a.beta, alpha, __ldg(D + r), __ldg(D + r + 1), __ldg(D12 + r));
  if (KIND == LK_CYC_VEL) return row_cyc(a.beta, alpha, __ldg(D + r), __ldg(D + r + 1), __ldg(D12 + r));
  return row_T(a.beta, alpha, __ldg(D + r - 1), __ldg(D + r), __ldg(D + r + 1), __ldg(D12 + r - 1),
               __ldg(D12 + r), a.l0, a.l0, a.l0, a.r0);
}

// number of rows of the system (0..m) and the interior rows loaded/stored
template <int KIND>
__device__ __forceinline__ int rows_m(int n) {
  return KIND == LK_UL_V ? n : n + 1;
}

// per-line table layout (length L = n+2 per array): UL lines store
// l, dm, rdm, up; cyclic lines store a, gam, bet, rbet, z and den at the end
__host__ __device__ inline size_t line_table_stride(int kind, int n) {
  return (kind <= LK_UL_T ? 4 : 5) * (size_t)(n + 2) + 1;
}

template <int DIR, int KIND, bool EXACT>
__global__ void __launch_bounds__(32) k_lines(Dims d, double* __restrict__ f, LineArgs a,
                                              LineTab tb, const int* __restrict__ slots,
                                              const double* __restrict__ ltab, int pitch) {
  extern __shared__ double sm[];
  const int lane = threadIdx.x;
  const int n = DIR == 0 ? d.nx : (DIR == 1 ? d.ny : d.nz);  // line length (interior)
  const int m = rows_m<KIND>(n);
  const int rlo = 1, rhi = (KIND == LK_UL_V) ? n - 1 : n;   // rows holding the rhs
  int nl, l0, k = 0, j = 0;
  long es, lstride;
  if (DIR == 1) {  // (i,k): 32 consecutive i
    nl = d.nx; l0 = blockIdx.x * 32; k = 1 + blockIdx.y; es = d.sx; lstride = 1;
  } else if (DIR == 2) {  // (i,j): 32 consecutive i
    nl = d.nx; l0 = blockIdx.x * 32; j = 1 + blockIdx.y; es = d.sy; lstride = 1;
  } else {  // (j,k): 32 consecutive j
    nl = a.jtop; l0 = blockIdx.x * 32; k = 1 + blockIdx.y; es = 1; lstride = d.sx;
  }
  const int nvalid = min(32, nl - l0);
  long base0;
  if (DIR == 1) base0 = d.P(1 + l0, 0, k);
  else if (DIR == 2) base0 = d.P(1 + l0, j, 0);
  else base0 = d.P(0, 1 + l0, k);
  // ---------------------------------------------------------- load
  if (DIR == 0) {
    for (int t = 0; t < nvalid; ++t) {
      const double* src = f + base0 + t * lstride;
      for (int r = rlo + lane; r <= rhi; r += 32) cp_async8(sm + t * pitch + r, src + r);
    }
  } else if (lane < nvalid) {
    const double* src = f + base0 + lane * lstride;
    for (int r = rlo; r <= rhi; ++r) cp_async8(sm + lane * pitch + r, src + r * es);
  }
  cp_async_wait_all();
  __syncwarp();
  // ---------------------------------------------------------- solve
  if (lane < nvalid) {
    double* s = sm + lane * pitch;
    long lineid = (DIR == 0) ? (long)(l0 + lane) + (long)a.jtop * (k - 1)
                : (DIR == 1) ? (long)(l0 + lane) + (long)d.nx * (k - 1)
                             : (long)(l0 + lane) + (long)d.nx * (j - 1);
    const int slot = slots[lineid];
    const int L = n + 2;
    // the recurrences run on registers in batches of LB rows: every load of
    // a batch (shared-memory rows and table entries) is issued before the
    // batch's dependent chain starts
    constexpr int LB = 8;
    if (KIND <= LK_UL_T) {
      // UL elimination of implicit_uy/vy/Ty (nse_dominik.f:1549-1570) with the
      // coefficient sweep of this line from its table
      const double *Tl = tb.l, *Tdm = tb.dm, *Trdm = tb.rdm, *Tup = tb.up;
      if (slot >= 0) {
        const double* b = ltab + (size_t)slot * line_table_stride(KIND, n);
        Tl = b; Tdm = b + L; Trdm = b + 2 * L; Tup = b + 3 * L;
      }
      double ut = a.fb;
      s[0] = a.ft;  // the boundary rhs of row 0, read like the other rows
      for (int r0 = m; r0 >= 1; r0 -= LB) {
        double dv[LB], uv[LB], rv[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 - q;
          if (r >= 1) {
            dv[q] = EXACT ? __ldg(Tdm + r) : __ldg(Trdm + r);
            uv[q] = __ldg(Tup + r - 1);
            rv[q] = s[r - 1];
          }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 - q;
          if (r >= 1) {
            double upr = EXACT ? ut / dv[q] : ut * dv[q];
            s[r] = upr;
            ut = rv[q] - uv[q] * upr;
          }
        }
      }
      double x = EXACT ? ut / __ldg(Tdm) : ut * __ldg(Trdm);
      s[0] = x;
      for (int r0 = 1; r0 <= m; r0 += LB) {
        double lv[LB], sv[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 + q;
          if (r <= m) { lv[q] = __ldg(Tl + r); sv[q] = s[r]; }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 + q;
          if (r <= m) { x = sv[q] - lv[q] * x; s[r] = x; }
        }
      }
    } else {
      // cyclic (periodic_implicit.f:67-93) on rows 0..n+1 with ft = fb = 0
      const double gamma = 1.0, beta = -1.0;
      const double *Ta = tb.a, *Tg = tb.gam, *Tb = tb.bet, *Trb = tb.rbet, *Tz = tb.z;
      double den = tb.den;
      if (slot >= 0) {
        const double* b = ltab + (size_t)slot * line_table_stride(KIND, n);
        Ta = b; Tg = b + L; Tb = b + 2 * L; Trb = b + 3 * L; Tz = b + 4 * L;
        den = __ldg(b + 5 * L);
      }
      double x = EXACT ? 0.0 / __ldg(Tb) : 0.0 * __ldg(Trb);
      s[0] = x;
      s[n + 1] = 0.0;  // rhs of row n+1 (fb)
      // forward sweep over rows 1..n+1 (row n+1 has a = 1)
      for (int r0 = 1; r0 <= n + 1; r0 += LB) {
        double av[LB], bv[LB], sv[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 + q;
          if (r <= n + 1) {
            av[q] = (r == n + 1) ? 1.0 : __ldg(Ta + r);
            bv[q] = EXACT ? __ldg(Tb + r) : __ldg(Trb + r);
            sv[q] = s[r];
          }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 + q;
          if (r <= n + 1) {
            double t = sv[q] - av[q] * x;
            x = EXACT ? t / bv[q] : t * bv[q];
            s[r] = x;
          }
        }
      }
      double xn1 = x;
      for (int r0 = n; r0 >= 0; r0 -= LB) {
        double gv[LB], sv[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 - q;
          if (r >= 0) { gv[q] = __ldg(Tg + r + 1); sv[q] = s[r]; }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          int r = r0 - q;
          if (r >= 0) { x = sv[q] - gv[q] * x; s[r] = x; }
        }
      }
      double fact = EXACT ? (x + beta * xn1 / gamma) / den : (x + beta * xn1 / gamma) * (1.0 / den);
#pragma unroll 8
      for (int r = 0; r <= n + 1; ++r) s[r] = s[r] - fact * __ldg(Tz + r);
    }
  }
  __syncwarp();
  // ---------------------------------------------------------- store
  // interior rows only: the ghost rows the reference writes are dead in the
  // resident step (set_bc rewrites every ghost before the projection reads)
  if (DIR == 0) {
    for (int t = 0; t < nvalid; ++t) {
      double* dst = f + base0 + t * lstride;
      for (int r = rlo + lane; r <= rhi; r += 32) dst[r] = sm[t * pitch + r];
    }
  } else if (lane < nvalid) {
    double* dst = f + base0 + lane * lstride;
#pragma unroll 4
    for (int r = rlo; r <= rhi; ++r) dst[r * es] = sm[lane * pitch + r];
  }
}

// coefficient sweep of a whole line of KIND with per-row matrix rows rowfn(r)
// (r = 1..n; rows 0 and n+1/m are the reference's boundary rows), into the
// table arrays; the arithmetic is that of ul_line / cyc_line
template <int KIND, class RowFn>
__device__ void sweep_table(int n, const LineArgs& a, const RowFn& row, double* l, double* dm,
                            double* rdm, double* up, double* aa, double* gam, double* bet,
                            double* rbet, double* z, double* den) {
  if (KIND <= LK_UL_T) {
    const int m = (KIND == LK_UL_V) ? n : n + 1;
    const double up0 = (KIND == LK_UL_V) ? 0.0 : 1.0;
    double aa_ = 1.0, lo = (KIND == LK_UL_V) ? 0.0 : 1.0;
    dm[m] = 1.0;
    for (int r = m; r >= 1; --r) {
      double lr = lo / aa_;
      l[r] = lr;
      Row rp;
      if (r - 1 == 0) { rp.lo = 0.0; rp.di = 1.0; rp.up = up0; }
      else rp = row(r - 1);
      up[r - 1] = rp.up;
      aa_ = rp.di - rp.up * lr;
      dm[r - 1] = aa_;
      lo = rp.lo;
    }
    for (int r = 0; r <= m; ++r) rdm[r] = 1.0 / dm[r];
    up[m] = 0.0;
    l[0] = 0.0;
  } else {
    const double gamma = 1.0, alph = -1.0, beta = -1.0;
    double b_ = 0.0 - gamma;
    bet[0] = b_;
    double zz = gamma / b_;
    z[0] = zz;
    aa[0] = 0.0;
    gam[0] = 0.0;
    double cprev = 1.0;
    for (int r = 1; r <= n + 1; ++r) {
      double av, bv, cv, uv;
      if (r == n + 1) { av = 1.0; bv = 0.0 - alph * beta / gamma; cv = 0.0; uv = alph; }
      else { Row rw = row(r); av = rw.lo; bv = rw.di; cv = rw.up; uv = 0.0; }
      double gm = cprev / b_;
      b_ = bv - av * gm;
      zz = (uv - av * zz) / b_;
      aa[r] = av;
      gam[r] = gm;
      bet[r] = b_;
      z[r] = zz;
      cprev = cv;
    }
    double zn1 = zz;
    for (int r = n; r >= 0; --r) {
      zz = z[r] - gam[r + 1] * zz;
      z[r] = zz;
    }
    for (int r = 0; r <= n + 1; ++r) rbet[r] = 1.0 / bet[r];
    *den = 1.0 + zz + beta * zn1 / gamma;
  }
}

// table of a mask-free line (alpha = 1): KIND, line length n
template <int KIND>
__device__ void build_table(int n, const double* D, const double* D12, const LineArgs& a,
                            double* l, double* dm, double* rdm, double* up, double* aa,
                            double* gam, double* bet, double* rbet, double* z, double* den) {
  const double alpha = a.dt * a.eta * 0.0 + 1.0;
  auto row = [&](int r) -> Row {
    if (KIND == LK_UL_U) return row_uy(a.beta, alpha, D12[r - 1], D12[r], D[r]);
    if (KIND == LK_UL_V) return row_vy(a.beta, alpha, D[r], D[r + 1], D12[r]);
    if (KIND == LK_CYC_VEL) return row_cyc(a.beta, alpha, D[r], D[r + 1], D12[r]);
    return row_T(a.beta, alpha, D[r - 1], D[r], D[r + 1], D12[r - 1], D12[r], a.l0, a.l0, a.l0,
                 a.r0);
  };
  sweep_table<KIND>(n, a, row, l, dm, rdm, up, aa, gam, bet, rbet, z, den);
}

}  // namespace nse
