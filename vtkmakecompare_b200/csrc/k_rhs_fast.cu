// k_rhs_fast.cu -- the FP64-storage right-hand-side kernels (templates in
// k_rhs_fast.cuh) and the pipelined correction of MKP (mkp.f:141-217).
#include "k_rhs_fast.cuh"

namespace nse {

int ring_wait_error_f32();  // k_rhs_f32.cu
int ring_wait_error() {
  const int a = take_ring_wait_err(), b = ring_wait_error_f32();
  return a ? a : b;
}

void launch_rhs_fast(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                     const double* u, const double* v, const double* w, const double* T,
                     const double* u_ta, const double* v_ta, const double* w_ta,
                     double* u_pre, double* v_pre, double* w_pre, double* T_pre,
                     const double* c1, double* u_a, double* v_a, double* w_a, double* u_T,
                     cudaStream_t s, int shape) {
  rhs_fast<double, double>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre, v_pre, w_pre,
                           T_pre, c1, u_a, v_a, w_a, u_T, s, shape);
}

}  // namespace nse

namespace nse {

// mkp.f:141-217 (gradient, correction, pressure, u_ep2, u_ta, divu) in the
// fast form: reciprocal metrics and FMA.  One thread per cell of 0..n.
__global__ void __launch_bounds__(256) k_correct_fast(
    Dims d, GridRcp rg, const double* __restrict__ PHI, const double* __restrict__ ut,
    const double* __restrict__ vt, const double* __restrict__ wt, double* __restrict__ p,
    double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
    double* __restrict__ u_ta, double* __restrict__ v_ta, double* __restrict__ w_ta,
    double* __restrict__ u_ep2, double* __restrict__ v_ep2, double* __restrict__ w_ep2,
    double* __restrict__ divu, double dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long c = d.P(i, j, k);
  double ph = LD(PHI, c);
  double phx = LD(PHI, c + 1), phy = LD(PHI, c + d.sx), phz = LD(PHI, c + d.sy);
  double gx = (phx - ph) * LD(rg.rdx12, i);
  double gy = (phy - ph) * LD(rg.rdy12, j);
  double gz = (phz - ph) * LD(rg.rdz12, k);
  double un = LD(ut, c) - dt * gx;
  double vn = LD(vt, c) - dt * gy;
  double wn = LD(wt, c) - dt * gz;
  u[c] = un;
  v[c] = vn;
  w[c] = wn;
  if (i >= 1 && j >= 1 && k >= 1) {
    p[c] = ph;
    double pxp = (i < d.nx) ? phx : p[c + 1];
    double pyp = (j < d.ny) ? phy : p[c + d.sx];
    double pzp = (k < d.nz) ? phz : p[c + d.sy];
    double ux = u_ta[c], vx = v_ta[c], wx = w_ta[c];
    u_ep2[c] = ux - dt * (pxp - ph) * LD(rg.rdx12, i);
    v_ep2[c] = vx - dt * (pyp - ph) * LD(rg.rdy12, j);
    w_ep2[c] = wx - dt * (pzp - ph) * LD(rg.rdz12, k);
    double um = LD(ut, c - 1) - dt * ((ph - LD(PHI, c - 1)) * LD(rg.rdx12, i - 1));
    double vm = LD(vt, c - d.sx) - dt * ((ph - LD(PHI, c - d.sx)) * LD(rg.rdy12, j - 1));
    double wm = LD(wt, c - d.sy) - dt * ((ph - LD(PHI, c - d.sy)) * LD(rg.rdz12, k - 1));
    divu[c] = (un - um) * LD(rg.rdx, i) + (vn - vm) * LD(rg.rdy, j) + (wn - wm) * LD(rg.rdz, k);
  }
  u_ta[c] = dt * gx;
  v_ta[c] = dt * gy;
  w_ta[c] = dt * gz;
}

void launch_correct_fast(const Dims& d, const GridRcp& rg, const double* PHI, const double* ut,
                         const double* vt, const double* wt, double* p, double* u, double* v,
                         double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                         double* v_ep2, double* w_ep2, double* divu, double dt, cudaStream_t s) {
  dim3 block(64, 4, 1);
  dim3 grid((d.nx + 1 + 63) / 64, (d.ny + 1 + 3) / 4, d.nz + 1);
  count_launch();
  k_correct_fast<<<grid, block, 0, s>>>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta, w_ta,
                                        u_ep2, v_ep2, w_ep2, divu, dt);
}

}  // namespace nse

namespace nse {

// ----------------------------------------------------- pipelined correction
// mkp.f:141-217 for interior cells (1..n in every direction), marching in z
// like k_rhs_fast: a ring of planes of phi (FP64), u*, v*, w* (one-cell halo)
// and the old u_ta, v_ta, w_ta (interior) filled NS-3 planes ahead by
// cp.async.  H is the storage type of u*, u_ta, u_ep2 and divu (float in the
// mixed-precision form); the correction itself is evaluated in FP64.
template <class H, int TY>
__host__ __device__ constexpr int cslot_bytes() {
  return SXW * (TY + 2) * 8 + 3 * SXW * (TY + 2) * (int)sizeof(H) +
         3 * TXW * TY * (int)sizeof(H);
}

template <class H, int TY, int NS>
__device__ __forceinline__ void load_plane_c(char* sm, const Dims& d, int i0, int j0, int K,
                                             int kmax, const double* PHI, const H* UT,
                                             const H* VT, const H* WT, const H* UA,
                                             const H* VA, const H* WA) {
  if (K <= kmax) {
    constexpr int PLANE = SXW * (TY + 2), TILE = TXW * TY;
    char* slot = sm + (K % NS) * cslot_bytes<H, TY>();
    double* ph = reinterpret_cast<double*>(slot);
    H* fl = reinterpret_cast<H*>(slot + PLANE * 8);
    const int tid = threadIdx.y * TXW + threadIdx.x;
    for (int e = tid; e < PLANE; e += TILE) {
      int tx = e % SXW, ty = e / SXW;
      int i = i0 - 1 + tx, j = j0 - 1 + ty;
      if (i > d.nx + 1 || j > d.ny + 1) continue;
      long c = d.P(i, j, K);
      cp_async8(ph + e, PHI + c);
      cp_async8(fl + e, UT + c);
      cp_async8(fl + PLANE + e, VT + c);
      cp_async8(fl + 2 * PLANE + e, WT + c);
    }
    int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i <= d.nx && j <= d.ny && K >= 1 && K <= d.nz) {
      long c = d.P(i, j, K);
      H* h = fl + 3 * PLANE + tid;
      cp_async8(h, UA + c);
      cp_async8(h + TILE, VA + c);
      cp_async8(h + 2 * TILE, WA + c);
    }
  }
  cp_async_commit();
}

// ring slot of the correction (in doubles): phi, then u*, v*, w* and the old
// u_ta, v_ta, w_ta.  TM, the ring's fill: 0 cp.async (u*, v*, w* as halo
// planes, the old u_ta as interior tiles); 1 TMA with the same buffers,
// 128-byte aligned and 34 wide (boxes from x = i0-1); 2 TMA with each buffer
// holding only what the correction reads of it: phi with its full halo, u*
// the tile rows with the x halo, v* the rows j0-1..j0+TY-1, w* and the old
// u_ta the tile rows (13 % less shared memory than 1, so more CTAs fit).
// Offsets of u*, v*, w* and the old u_ta from the start of u* (in elements
// of H) and the index of this thread's cell (its neighbour at x or y offset
// o) in each.
template <class H, int TY, int TM>
struct CorrLay {
  static constexpr int PLANE = SXW * (TY + 2), TILE = TXW * TY;
  static constexpr int FP = TM ? ru16(PLANE) : PLANE;            // phi buffer (doubles)
  static constexpr int US = TM == 2 ? ru16(SXW * TY) : FP;        // u* and w* buffers
  static constexpr int VS = TM == 2 ? ru16(SXW * (TY + 1)) : FP;  // v* buffer
  static constexpr int HS = TM ? ru16(SXW * TY) : TILE;           // old u_ta tiles
  static constexpr int VO = US, WO = US + VS, HO = 2 * US + VS;
  static constexpr int SLOT = TM ? (FP + HO + 3 * HS) * 8 : cslot_bytes<H, TY>();
  static __device__ __forceinline__ int ui(int tx, int ty, int o) {
    return TM == 2 ? ty * SXW + tx + 1 + o : (ty + 1) * SXW + tx + 1 + o;
  }
  static __device__ __forceinline__ int vi(int tx, int ty, int o) {
    return (ty + 1 + o) * SXW + tx + 1;
  }
  static __device__ __forceinline__ int wi(int tx, int ty) {
    return TM == 2 ? ty * SXW + tx + 1 : (ty + 1) * SXW + tx + 1;
  }
  static __device__ __forceinline__ int he(int tx, int ty) {
    return TM ? ty * SXW + tx + 1 : ty * TXW + tx;
  }
};

template <int TY, int NS, int TM>
__device__ __forceinline__ void load_plane_c_tma(char* sm, uint64_t* bars, const CorrMaps& tm,
                                                 int i0, int j0, int K, int k0, int kmax) {
  using L = CorrLay<double, TY, TM>;
  if (K > kmax) return;
  const int r = K - (k0 - 1);
  double* slot = reinterpret_cast<double*>(sm + (r % NS) * L::SLOT);
  uint64_t* bar = &bars[r % NS];
  double* fl = slot + L::FP;
  if constexpr (TM == 1) {
    constexpr unsigned HALO = SXW * (TY + 2) * 8, HB = SXW * TY * 8;
    mbar_expect_tx(bar, 4 * HALO + 3 * HB);
    tma_load_3d(slot, &tm.m[0], i0 - 1, j0 - 1, K, bar);
    for (int f = 0; f < 3; ++f) tma_load_3d(fl + f * L::FP, &tm.m[1 + f], i0 - 1, j0 - 1, K, bar);
  } else {
    constexpr unsigned B = SXW * 8;  // bytes of one box row
    mbar_expect_tx(bar, B * ((TY + 2) + TY + (TY + 1) + TY + 3 * TY));
    tma_load_3d(slot, &tm.m[0], i0 - 1, j0 - 1, K, bar);
    tma_load_3d(fl, &tm.m[1], i0 - 1, j0, K, bar);
    tma_load_3d(fl + L::VO, &tm.m[2], i0 - 1, j0 - 1, K, bar);
    tma_load_3d(fl + L::WO, &tm.m[3], i0 - 1, j0, K, bar);
  }
  for (int f = 0; f < 3; ++f)
    tma_load_3d(fl + L::HO + f * L::HS, &tm.m[4 + f], i0 - 1, j0, K, bar);
}

template <class H, int TY, int NS, int MINB, int TM, int KC = CKCHUNK>
__global__ void __launch_bounds__(TXW * TY, MINB) k_correct_pipe(
    Dims d, GridRcp rg, const double* __restrict__ PHI, const H* __restrict__ UT,
    const H* __restrict__ VT, const H* __restrict__ WT, double* __restrict__ p,
    double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
    H* __restrict__ u_ta, H* __restrict__ v_ta, H* __restrict__ w_ta, H* __restrict__ u_ep2,
    H* __restrict__ v_ep2, H* __restrict__ w_ep2, H* __restrict__ divu, double dt,
    const __grid_constant__ CorrMaps tm) {
  extern __shared__ __align__(128) char smc[];
  char* sm = smc;
  using Lay = CorrLay<H, TY, TM>;
  constexpr bool TMA = TM != 0;
  constexpr int PLANE = Lay::FP, TILE = Lay::HS, F = NS - 3;
  const int i0 = 1 + blockIdx.x * TXW, j0 = 1 + blockIdx.y * TY;
  const int I = i0 + threadIdx.x, J = j0 + threadIdx.y;
  const bool valid = (I <= d.nx) && (J <= d.ny);
  const int k0 = 1 + blockIdx.z * KC;
  const int k1 = min(d.nz, k0 + KC - 1);
  const int kmax = k1 + 1;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + NS * Lay::SLOT);
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  if constexpr (TMA) {
    const bool aligned = ((smem_u32(sm) & 127) == 0) &&
                         ((reinterpret_cast<uintptr_t>(&tm.m[0]) & 63) == 0);
    if (lead) {
      for (int q = 0; q < NS; ++q) mbar_init(&bars[q], 1);
      mbar_fence_init();
      if (!aligned) atomicExch(&g_ring_wait_err, 2);
    }
    __syncthreads();
    if (!aligned) return;
    if (lead)
      for (int q = -1; q <= F; ++q)
        load_plane_c_tma<TY, NS, TM>(sm, bars, tm, i0, j0, k0 + q, k0, kmax);
    ring_wait<NS>(bars, k0 - 1, k0);
    ring_wait<NS>(bars, k0, k0);
  } else {
    for (int q = -1; q <= F; ++q)
      load_plane_c<H, TY, NS>(sm, d, i0, j0, k0 + q, kmax, PHI, UT, VT, WT, u_ta, v_ta, w_ta);
    cp_async_wait<F - 1>();
    __syncthreads();
  }
  double rx = 0, rx12 = 0, rx12m = 0, ry = 0, ry12 = 0, ry12m = 0;
  if (valid) {
    rx = LD(rg.rdx, I); rx12 = LD(rg.rdx12, I); rx12m = LD(rg.rdx12, I - 1);
    ry = LD(rg.rdy, J); ry12 = LD(rg.rdy12, J); ry12m = LD(rg.rdy12, J - 1);
  }
  const int e0 = (threadIdx.y + 1) * SXW + threadIdx.x + 1;
  const int t0 = Lay::he(threadIdx.x, threadIdx.y);
  for (int K = k0; K <= k1; ++K) {
    if constexpr (TMA) {
      if (lead) load_plane_c_tma<TY, NS, TM>(sm, bars, tm, i0, j0, K + 1 + F, k0, kmax);
      ring_wait<NS>(bars, K + 1, k0);
    } else {
      load_plane_c<H, TY, NS>(sm, d, i0, j0, K + 1 + F, kmax, PHI, UT, VT, WT, u_ta, v_ta,
                              w_ta);
    }
    if (valid) {
      constexpr int SB = Lay::SLOT;
      auto slot_of = [&](int P) { return TMA ? (P - (k0 - 1)) % NS : P % NS; };
      const char* sm_m = sm + slot_of(K - 1) * SB;
      const char* sm_c = sm + slot_of(K) * SB;
      const char* sm_p = sm + slot_of(K + 1) * SB;
      const double* qm = reinterpret_cast<const double*>(sm_m);
      const double* qc = reinterpret_cast<const double*>(sm_c);
      const double* qp = reinterpret_cast<const double*>(sm_p);
      const H* fm = reinterpret_cast<const H*>(sm_m + PLANE * 8);
      const H* fc = reinterpret_cast<const H*>(sm_c + PLANE * 8);
#define PH(pl, dxo, dyo) (pl)[e0 + (dyo) * SXW + (dxo)]
      const int tx = threadIdx.x, ty = threadIdx.y;
      const long c = d.P(I, J, K);
      const double rz = LD(rg.rdz, K), rz12 = LD(rg.rdz12, K), rz12m = LD(rg.rdz12, K - 1);
      const double ph = PH(qc, 0, 0), phx = PH(qc, 1, 0), phy = PH(qc, 0, 1), phz = PH(qp, 0, 0),
                   phxm = PH(qc, -1, 0), phym = PH(qc, 0, -1), phzm = PH(qm, 0, 0);
      const double gx = (phx - ph) * rx12, gy = (phy - ph) * ry12, gz = (phz - ph) * rz12;
      const double un = (double)fc[Lay::ui(tx, ty, 0)] - dt * gx;
      const double vn = (double)fc[Lay::VO + Lay::vi(tx, ty, 0)] - dt * gy;
      const double wn = (double)fc[Lay::WO + Lay::wi(tx, ty)] - dt * gz;
      const double um = (double)fc[Lay::ui(tx, ty, -1)] - dt * ((ph - phxm) * rx12m);
      const double vm = (double)fc[Lay::VO + Lay::vi(tx, ty, -1)] - dt * ((ph - phym) * ry12m);
      const double wm = (double)fm[Lay::WO + Lay::wi(tx, ty)] - dt * ((ph - phzm) * rz12m);
#undef PH
      const H* old = fc + Lay::HO + t0;
      u[c] = un;
      v[c] = vn;
      w[c] = wn;
      p[c] = ph;
      const double pxp = (I < d.nx) ? phx : p[c + 1];
      const double pyp = (J < d.ny) ? phy : p[c + d.sx];
      const double pzp = (K < d.nz) ? phz : p[c + d.sy];
      u_ep2[c] = (H)((double)old[0] - dt * (pxp - ph) * rx12);
      v_ep2[c] = (H)((double)old[TILE] - dt * (pyp - ph) * ry12);
      w_ep2[c] = (H)((double)old[2 * TILE] - dt * (pzp - ph) * rz12);
      divu[c] = (H)((un - um) * rx + (vn - vm) * ry + (wn - wm) * rz);
      u_ta[c] = (H)(dt * gx);
      v_ta[c] = (H)(dt * gy);
      w_ta[c] = (H)(dt * gz);
    }
    if constexpr (!TMA) cp_async_wait<F - 1>();
    __syncthreads();
  }
}

// the same correction on the cells of 0..n with i, j or k equal to 0 (the
// ghost faces MKP also writes)
template <class H>
__global__ void k_correct_faces(Dims d, GridRcp rg, const double* __restrict__ PHI,
                                const H* __restrict__ ut, const H* __restrict__ vt,
                                const H* __restrict__ wt, double* __restrict__ u,
                                double* __restrict__ v, double* __restrict__ w,
                                H* __restrict__ u_ta, H* __restrict__ v_ta,
                                H* __restrict__ w_ta, double dt) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  long nA = (long)(ny + 1) * (nz + 1);  // i = 0
  long nB = (long)nx * (nz + 1);        // j = 0, i >= 1
  long nC = (long)nx * ny;              // k = 0, i,j >= 1
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (t < nA) { i = 0; j = (int)(t % (ny + 1)); k = (int)(t / (ny + 1)); }
  else if (t < nA + nB) { long r = t - nA; j = 0; i = 1 + (int)(r % nx); k = (int)(r / nx); }
  else if (t < nA + nB + nC) { long r = t - nA - nB; k = 0; i = 1 + (int)(r % nx); j = 1 + (int)(r / nx); }
  else return;
  long c = d.P(i, j, k);
  double ph = LD(PHI, c);
  double gx = (LD(PHI, c + 1) - ph) * LD(rg.rdx12, i);
  double gy = (LD(PHI, c + d.sx) - ph) * LD(rg.rdy12, j);
  double gz = (LD(PHI, c + d.sy) - ph) * LD(rg.rdz12, k);
  u[c] = (double)LD(ut, c) - dt * gx;
  v[c] = (double)LD(vt, c) - dt * gy;
  w[c] = (double)LD(wt, c) - dt * gz;
  u_ta[c] = (H)(dt * gx);
  v_ta[c] = (H)(dt * gy);
  w_ta[c] = (H)(dt * gz);
}

template <class H, int TY, int NS, int MINB, int TM = 0, int KC = CKCHUNK>
static bool correct_go(const Dims& d, const GridRcp& rg, const double* PHI, const H* ut,
                       const H* vt, const H* wt, double* p, double* u, double* v, double* w,
                       H* u_ta, H* v_ta, H* w_ta, H* u_ep2, H* v_ep2, H* w_ep2, H* divu,
                       double dt, cudaStream_t s) {
  CorrMaps tm;
  size_t smem = (size_t)NS * CorrLay<H, TY, TM>::SLOT;
  if constexpr (TM != 0) {
    const void* f[7] = {PHI, ut, vt, wt, u_ta, v_ta, w_ta};
    // box rows per field: phi, u*, v*, w* with the y halo (TM 1), or phi
    // with it, u* and w* the tile rows, v* the row below too (TM 2)
    const int rows[7] = {TY + 2, TM == 1 ? TY + 2 : TY, TM == 1 ? TY + 2 : TY + 1,
                         TM == 1 ? TY + 2 : TY, TY, TY, TY};
    bool ok = true;
    for (int q = 0; q < 7; ++q) ok = ok && ring_map(&tm.m[q], d, f[q], SXW, rows[q]);
    if (!ok) return false;
    smem += NS * sizeof(uint64_t);
  } else {
    memset(&tm, 0, sizeof(tm));
  }
  dim3 block(TXW, TY, 1);
  dim3 grid((d.nx + TXW - 1) / TXW, (d.ny + TY - 1) / TY, (d.nz + KC - 1) / KC);
  auto kern = k_correct_pipe<H, TY, NS, MINB, TM, KC>;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  count_launch();
  kern<<<grid, block, smem, s>>>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta, w_ta, u_ep2,
                                 v_ep2, w_ep2, divu, dt, tm);
  return true;
}

// launch shape: 0 the storage type's default (CorrShape), 1 32x8 tiles with a
// 5-plane ring and two CTAs per SM, 2 32x4 tiles with 4 planes and four CTAs,
// 3 32x8 tiles with 4 planes and three CTAs; FP64 storage also the TMA ring:
// 4 32x4 tiles with 4 planes and five CTAs per SM, 5 32x4 with 5 planes and
// four CTAs, 6 32x8 with 4 planes and three CTAs, 7 32x4 with 7 planes and
// three CTAs, 8 32x4 with 6 planes and three CTAs, and with 16 z planes per
// CTA instead of 8: 9 32x4 with 5 planes and four CTAs, 10 32x4 with 4 planes
// and five CTAs; the trimmed TMA ring (CorrLay, TM 2): 11 32x4 with 5 planes
// and five CTAs, 12 32x4 with 4 planes and six CTAs, 13 as 11 with 16 z
// planes per CTA, 14 32x4 with 5 planes and four CTAs; 15 the full TMA ring,
// 32x4 with 5 planes and three CTAs (each cell computed the same way; a TMA
// shape whose maps cannot be made runs the default)
template <class H>
static void correct_pipe(const Dims& d, const GridRcp& rg, const double* PHI, const H* ut,
                         const H* vt, const H* wt, double* p, double* u, double* v, double* w,
                         H* u_ta, H* v_ta, H* w_ta, H* u_ep2, H* v_ep2, H* w_ep2, H* divu,
                         double dt, cudaStream_t s, int shape) {
  using Sh = CorrShape<H>;
#define NSE_CORR_GO(TY_, NS_, MB_)                                                           \
  correct_go<H, TY_, NS_, MB_>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta, w_ta, u_ep2,  \
                               v_ep2, w_ep2, divu, dt, s)
#define NSE_CORR_TMA(TY_, NS_, MB_)                                                          \
  done = correct_go<H, TY_, NS_, MB_, 1>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta,  \
                                         w_ta, u_ep2, v_ep2, w_ep2, divu, dt, s)
#define NSE_CORR_TMA16(TY_, NS_, MB_)                                                            \
  done = correct_go<H, TY_, NS_, MB_, 1, 16>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta,  \
                                             w_ta, u_ep2, v_ep2, w_ep2, divu, dt, s)
#define NSE_CORR_TRIM(TY_, NS_, MB_, KC_)                                                       \
  done = correct_go<H, TY_, NS_, MB_, 2, KC_>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta,  \
                                              w_ta, u_ep2, v_ep2, w_ep2, divu, dt, s)
  bool done = false;
  if constexpr (sizeof(H) == 8) {
    if (shape == 4) NSE_CORR_TMA(4, 4, 5);
    else if (shape == 5) NSE_CORR_TMA(4, 5, 4);
    else if (shape == 6) NSE_CORR_TMA(8, 4, 3);
    else if (shape == 7) NSE_CORR_TMA(4, 7, 3);
    else if (shape == 8) NSE_CORR_TMA(4, 6, 3);
    else if (shape == 9) NSE_CORR_TMA16(4, 5, 4);
    else if (shape == 10) NSE_CORR_TMA16(4, 4, 5);
    else if (shape == 11) NSE_CORR_TRIM(4, 5, 5, 8);
    else if (shape == 12) NSE_CORR_TRIM(4, 4, 6, 8);
    else if (shape == 13) NSE_CORR_TRIM(4, 5, 5, 16);
    else if (shape == 14) NSE_CORR_TRIM(4, 5, 4, 8);
    else if (shape == 15) NSE_CORR_TMA(4, 5, 3);
  }
#undef NSE_CORR_TMA
#undef NSE_CORR_TMA16
#undef NSE_CORR_TRIM
  if (!done && shape >= 4) shape = 0;
  if (!done) switch (shape) {
    case 1: NSE_CORR_GO(8, 5, 2); break;
    case 2: NSE_CORR_GO(4, 4, 4); break;
    case 3: NSE_CORR_GO(8, 4, 3); break;
    default: NSE_CORR_GO(Sh::TY, Sh::NS, Sh::MINB); break;
  }
#undef NSE_CORR_GO
  long nf = (long)(d.ny + 1) * (d.nz + 1) + (long)d.nx * (d.nz + 1) + (long)d.nx * d.ny;
  count_launch();
  k_correct_faces<H><<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(d, rg, PHI, ut, vt, wt, u, v,
                                                                  w, u_ta, v_ta, w_ta, dt);
}

void launch_correct_pipe(const Dims& d, const GridRcp& rg, const double* PHI, const double* ut,
                         const double* vt, const double* wt, double* p, double* u, double* v,
                         double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                         double* v_ep2, double* w_ep2, double* divu, double dt, cudaStream_t s,
                         int shape) {
  correct_pipe<double>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta, w_ta, u_ep2, v_ep2,
                       w_ep2, divu, dt, s, shape);
}

void launch_correct_f32(const Dims& d, const GridRcp& rg, const double* PHI, const float* ut,
                        const float* vt, const float* wt, double* p, double* u, double* v,
                        double* w, float* u_ta, float* v_ta, float* w_ta, float* u_ep2,
                        float* v_ep2, float* w_ep2, float* divu, double dt, cudaStream_t s,
                        int shape) {
  correct_pipe<float>(d, rg, PHI, ut, vt, wt, p, u, v, w, u_ta, v_ta, w_ta, u_ep2, v_ep2, w_ep2,
                      divu, dt, s, shape);
}

}  // namespace nse
