// k_rhs_fast.cuh -- fused right-hand side of the resident step, fast form.
//
// The kernel templates; k_rhs_fast.cu instantiates the FP64-storage kernels
// and k_rhs_f32.cu the FP32-storage ones of the mixed-precision form.
//
// The same terms as k_rhs_fused (set_convect :774-825, set_convection_for_
// scalar :852-879, set_conduction :903-939, set_diffusion_for_scalar
// :969-999, set_immersed_boundary :1089-1123, set_explicit :1165-1283,
// set_explicit_for_tempreture :1313-1339, the penalised updates :387-396
// and :1358-1433 of nse_dominik.f), written with the divisions by grid
// spacings replaced by multiplications with tabulated reciprocals and with
// FMA contraction (results agree with the reference form to rounding).
// With uniform material properties the harmonic-mean conductivity of the
// scalar diffusion is the conductivity itself.  Where the penalisation mask
// and its face averages vanish the immersed-boundary term is an exact zero,
// so u_ta is not read and the implicit penalisation is the identity.
// A CTA covers 32 x TY cells of an (x,y) tile and marches over KCHUNK planes
// in z; the halo planes of u, v, w, T sit in a shared-memory ring that is
// filled ahead with asynchronous copies (cp.async) while the current plane
// is computed; the ring holds NS planes (k-1, k, k+1 in use, NS-3 in
// flight) of u, v, w, T and the mask with a one-cell halo and of the four
// AB2 histories, so every input is read from HBM about once.  The tile
// height, ring depth and CTAs per SM are chosen per storage type (RhsShape):
// the FP64 kernel needs ~150 registers per thread without spilling, so it
// runs 32 x 4 tiles, three CTAs per SM.
#pragma once
#include <string.h>

#include "common.cuh"
#include "tma.cuh"

namespace nse {

#define LD(p, i) __ldg((p) + (i))

#ifndef NSE_RHS_KCHUNK
#define NSE_RHS_KCHUNK 16
#endif
constexpr int KCHUNK = NSE_RHS_KCHUNK;  // z planes per CTA
#ifndef NSE_CORR_KCHUNK
#define NSE_CORR_KCHUNK 8
#endif
constexpr int CKCHUNK = NSE_CORR_KCHUNK;  // z planes per CTA of the correction
constexpr int TXW = 32;              // interior tile width of a CTA (x)
constexpr int SXW = TXW + 2;         // with the halo
// a ring slot holds plane K of: u, v, w, T, c1 (halo, SXW x (TY+2) each) and
// the four AB2 histories (interior, TXW x TY); its size in bytes is
// slot_bytes<H, TY>() below

// launch shapes (tile height TY, ring slots NS, CTAs per SM MINB), measured
// at 256x192x256 on B200: FP64 32x8 tiles with two CTAs per SM spilled at
// the 128-register cap (0.636 ms per RHS); 32x4 tiles with three CTAs per
// SM and no spills take 0.474 ms.  FP32 storage and arithmetic fits 117
// registers and keeps 32x8 tiles, two CTAs per SM (0.390 ms; one CTA of
// 32x16 took 0.455 ms).
template <class H, class CT> struct RhsShape { static constexpr int TY = 4, NS = 5, MINB = 3; };
template <> struct RhsShape<float, float> { static constexpr int TY = 8, NS = 5, MINB = 2; };
template <> struct RhsShape<float, double> { static constexpr int TY = 8, NS = 5, MINB = 2; };
// the correction: FP64 32x4 tiles, four CTAs per SM (0.443 against 0.451 ms
// for 32x8); FP32 storage 32x8 tiles, two CTAs per SM
template <class H> struct CorrShape { static constexpr int TY = 4, NS = 5, MINB = 4; };
template <> struct CorrShape<float> { static constexpr int TY = 8, NS = 5, MINB = 2; };

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(float* smem, const float* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// bytes of one ring slot: five halo planes of FP64 fields, then four tiles of
// the AB2 histories in their storage type H
template <class H, int TY>
__host__ __device__ constexpr int slot_bytes() {
  return 5 * SXW * (TY + 2) * 8 + 4 * TXW * TY * (int)sizeof(H);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// plane K into ring slot K mod NS (one commit group, possibly empty)
template <class H, int TY, int NS>
__device__ __forceinline__ void load_plane(char* sm, const Dims& d, int i0, int j0, int K,
                                           int kmax, const double* U, const double* V,
                                           const double* W, const double* T, const double* C1,
                                           const H* UP, const H* VP, const H* WP,
                                           const H* TP) {
  if (K <= kmax) {
    constexpr int PLANE = SXW * (TY + 2), TILE = TXW * TY;
    double* slot = reinterpret_cast<double*>(sm + (K % NS) * slot_bytes<H, TY>());
    const int tid = threadIdx.y * TXW + threadIdx.x;
    for (int e = tid; e < PLANE; e += TILE) {
      int tx = e % SXW, ty = e / SXW;
      int i = i0 - 1 + tx, j = j0 - 1 + ty;
      if (i > d.nx + 1 || j > d.ny + 1) continue;
      long c = d.P(i, j, K);
      cp_async8(slot + e, U + c);
      cp_async8(slot + PLANE + e, V + c);
      cp_async8(slot + 2 * PLANE + e, W + c);
      cp_async8(slot + 3 * PLANE + e, T + c);
      if (i >= 1 && i <= d.nx && j >= 1 && j <= d.ny && K >= 1 && K <= d.nz)
        cp_async8(slot + 4 * PLANE + e, C1 + d.C(i, j, K));
    }
    int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i <= d.nx && j <= d.ny && K >= 1 && K <= d.nz) {
      long c = d.P(i, j, K);
      H* h = reinterpret_cast<H*>(slot + 5 * PLANE) + tid;
      cp_async8(h, UP + c);
      cp_async8(h + TILE, VP + c);
      cp_async8(h + 2 * TILE, WP + c);
      cp_async8(h + 3 * TILE, TP + c);
    }
  }
  cp_async_commit();
}

// ------------------------------------------------ TMA ring (FP64 form)
// The same ring filled by tensor-memory-accelerator copies: one thread issues,
// per plane, one box copy per field (u, v, w, T: 34 x (TY+2) halo boxes at
// x = i0-1, which is a multiple of 32 and so 16-byte aligned; c1, whose
// (nx,ny,nz) layout puts cell I at x = I-1, a 36 x (TY+2) box at c1-x = i0-3;
// the four histories 34 x TY boxes at x = i0-1) and the plane's mbarrier
// counts the bytes in.  Boxes reaching past the arrays read zeros, which no
// valid cell uses.  Fields sit in 128-byte aligned sub-buffers of the slot.
// Only plain (non-multicast) loads of this GPU's own fields are issued, and
// every wait is bounded (g_ring_wait_err, read by the host).
constexpr int ru16(int n) { return (n + 15) & ~15; }  // doubles, rounded to 128 bytes
struct alignas(64) RhsMaps {
  CUtensorMap m[9];  // u, v, w, T, c1, u_pre, v_pre, w_pre, T_pre
};
struct alignas(64) CorrMaps {
  CUtensorMap m[7];  // phi, u*, v*, w*, u_ta, v_ta, w_ta
};
// per translation unit (each of k_rhs_fast.cu and k_rhs_f32.cu has its own)
static __device__ int g_ring_wait_err = 0;
// this translation unit's ring-wait error word, cleared once read
static inline int take_ring_wait_err() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_ring_wait_err, sizeof(int)) != cudaSuccess) return 0;
  if (v) {
    const int z = 0;
    cudaMemcpyToSymbol(g_ring_wait_err, &z, sizeof(int));
  }
  return v;
}

// shared-memory layout of one RHS ring slot (in doubles).  TM, the ring's
// fill: 0 cp.async for every field; 1 TMA for every field (FP64 storage);
// 2 TMA for the five FP64 halo planes and cp.async for the FP32 history
// tiles (mixed form: a padded FP32 field's row pitch, (nx+2)*4 bytes, is not
// the multiple of 16 bytes a tensor map needs).  TMA buffers are padded to
// 128 bytes and use the boxes' pitches.
template <class H, int TY, int TM>
struct RhsLay {
  static constexpr int PLANE = SXW * (TY + 2), TILE = TXW * TY;
  static constexpr int FP = TM ? ru16(PLANE) : PLANE;             // field stride
  static constexpr int C1W = TM ? 36 : SXW;                       // c1 row pitch
  static constexpr int C1P = TM ? ru16(36 * (TY + 2)) : PLANE;    // c1 buffer
  static constexpr int HS = TM == 1 ? ru16(SXW * TY) : TILE;      // history stride (H)
  static constexpr int HOFF = 4 * FP + C1P;                        // first history
  static constexpr int SLOT = TM == 1 ? (HOFF + 4 * HS) * 8
                              : TM == 2 ? HOFF * 8 + ((4 * TILE * (int)sizeof(H) + 127) & ~127)
                                        : slot_bytes<H, TY>();
  // this thread's cell in the c1 buffer and in a history tile
  static __device__ __forceinline__ int c1e(int tx, int ty) {
    return TM ? (ty + 1) * 36 + tx + 2 : (ty + 1) * SXW + tx + 1;
  }
  static __device__ __forceinline__ int he(int tx, int ty) {
    return TM == 1 ? ty * SXW + tx + 1 : ty * TXW + tx;
  }
};

// wait for plane P of the TMA ring (slot and phase counted from plane k0-1)
template <int NS>
__device__ __forceinline__ void ring_wait(uint64_t* bars, int P, int k0) {
  const int r = P - (k0 - 1);
  if (!tma_wait(&bars[r % NS], (unsigned)((r / NS) & 1)) && threadIdx.x == 0 && threadIdx.y == 0)
    atomicExch(&g_ring_wait_err, 1);
}

// plane K of u, v, w, T, c1 (and with TM = 1 the histories) into its slot
// by TMA (one issuing thread)
template <class H, int TY, int NS, int TM>
__device__ __forceinline__ void load_plane_tma(char* sm, uint64_t* bars, const RhsMaps& tm,
                                               int i0, int j0, int K, int k0, int kmax) {
  using L = RhsLay<H, TY, TM>;
  if (K > kmax) return;
  const int r = K - (k0 - 1);
  double* slot = reinterpret_cast<double*>(sm + (r % NS) * L::SLOT);
  uint64_t* bar = &bars[r % NS];
  constexpr unsigned HALO = SXW * (TY + 2) * 8, C1B = 36 * (TY + 2) * 8, HB = SXW * TY * 8;
  mbar_expect_tx(bar, 4 * HALO + C1B + (TM == 1 ? 4 * HB : 0));
  for (int f = 0; f < 4; ++f) tma_load_3d(slot + f * L::FP, &tm.m[f], i0 - 1, j0 - 1, K, bar);
  tma_load_3d(slot + 4 * L::FP, &tm.m[4], i0 - 3, j0 - 2, K - 1, bar);
  if constexpr (TM == 1)
    for (int f = 0; f < 4; ++f)
      tma_load_3d(slot + L::HOFF + f * L::HS, &tm.m[5 + f], i0 - 1, j0, K, bar);
}
// TM = 2: the history tiles of plane K by cp.async (one commit group, empty
// past kmax or outside the interior)
template <class H, int TY, int NS>
__device__ __forceinline__ void load_hist_async(char* sm, const Dims& d, int i0, int j0, int K,
                                                int k0, int kmax, const H* UP, const H* VP,
                                                const H* WP, const H* TP) {
  using L = RhsLay<H, TY, 2>;
  constexpr int TILE = TXW * TY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  if (K <= kmax && i <= d.nx && j <= d.ny && K >= 1 && K <= d.nz) {
    const int r = K - (k0 - 1);
    H* h = reinterpret_cast<H*>(reinterpret_cast<double*>(sm + (r % NS) * L::SLOT) + L::HOFF) +
           threadIdx.y * TXW + threadIdx.x;
    const long c = d.P(i, j, K);
    cp_async8(h, UP + c);
    cp_async8(h + TILE, VP + c);
    cp_async8(h + 2 * TILE, WP + c);
    cp_async8(h + 3 * TILE, TP + c);
  }
  cp_async_commit();
}

// H: storage type of the histories, u_ta and the outputs (double; float in
// the mixed-precision form); CT: arithmetic type (FP32 arithmetic rounds the
// FP64 state as it is read from the ring).  TM: how the ring is filled (see
// RhsLay; tm holds the tensor maps of a TMA fill).
template <class H, class CT, int TY, int NS, int MINB, int TM>
__global__ void __launch_bounds__(TXW * TY, MINB) k_rhs_fast(
    Dims d, GridDev g, GridRcp rg, StepParams sp, const double* __restrict__ U,
    const double* __restrict__ V, const double* __restrict__ W, const double* __restrict__ T,
    const H* __restrict__ U_TA, const H* __restrict__ V_TA, const H* __restrict__ W_TA,
    H* __restrict__ U_PRE, H* __restrict__ V_PRE, H* __restrict__ W_PRE, H* __restrict__ T_PRE,
    const double* __restrict__ C1, H* __restrict__ U_A, H* __restrict__ V_A,
    H* __restrict__ W_A, H* __restrict__ U_T, const __grid_constant__ RhsMaps tm) {
  extern __shared__ __align__(128) char smc[];
  char* sm = smc;
  using Lay = RhsLay<H, TY, TM>;
  constexpr bool TMA = TM != 0;
  constexpr int PLANE = Lay::FP, TILE = Lay::HS;
  constexpr int F = NS - 3;  // planes in flight
  const int i0 = 1 + blockIdx.x * TXW, j0 = 1 + blockIdx.y * TY;
  const int I = i0 + threadIdx.x, J = j0 + threadIdx.y;
  const bool valid = (I <= d.nx) && (J <= d.ny);
  const int k0 = 1 + blockIdx.z * KCHUNK;
  const int k1 = min(d.nz, k0 + KCHUNK - 1);
  const int kmax = k1 + 1;  // last plane any iteration reads
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + NS * Lay::SLOT);
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  // the chunk's z spacings and reciprocals (planes k0-1 .. k0+KCHUNK), staged
  // once instead of loaded per plane; the barrier before the march publishes
  // them
  __shared__ double zt[3][KCHUNK + 2];
  // (issued after the prologue's copies, so the ring fills while these
  // few loads are in flight)
  auto stage_z = [&]() {
    for (int t = threadIdx.y * TXW + threadIdx.x; t < 3 * (KCHUNK + 2); t += TXW * TY) {
      const int q = t / (KCHUNK + 2), kk = k0 - 1 + t % (KCHUNK + 2);
      if (kk <= d.nz + 1) zt[q][t % (KCHUNK + 2)] = q == 0 ? g.dz[kk] : q == 1 ? rg.rdz[kk] : rg.rdz12[kk];
    }
  };
  if constexpr (TMA) {
    // the copies need 128-byte aligned buffers and a 64-byte aligned map; a
    // launch that finds otherwise records the error (its cells then read
    // zeros from the never-filled ring, and the host reports the error)
    const bool aligned = ((smem_u32(sm) & 127) == 0) &&
                         ((reinterpret_cast<uintptr_t>(&tm.m[0]) & 63) == 0);
    if (lead) {
      for (int q = 0; q < NS; ++q) mbar_init(&bars[q], 1);
      mbar_fence_init();
      if (!aligned) atomicExch(&g_ring_wait_err, 2);
    }
    __syncthreads();
    if (!aligned) return;
    // prologue: planes k0-1 .. k0+F
    if (lead)
      for (int q = -1; q <= F; ++q)
        load_plane_tma<H, TY, NS, TM>(sm, bars, tm, i0, j0, k0 + q, k0, kmax);
    if constexpr (TM == 2)
      for (int q = -1; q <= F; ++q)
        load_hist_async<H, TY, NS>(sm, d, i0, j0, k0 + q, k0, kmax, U_PRE, V_PRE, W_PRE, T_PRE);
    stage_z();
    if constexpr (TM == 2) cp_async_wait<F - 1>();
    __syncthreads();
    ring_wait<NS>(bars, k0 - 1, k0);
    ring_wait<NS>(bars, k0, k0);
  } else {
    // prologue: planes k0-1 .. k0+F (the last F-1 stay in flight)
    for (int q = -1; q <= F; ++q)
      load_plane<H, TY, NS>(sm, d, i0, j0, k0 + q, kmax, U, V, W, T, C1, U_PRE, V_PRE, W_PRE,
                            T_PRE);
    stage_z();
    cp_async_wait<F - 1>();
    __syncthreads();
  }
  using R = CT;  // arithmetic type
  const R DT = (R)sp.dt;
  const R a1 = (sp.l == 1) ? R(1) : R(1.5), a2 = (sp.l == 1) ? R(0) : R(-0.5);
  const R kd = (R)(sp.dt / sp.Re * 0.5);
  const R r0 = (R)sp.rho_cp, rr0 = (R)(1.0 / sp.rho_cp), l0 = (R)sp.thc;
  const R kT = (R)(0.5 / sp.Re / sp.Sc / sp.rho_cp * sp.dt);
  R dx = 0, dxp = 0, dxm = 0, rx = 0, rxp = 0, rx12 = 0, rx12m = 0;
  R dy = 0, dyp = 0, dym = 0, ry = 0, ryp = 0, ry12 = 0, ry12m = 0;
  if (valid) {
    dx = LD(g.dx, I); dxp = LD(g.dx, I + 1); dxm = LD(g.dx, I - 1);
    rx = LD(rg.rdx, I); rxp = LD(rg.rdx, I + 1);
    rx12 = LD(rg.rdx12, I); rx12m = LD(rg.rdx12, I - 1);
    dy = LD(g.dy, J); dyp = LD(g.dy, J + 1); dym = LD(g.dy, J - 1);
    ry = LD(rg.rdy, J); ryp = LD(rg.rdy, J + 1);
    ry12 = LD(rg.rdy12, J); ry12m = LD(rg.rdy12, J - 1);
  }
  const int e0 = (threadIdx.y + 1) * SXW + threadIdx.x + 1;  // this cell in a halo plane
  const int t0 = Lay::he(threadIdx.x, threadIdx.y);          // this cell in a history tile
  const int ec = Lay::c1e(threadIdx.x, threadIdx.y);         // this cell in the c1 plane
  for (int K = k0; K <= k1; ++K) {
    // plane K+1+F goes into the slot of plane K-2, free since the barrier
    // that ended the previous iteration
    if constexpr (TMA) {
      if (lead) load_plane_tma<H, TY, NS, TM>(sm, bars, tm, i0, j0, K + 1 + F, k0, kmax);
      if constexpr (TM == 2)
        load_hist_async<H, TY, NS>(sm, d, i0, j0, K + 1 + F, k0, kmax, U_PRE, V_PRE, W_PRE,
                                   T_PRE);
      ring_wait<NS>(bars, K + 1, k0);
    } else {
      load_plane<H, TY, NS>(sm, d, i0, j0, K + 1 + F, kmax, U, V, W, T, C1, U_PRE, V_PRE,
                            W_PRE, T_PRE);
    }
    if (valid) {
      constexpr int SB = Lay::SLOT;
      // ring slot of plane K: K mod NS, or counted from k0-1 in the TMA ring
      auto slot_of = [&](int P) { return TMA ? (P - (k0 - 1)) % NS : P % NS; };
      const double* pm = reinterpret_cast<const double*>(sm + slot_of(K - 1) * SB);
      const double* pc = reinterpret_cast<const double*>(sm + slot_of(K) * SB);
      const double* pp = reinterpret_cast<const double*>(sm + slot_of(K + 1) * SB);
      const long c = d.P(I, J, K);
      const int kz = K - k0 + 1;  // plane K in the staged z tables
      const R dz = zt[0][kz], dzp = zt[0][kz + 1], dzm = zt[0][kz - 1];
      const R rz = zt[1][kz], rzp = zt[1][kz + 1];
      const R rz12 = zt[2][kz], rz12m = zt[2][kz - 1];
      // neighbourhood from shared memory (field f at offset f*PLANE), each
      // component's values loaded where they are used: short live ranges keep
      // the register count low
#define AT(pl, f, dxo, dyo) (R)(pl)[(f) * PLANE + e0 + (dyo) * SXW + (dxo)]
#define C1AT(pl, dxo, dyo) (R)(pl)[4 * PLANE + ec + (dyo) * Lay::C1W + (dxo)]
      // masks (set_immersed_boundary :1037-1080) and AB2 histories
      const R cc1 = C1AT(pc, 0, 0);
      const R c2 = (I < d.nx) ? (cc1 + C1AT(pc, 1, 0)) * R(0.5) : cc1;
      const R c3 = (J < d.ny) ? (cc1 + C1AT(pc, 0, 1)) * R(0.5) : cc1;
      const R c4 = (K < d.nz) ? (cc1 + C1AT(pp, 0, 0)) * R(0.5) : cc1;
      const H* hist = reinterpret_cast<const H*>(pc + Lay::HOFF) + t0;
      const bool solid = (c2 != R(0)) || (c3 != R(0)) || (c4 != R(0)) || (cc1 != R(0));
    // u
    {
      const R uc = AT(pc, 0, 0, 0), uxp = AT(pc, 0, 1, 0), uxm = AT(pc, 0, -1, 0),
              uyp = AT(pc, 0, 0, 1), uym = AT(pc, 0, 0, -1), uzp = AT(pp, 0, 0, 0),
              uzm = AT(pm, 0, 0, 0);
      const R vc = AT(pc, 1, 0, 0), vxp = AT(pc, 1, 1, 0), vym = AT(pc, 1, 0, -1),
              vxpym = AT(pc, 1, 1, -1);
      const R wc = AT(pc, 2, 0, 0), wxp = AT(pc, 2, 1, 0), wzm = AT(pm, 2, 0, 0),
              wxpzm = AT(pm, 2, 1, 0);
      R s1 = uc + uxp, s2 = uc + uxm;
      R U1 = (s1 * s1 - s2 * s2) * rx12;
      R U2 = ((vxp * dxp + vc * dx) * (uyp + uc) - (vxpym * dxp + vym * dx) * (uc + uym)) *
                  rx12 * ry;
      R U3 = ((wxp * dxp + wc * dx) * (uzp + uc) - (wxpzm * dxp + wzm * dx) * (uc + uzm)) *
                  rx12 * rz;
      R uv = R(0.25) * (-U1 - U2 - U3) * DT + (R)sp.force * DT;
      R L = ((uxp - uc) * rxp - (uc - uxm) * rx) * rx12 +
                 ((uyp - uc) * ry12 - (uc - uym) * ry12m) * ry +
                 ((uzp - uc) * rz12 - (uc - uzm) * rz12m) * rz;
      R ua = a1 * uv + a2 * (R)hist[0] + kd * L;
      U_PRE[c] = uv;
      if (solid && c2 != R(0)) {
        ua += (R)sp.eta * c2 * LD(U_TA, c) * DT;
        U_A[c] = (uc + ua) / (R(1) + (R)sp.eta * c2 * DT);
      } else {
        U_A[c] = uc + ua;
      }
    }
    // v
    {
      const R uc = AT(pc, 0, 0, 0), uyp = AT(pc, 0, 0, 1), uxm = AT(pc, 0, -1, 0),
              uxmyp = AT(pc, 0, -1, 1);
      const R vc = AT(pc, 1, 0, 0), vxp = AT(pc, 1, 1, 0), vxm = AT(pc, 1, -1, 0),
              vyp = AT(pc, 1, 0, 1), vym = AT(pc, 1, 0, -1), vzp = AT(pp, 1, 0, 0),
              vzm = AT(pm, 1, 0, 0);
      const R wc = AT(pc, 2, 0, 0), wyp = AT(pc, 2, 0, 1), wzm = AT(pm, 2, 0, 0),
              wypzm = AT(pm, 2, 0, 1);
      R V1 = ((uyp * dyp + uc * dy) * (vxp + vc) - (uxmyp * dyp + uxm * dy) * (vc + vxm)) *
                  ry12 * rx;
      R s1 = vc + vyp, s2 = vc + vym;
      R V2 = (s1 * s1 - s2 * s2) * ry12;
      R V3 = ((wyp * dyp + wc * dy) * (vzp + vc) - (wypzm * dyp + wzm * dy) * (vc + vzm)) *
                  ry12 * rz;
      R vv = R(0.25) * (-V1 - V2 - V3) * DT;
      R L = ((vxp - vc) * rx12 - (vc - vxm) * rx12m) * rx +
                 ((vyp - vc) * ryp - (vc - vym) * ry) * ry12 +
                 ((vzp - vc) * rz12 - (vc - vzm) * rz12m) * rz;
      R va = a1 * vv + a2 * (R)hist[TILE] + kd * L;
      V_PRE[c] = vv;
      if (solid && c3 != R(0)) va += (R)sp.eta * c3 * LD(V_TA, c) * DT;
      if (J == d.ny) va = R(0);  // set_bc(u_a,v_a,...) zeroes v_a(:,ny,:)
      if (solid && c3 != R(0)) V_A[c] = (vc + va) / (R(1) + (R)sp.eta * c3 * DT);
      else V_A[c] = vc + va;
    }
    // w
    {
      const R uc = AT(pc, 0, 0, 0), uzp = AT(pp, 0, 0, 0), uxm = AT(pc, 0, -1, 0),
              uxmzp = AT(pp, 0, -1, 0);
      const R vc = AT(pc, 1, 0, 0), vzp = AT(pp, 1, 0, 0), vym = AT(pc, 1, 0, -1),
              vymzp = AT(pp, 1, 0, -1);
      const R wc = AT(pc, 2, 0, 0), wxp = AT(pc, 2, 1, 0), wxm = AT(pc, 2, -1, 0),
              wyp = AT(pc, 2, 0, 1), wym = AT(pc, 2, 0, -1), wzp = AT(pp, 2, 0, 0),
              wzm = AT(pm, 2, 0, 0);
      R W1 = ((uzp * dzp + uc * dz) * (wxp + wc) - (uxmzp * dzp + uxm * dz) * (wc + wxm)) *
                  rz12 * rx;
      R W2 = ((vzp * dzp + vc * dz) * (wyp + wc) - (vymzp * dzp + vym * dz) * (wc + wym)) *
                  rz12 * ry;
      R s1 = wc + wzp, s2 = wc + wzm;
      R W3 = (s1 * s1 - s2 * s2) * rz12;
      R wv = R(0.25) * (-W1 - W2 - W3) * DT;
      R L = ((wxp - wc) * rx12 - (wc - wxm) * rx12m) * rx +
                 ((wyp - wc) * ry12 - (wc - wym) * ry12m) * ry +
                 ((wzp - wc) * rzp - (wc - wzm) * rz) * rz12;
      R wa = a1 * wv + a2 * (R)hist[2 * TILE] + kd * L;
      W_PRE[c] = wv;
      if (solid && c4 != R(0)) {
        wa += (R)sp.eta * c4 * LD(W_TA, c) * DT;
        W_A[c] = (wc + wa) / (R(1) + (R)sp.eta * c4 * DT);
      } else {
        W_A[c] = wc + wa;
      }
    }
    // T
    {
      const R uc = AT(pc, 0, 0, 0), uxm = AT(pc, 0, -1, 0);
      const R vc = AT(pc, 1, 0, 0), vym = AT(pc, 1, 0, -1);
      const R wc = AT(pc, 2, 0, 0), wzm = AT(pm, 2, 0, 0);
      const R tc = AT(pc, 3, 0, 0), txp = AT(pc, 3, 1, 0), txm = AT(pc, 3, -1, 0),
              typ = AT(pc, 3, 0, 1), tym = AT(pc, 3, 0, -1), tzp = AT(pp, 3, 0, 0),
              tzm = AT(pm, 3, 0, 0);
      R UT = (-((r0 * txm * dx + r0 * tc * dxm) * uxm) * R(0.5) * rx12m +
                   ((r0 * tc * dxp + r0 * txp * dx) * uc) * R(0.5) * rx12) *
                  rx;
      R VT = (-((r0 * tym * dy + r0 * tc * dym) * vym) * R(0.5) * ry12m +
                   ((r0 * tc * dyp + r0 * typ * dy) * vc) * R(0.5) * ry12) *
                  ry;
      R WT = (-((r0 * tzm * dz + r0 * tc * dzm) * wzm) * R(0.5) * rz12m +
                   ((r0 * tc * dzp + r0 * tzp * dz) * wc) * R(0.5) * rz12) *
                  rz;
      R vt = (-UT - VT - WT) * DT * rr0 + (R)sp.source * DT;
      R D1 = (l0 * (txp - tc) * rx12 - l0 * (tc - txm) * rx12m) * rx;
      R D2 = (l0 * (typ - tc) * ry12 - l0 * (tc - tym) * ry12m) * ry;
      R D3 = (l0 * (tzp - tc) * rz12 - l0 * (tc - tzm) * rz12m) * rz;
      R ut = a1 * vt + a2 * (R)hist[3 * TILE] + kT * (D1 + D2 + D3);
      T_PRE[c] = vt;
      if (cc1 != R(0)) {
        R pen = (R)sp.eta * cc1 * DT;
        U_T[c] = (tc + ut + pen * (R)sp.tsolid) / (R(1) + pen);
      } else {
        U_T[c] = tc + ut;
      }
    }
#undef AT
#undef C1AT
    }  // valid
    if constexpr (TM != 1) cp_async_wait<F - 1>();
    __syncthreads();
  }
}

// tensor maps of the TMA ring: the padded FP64 fields (box 34 x (TY+2) or
// 34 x TY) and the (nx,ny,nz) mask (box 36 x (TY+2)); false when a field is
// not 16-byte aligned or the driver rejects a map
static bool ring_map(CUtensorMap* m, const Dims& d, const void* p, int bx, int by) {
  if (((uintptr_t)p & 15) != 0 || ((d.nx + 2) * 8) % 16 != 0) return false;
  return tma_encode_3d(m, p, true, d.nx + 2, d.ny + 2, d.nz + 2, (long)(d.nx + 2) * 8,
                       (long)(d.nx + 2) * (d.ny + 2) * 8, bx, by, 1);
}
static bool mask_map(CUtensorMap* m, const Dims& d, const void* p, int by) {
  if (((uintptr_t)p & 15) != 0 || (d.nx * 8) % 16 != 0) return false;
  return tma_encode_3d(m, p, true, d.nx, d.ny, d.nz, (long)d.nx * 8, (long)d.nx * d.ny * 8, 36,
                       by, 1);
}

template <class H, class CT, int TY, int NS, int MINB, int TM = 0>
static bool rhs_go(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                   const double* u, const double* v, const double* w, const double* T,
                   const H* u_ta, const H* v_ta, const H* w_ta, H* u_pre, H* v_pre, H* w_pre,
                   H* T_pre, const double* c1, H* u_a, H* v_a, H* w_a, H* u_T, cudaStream_t s) {
  RhsMaps tm;
  memset(&tm, 0, sizeof(tm));
  size_t smem = (size_t)NS * RhsLay<H, TY, TM>::SLOT;
  if constexpr (TM != 0) {
    const void* f[4] = {u, v, w, T};
    const void* h[4] = {u_pre, v_pre, w_pre, T_pre};
    bool ok = mask_map(&tm.m[4], d, c1, TY + 2);
    for (int q = 0; q < 4; ++q) {
      ok = ok && ring_map(&tm.m[q], d, f[q], SXW, TY + 2);
      if constexpr (TM == 1) ok = ok && ring_map(&tm.m[5 + q], d, h[q], SXW, TY);
    }
    if (!ok) return false;
    smem += NS * sizeof(uint64_t);
  }
  dim3 block(TXW, TY, 1);
  dim3 grid((d.nx + TXW - 1) / TXW, (d.ny + TY - 1) / TY, (d.nz + KCHUNK - 1) / KCHUNK);
  auto kern = k_rhs_fast<H, CT, TY, NS, MINB, TM>;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  count_launch();
  kern<<<grid, block, smem, s>>>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre, v_pre, w_pre,
                                 T_pre, c1, u_a, v_a, w_a, u_T, tm);
  return true;
}

// launch shape: 0 the storage type's default (RhsShape), 1 32x4 tiles with a
// 4-plane ring and four CTAs per SM, 2 32x8 tiles with a 5-plane ring and two
// CTAs per SM, 3 32x8 tiles with a 4-plane ring and two CTAs per SM; the TMA
// ring (every field in FP64 storage; the halo planes, with cp.async history
// tiles, in FP32 storage): 4 32x4 tiles with 5 planes and three CTAs per SM,
// 5 32x4 with 4 planes and four CTAs, 6 32x8 with 4 planes and two CTAs
// (every shape computes each cell the same way; the context's autotuner
// picks one; a TMA shape whose maps cannot be made runs the default)
template <class H, class CT>
static void rhs_fast(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                     const double* u, const double* v, const double* w, const double* T,
                     const H* u_ta, const H* v_ta, const H* w_ta, H* u_pre, H* v_pre, H* w_pre,
                     H* T_pre, const double* c1, H* u_a, H* v_a, H* w_a, H* u_T,
                     cudaStream_t s, int shape) {
  using Sh = RhsShape<H, CT>;
#define NSE_RHS_GO(TY_, NS_, MB_)                                                           \
  rhs_go<H, CT, TY_, NS_, MB_>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre, v_pre,    \
                               w_pre, T_pre, c1, u_a, v_a, w_a, u_T, s)
  constexpr int TM = sizeof(H) == 8 ? 1 : 2;
#define NSE_RHS_TMA(TY_, NS_, MB_)                                                              \
  done = rhs_go<H, CT, TY_, NS_, MB_, TM>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre,    \
                                          v_pre, w_pre, T_pre, c1, u_a, v_a, w_a, u_T, s)
  {
    bool done = false;
    if (shape == 4) NSE_RHS_TMA(4, 5, 3);
    else if (shape == 5) NSE_RHS_TMA(4, 4, 4);
    else if (shape == 6) NSE_RHS_TMA(8, 4, 2);
    if (done) return;
    if (shape >= 4) shape = 0;
  }
#undef NSE_RHS_TMA
  switch (shape) {
    case 1: NSE_RHS_GO(4, 4, 4); break;
    case 2: NSE_RHS_GO(8, 5, 2); break;
    case 3: NSE_RHS_GO(8, 4, 2); break;
    default: NSE_RHS_GO(Sh::TY, Sh::NS, Sh::MINB); break;
  }
#undef NSE_RHS_GO
}

}  // namespace nse
