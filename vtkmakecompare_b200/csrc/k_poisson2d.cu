// k_poisson2d.cu -- the FFT Poisson solve of MKP (mkp.f:9-320) in three
// passes over HBM for 256-point transforms in x and z (the reference's
// P2S -> SPN/SP0B -> S2P/PHIBC, p2s_fftw2d.f:5-223, mkp.f:223-320):
//
//  * k_p2s256: the whole P2S of one y-plane in one launch.  A cluster of 8
//    CTAs owns the plane: CTA r transforms the z rows 32r..32r+31 along x
//    (two real rows packed as one complex 256-point FFT, register-resident
//    16 x 16 scheme) and keeps its 32 x 129 half-spectrum rows in shared
//    memory; after a cluster barrier it transforms the kx columns
//    16r..16r+15 along z, reading the column's 256 values from the eight
//    CTAs' shared memory (distributed shared memory), and writes the
//    spectrum, scaled by 1/(NX*NZ).  The kx = 0 and kx = NX/2 columns are
//    real after the x transform; CTA 0 transforms them together as one
//    complex column and separates them with the Hermitian identities.  The
//    plane crosses HBM once each way: read NX*NZ reals, write the half
//    spectrum.
//  * k_spn_part: SPN + SP0B, one (kx, kz) system per 16 lanes of a warp,
//    partitioned (16 partitions of m = ny/16 rows, rows in registers),
//    pivots computed on the fly from AC and KXZ (no tables to read).
//  * k_s2p256: S2P and PHIBC of one plane in one launch, the same cluster
//    scheme in reverse (z columns, then x rows), writing the plane with its
//    periodic x/z ghosts and, for J = 1 and NY, the Neumann ghost planes.
//
// Global memory traffic per solve: read and write the real field once,
// read and write the half spectrum twice -- the algorithmic 2*8*N + 4*16*Hs
// bytes.  This file keeps FMA contraction (the transform is a different
// algorithm from FFTW's in any case).
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"
#include "fft_core.cuh"
#include "tma.cuh"

namespace cg = cooperative_groups;

namespace nse {

namespace {

constexpr int kCl = 8;             // CTAs per plane (the cluster)
constexpr int kN = 256;            // transform length in x and z
constexpr int kRows = kN / kCl;    // 32 z rows per CTA in the x transforms
constexpr int kXLD = kRows + 1;    // kz pitch of a CTA's slab X[kx][kz] (forward)
constexpr int kCols = 16;          // kx columns per CTA in the z transforms
constexpr int kZLD = kN + 1;       // kz pitch of a CTA's slab X[col][kz] (inverse)
constexpr int kEx = 16 * 17;       // per-16-thread exchange buffer (complex)
// shared memory of both plane kernels: the exchange buffers of 16 transforms
// (aliased with the spectrum slab once the slab has been read) and the
// 256-entry buffer of the packed kx = 0 / NX/2 column
constexpr size_t kSlabForward = (size_t)(kN / 2 + 1) * kXLD;   // 4257 complex
constexpr size_t kSlabInverse = (size_t)kCols * kZLD;           // 4112 complex
constexpr size_t kExAll = (size_t)16 * kEx;                     // 4352 complex
constexpr size_t kSlabMax = kSlabForward > kExAll ? kSlabForward : kExAll;
constexpr size_t kPlaneSmem = (kSlabMax + kN) * sizeof(double2);
static_assert(kSlabInverse <= kExAll, "inverse slab fits the exchange area");

__device__ __forceinline__ double2 dz2() { return make_double2(0.0, 0.0); }

// ------------------------------------------------------ forward (P2S) ----
__global__ void __cluster_dims__(kCl, 1, 1) __launch_bounds__(256, 2)
    k_p2s256(Dims d, double2* __restrict__ spec, long sj, long sk,
             const double* __restrict__ FP, const double2* __restrict__ twx,
             const double2* __restrict__ twz) {
  extern __shared__ __align__(16) double2 p2s_sm[];
  double2* X = p2s_sm;  // slab X[kx * kXLD + kz_local], or exchange
  double2* packed = p2s_sm + kSlabMax;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int J = 1 + blockIdx.y;
  const int tid = threadIdx.x;

  // x transforms: half-warp h owns z rows (ka, kb), thread b holds x[16a + b]
  {
    const int h = tid >> 4, b = tid & 15;
    const int kl = 2 * h;  // local row of ka
    const int ka = rank * kRows + kl, kb = ka + 1;
    double2 v[16];
    const double* ra = FP + d.P(0, J, ka);
    const double* rb = FP + d.P(0, J, kb);
#pragma unroll
    for (int a = 0; a < 16; ++a) v[a] = make_double2(ra[16 * a + b], rb[16 * a + b]);
    fft256_inner(v, b, twx, false);
    double2* E = X + h * kEx;
#pragma unroll
    for (int c = 0; c < 16; ++c) E[b * 17 + c] = v[c];
    __syncwarp();
#pragma unroll
    for (int bb = 0; bb < 16; ++bb) v[bb] = E[bb * 17 + b];
    dft16(v, false);  // thread b: Z[b + 16e] in v[e]
    __syncthreads();  // every exchange buffer is read: the slab may overwrite them
    // Hermitian split: the partner of Z[b + 16e] is Z[256 - b - 16e], held by
    // lane (16 - b) & 15 in register 15 - e (b > 0) or (16 - e) & 15 (b = 0)
#pragma unroll
    for (int e = 0; e <= 8; ++e) {
      const double2 give = (b == 0) ? v[(16 - e) & 15] : v[15 - e];
      double2 zr;
      zr.x = __shfl_sync(0xffffffffu, give.x, (16 - b) & 15, 16);
      zr.y = __shfl_sync(0xffffffffu, give.y, (16 - b) & 15, 16);
      const int kx = b + 16 * e;
      if (kx <= kN / 2) {
        const double2 z = v[e];
        X[kx * kXLD + kl] = make_double2((z.x + zr.x) * 0.5, (z.y - zr.y) * 0.5);
        X[kx * kXLD + kl + 1] = make_double2((z.y + zr.y) * 0.5, (zr.x - z.x) * 0.5);
      }
    }
  }
  cluster.sync();

  // z transforms: thread (col, b); column kx = 16 rank + col; CTA 0's column
  // 0 carries kx = 0 (real part) and kx = NX/2 (imaginary part)
  const int col = tid & 15, bz = tid >> 4;
  const int kx = rank * kCols + col;
  const bool pk = (rank == 0 && col == 0);
  double2 v[16];
#pragma unroll
  for (int a = 0; a < 16; ++a) {
    const double2* Xr = cluster.map_shared_rank(X, a >> 1);
    const int kzl = 16 * (a & 1) + bz;
    if (pk)
      v[a] = make_double2(Xr[kzl].x, Xr[(kN / 2) * kXLD + kzl].x);
    else
      v[a] = Xr[kx * kXLD + kzl];
  }
  cluster.sync();  // no CTA reads this slab any more
  fft256_inner(v, bz, twz, false);
  double2* S_ = X;  // [c][b][col]
#pragma unroll
  for (int c = 0; c < 16; ++c) S_[(c * 16 + bz) * 17 + col] = v[c];
  __syncthreads();
#pragma unroll
  for (int bb = 0; bb < 16; ++bb) v[bb] = S_[(bz * 16 + bb) * 17 + col];
  dft16(v, false);  // thread (col, c = bz): Y[c + 16e]
  const double nrm = 1.0 / ((double)kN * (double)kN);  // 2^-16, exact
#pragma unroll
  for (int e = 0; e < 16; ++e) v[e] = make_double2(v[e].x * nrm, v[e].y * nrm);
  double2* out = spec + sj * (J - 1);
  if (rank == 0) {
    // separate the packed column: F0 = (Y + conj(Y(-kz)))/2,
    // F(NX/2) = (Y - conj(Y(-kz)))/(2i)
    if (pk) {
#pragma unroll
      for (int e = 0; e < 16; ++e) packed[bz + 16 * e] = v[e];
    }
    __syncthreads();
    if (pk) {
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int kz = bz + 16 * e;
        const double2 y = v[e], yr = packed[(kN - kz) & (kN - 1)];
        out[sk * kz] = make_double2((y.x + yr.x) * 0.5, (y.y - yr.y) * 0.5);
        out[kN / 2 + sk * kz] = make_double2((y.y + yr.y) * 0.5, (yr.x - y.x) * 0.5);
      }
      return;
    }
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) out[kx + sk * (bz + 16 * e)] = v[e];
}

// ---------------------------------------------- inverse (S2P + PHIBC) ----
__global__ void __cluster_dims__(kCl, 1, 1) __launch_bounds__(256, 2)
    k_s2p256(Dims d, const double2* __restrict__ spec, long sj, long sk,
             double* __restrict__ FP, const double2* __restrict__ twx,
             const double2* __restrict__ twz) {
  extern __shared__ __align__(16) double2 s2p_sm[];
  double2* X = s2p_sm;  // slab X[col * kZLD + kz], or exchange
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int J = 1 + blockIdx.y;
  const int tid = threadIdx.x;
  const int ny = d.ny;
  {
    // z transforms of the kx columns 16 rank .. 16 rank + 15; CTA 0's column 0
    // transforms F(kx=0) + i F(kx=NX/2)
    const int col = tid & 15, bz = tid >> 4;
    const int kx = rank * kCols + col;
    const bool pk = (rank == 0 && col == 0);
    const double2* in = spec + sj * (J - 1);
    double2 v[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) {
      const long o = sk * (16 * a + bz);
      if (pk) {
        const double2 f0 = in[o], fn = in[kN / 2 + o];
        v[a] = make_double2(f0.x - fn.y, f0.y + fn.x);
      } else {
        v[a] = in[kx + o];
      }
    }
    fft256_inner(v, bz, twz, true);
    double2* S_ = X;
#pragma unroll
    for (int c = 0; c < 16; ++c) S_[(c * 16 + bz) * 17 + col] = v[c];
    __syncthreads();
#pragma unroll
    for (int bb = 0; bb < 16; ++bb) v[bb] = S_[(bz * 16 + bb) * 17 + col];
    dft16(v, true);  // thread (col, c = bz): column value at kz = c + 16e
    __syncthreads();  // exchange read by all: the slab may overwrite it
#pragma unroll
    for (int e = 0; e < 16; ++e) X[col * kZLD + bz + 16 * e] = v[e];
  }
  cluster.sync();
  // x transforms (c2r): half-warp h owns z rows (ka, kb); thread b gathers
  // A = X(kx, ka), B = X(kx, kb) for kx = b + 16q from CTA q
  const int h = tid >> 4, b = tid & 15;
  const int ka = rank * kRows + 2 * h, kb = ka + 1;
  double2 A[9], B[9];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double2* Xr = cluster.map_shared_rank(X, q);
    A[q] = Xr[b * kZLD + ka];
    B[q] = Xr[b * kZLD + kb];
  }
  {
    const double2* X0 = cluster.map_shared_rank(X, 0);
    const double2 pa = X0[ka], pb = X0[kb];  // packed column: (F0, F(NX/2)) parts
    A[8] = make_double2(pa.y, 0.0);
    B[8] = make_double2(pb.y, 0.0);
    if (b == 0) {
      A[0] = make_double2(pa.x, 0.0);
      B[0] = make_double2(pb.x, 0.0);
    }
  }
  cluster.sync();  // no CTA reads this slab any more
  double2* S_ = X + h * kEx;
  // Z = A + iB at kx, conj(A) + i conj(B) at N - kx (kx = 0 and N/2 real)
#pragma unroll
  for (int q = 0; q <= 8; ++q) {
    const int kx = b + 16 * q;
    if (kx > kN / 2) break;
    const double2 a = A[q], c = B[q];
    S_[kx] = make_double2(a.x - c.y, a.y + c.x);
    if (kx > 0 && kx < kN / 2) S_[kN - kx] = make_double2(a.x + c.y, c.x - a.y);
  }
  __syncwarp();
  double2 v[16];
#pragma unroll
  for (int a = 0; a < 16; ++a) v[a] = S_[16 * a + b];
  __syncwarp();
  fft256_inner(v, b, twx, true);
#pragma unroll
  for (int c = 0; c < 16; ++c) S_[b * 17 + c] = v[c];
  __syncwarp();
#pragma unroll
  for (int bb = 0; bb < 16; ++bb) v[bb] = S_[bb * 17 + b];
  dft16(v, true);  // thread b: sample i = b + 16e of row ka (real) and kb (imaginary)
  // the plane with its periodic x/z ghosts (S2P's wrap p2s_fftw2d.f:211-216
  // and PHIBC's x/z loops mkp.f:306-319: cell (I, K) = sample (I mod NX,
  // K mod NZ) for I = 0..NX+1, K = 0..NZ+1), and PHIBC's y ghost planes
  // (mkp.f:300-304: (I, 0|NY+1, K) = (I, 1|NY, K), I = 0..NX, K = 1..NZ)
  const int jg = (J == 1) ? 0 : ((J == ny) ? ny + 1 : -1);
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int i = b + 16 * e;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int k = r ? kb : ka;
      const double val = r ? v[e].y : v[e].x;
      const int nI = (i <= 1) ? 2 : 1, nK = (k <= 1) ? 2 : 1;
      for (int ii = 0; ii < nI; ++ii) {
        const int I = i + ii * kN;
        for (int kk = 0; kk < nK; ++kk) {
          const int K = k + kk * kN;
          FP[d.P(I, J, K)] = val;
          if (jg >= 0 && I <= kN && K >= 1 && K <= kN) FP[d.P(I, jg, K)] = val;
        }
      }
    }
  }
}

// ------------------------------------------------ SPN + SP0B, partitioned --
// System s = (kx, kz) = (s mod H, s div H) of mkp.f:239-254 (tridiagonal
// a = AC1, b = AC2 - KXZ, c = AC3 with the Neumann folds b(1) += a(1),
// b(NY) += c(NY)), rows J = 1..ny at spec[kx + sj (J-1) + sk kz].  Lane k of
// the system's 16 lanes owns rows r = kM .. kM + M - 1 (0-based) in registers.
// With the partition's first and last unknowns F, E, every interior row is
// x = g + F p + E q (interior Thomas solves with Dirichlet ends); the first
// and last rows then form a tridiagonal system in (F_0, E_0, F_1, E_1, ...),
// F is eliminated lane-locally (with one neighbour exchange), the 16
// unknowns E_k are found by parallel cyclic reduction over the 16 lanes
// (4 shuffle levels), F follows, and the interior rows are back-substituted.
// The mean mode (0, 0) runs SP0B's forward marching (mkp.f:263-290) on one
// lane from a staged copy of its column.
template <int M>
__global__ void __launch_bounds__(256, 2)
    k_spn_part(int H, int ny, int nsys, double2* __restrict__ spec, long sj, long sk,
               const double* __restrict__ AC, const double* __restrict__ KXZ) {
  __shared__ double acs[3 * 256];
  __shared__ double2 meanc[256];
  for (int r = threadIdx.x; r < ny; r += blockDim.x) {
    acs[r] = AC[r];
    acs[256 + r] = AC[ny + r];
    acs[512 + r] = AC[2 * ny + r];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int k = lane & 15;
  const unsigned hm = (lane < 16) ? 0x0000ffffu : 0xffff0000u;
  const int s = blockIdx.x * 16 + (threadIdx.x >> 4);
  if (s >= nsys) return;  // the whole half-warp
  const int kx = s % H, kz = s / H;
  double2* B = spec + kx + sk * kz;
  const int r0 = k * M;
  double2 dv[M];
#pragma unroll
  for (int t = 0; t < M; ++t) dv[t] = B[sj * (r0 + t)];

  if (s == 0) {
    // SP0B: phi(J=1) = 0, phi(J+1) = (D(J) - AC1 phi(J-1) - AC2 phi(J)) / AC3
#pragma unroll
    for (int t = 0; t < M; ++t) meanc[r0 + t] = dv[t];
    __syncwarp(hm);
    if (k == 0) {
      double2 pm = dz2(), pc = dz2();
      double2 Dj = meanc[0];
      meanc[0] = dz2();
      for (int J = 1; J <= ny - 1; ++J) {
        const double2 Dn = meanc[J];
        const double a1 = acs[J - 1], a2 = acs[256 + J - 1], a3 = acs[512 + J - 1];
        const double2 pn = make_double2((Dj.x - a1 * pm.x - a2 * pc.x) / a3,
                                        (Dj.y - a1 * pm.y - a2 * pc.y) / a3);
        meanc[J] = pn;
        pm = pc;
        pc = pn;
        Dj = Dn;
      }
    }
    __syncwarp(hm);
#pragma unroll
    for (int t = 0; t < M; ++t) B[sj * (r0 + t)] = meanc[r0 + t];
    return;
  }

  const double kxz = KXZ[kx + (long)H * kz];
  auto coef = [&](int r, double& a, double& b, double& c) {
    a = acs[r];
    b = acs[256 + r] - kxz;
    c = acs[512 + r];
    if (r == 0) { b = b + a; a = 0.0; }
    if (r == ny - 1) { b = b + c; c = 0.0; }
  };
  // interior rows t = 1..M-2 with Dirichlet ends: forward sweep of g (in dv),
  // p (response to F = 1) and the super-diagonal ratios cp
  double cp[M], pp[M];
  {
    double cprev = 0.0, pprev = 0.0;
    double2 gprev = dz2();
#pragma unroll
    for (int t = 1; t <= M - 2; ++t) {
      double a, b, c;
      coef(r0 + t, a, b, c);
      const double inv = 1.0 / (b - a * cprev);
      const double2 g = make_double2((dv[t].x - a * gprev.x) * inv, (dv[t].y - a * gprev.y) * inv);
      const double p = (t == 1 ? -a : -a * pprev) * inv;
      cp[t] = c * inv;
      pp[t] = p;
      dv[t] = g;
      gprev = g;
      pprev = p;
      cprev = cp[t];
    }
  }
  // g, p, q at the interior end rows (q: response to E = 1, q(M-2) = -cp(M-2))
  const double2 gL = dv[M - 2];
  const double pL = pp[M - 2], qL = -cp[M - 2];
  double2 g1 = gL;
  double p1 = pL, q1 = qL;
#pragma unroll
  for (int t = M - 3; t >= 1; --t) {
    g1 = make_double2(dv[t].x - cp[t] * g1.x, dv[t].y - cp[t] * g1.y);
    p1 = pp[t] - cp[t] * p1;
    q1 = -cp[t] * q1;
  }
  // reduced rows: first row (unknowns E_{k-1}, F_k, E_k), last row (F_k, E_k, F_{k+1})
  double as, bs, cs, ae, be, ce;
  coef(r0, as, bs, cs);
  coef(r0 + M - 1, ae, be, ce);
  const double sub_s = as, diag_s = bs + cs * p1, sup_s = cs * q1;
  const double2 rhs_s = make_double2(dv[0].x - cs * g1.x, dv[0].y - cs * g1.y);
  const double sub_e = ae * pL, diag_e = be + ae * qL, sup_e = ce;
  const double2 rhs_e = make_double2(dv[M - 1].x - ae * gL.x, dv[M - 1].y - ae * gL.y);
  // eliminate F_k and F_{k+1}: a tridiagonal system in E over the 16 lanes
  const double nd = __shfl_down_sync(hm, diag_s, 1, 16);
  const double nsub = __shfl_down_sync(hm, sub_s, 1, 16);
  const double nsup = __shfl_down_sync(hm, sup_s, 1, 16);
  const double nrx = __shfl_down_sync(hm, rhs_s.x, 1, 16);
  const double nry = __shfl_down_sync(hm, rhs_s.y, 1, 16);
  const double f = sub_e / diag_s;
  const double hh = (k < 15) ? sup_e / nd : 0.0;
  double al = -f * sub_s;
  double be_ = diag_e - f * sup_s - (k < 15 ? hh * nsub : 0.0);
  double ga = (k < 15) ? -hh * nsup : 0.0;
  double rx = rhs_e.x - f * rhs_s.x - (k < 15 ? hh * nrx : 0.0);
  double ry = rhs_e.y - f * rhs_s.y - (k < 15 ? hh * nry : 0.0);
#pragma unroll
  for (int st = 1; st < 16; st <<= 1) {
    const double am = __shfl_up_sync(hm, al, st, 16), bm = __shfl_up_sync(hm, be_, st, 16);
    const double gm = __shfl_up_sync(hm, ga, st, 16);
    const double xm = __shfl_up_sync(hm, rx, st, 16), ym = __shfl_up_sync(hm, ry, st, 16);
    const double ap = __shfl_down_sync(hm, al, st, 16), bp = __shfl_down_sync(hm, be_, st, 16);
    const double gp = __shfl_down_sync(hm, ga, st, 16);
    const double xp = __shfl_down_sync(hm, rx, st, 16), yp = __shfl_down_sync(hm, ry, st, 16);
    const bool hasm = k >= st, hasp = k + st < 16;
    const double k1 = hasm ? al / bm : 0.0;
    const double k2 = hasp ? ga / bp : 0.0;
    const double nal = hasm ? -k1 * am : 0.0;
    const double nga = hasp ? -k2 * gp : 0.0;
    be_ = be_ - (hasm ? k1 * gm : 0.0) - (hasp ? k2 * ap : 0.0);
    rx = rx - (hasm ? k1 * xm : 0.0) - (hasp ? k2 * xp : 0.0);
    ry = ry - (hasm ? k1 * ym : 0.0) - (hasp ? k2 * yp : 0.0);
    al = nal;
    ga = nga;
  }
  const double2 E = make_double2(rx / be_, ry / be_);
  const double Emx = __shfl_up_sync(hm, E.x, 1, 16), Emy = __shfl_up_sync(hm, E.y, 1, 16);
  const double2 Em = (k > 0) ? make_double2(Emx, Emy) : dz2();
  const double2 F = make_double2((rhs_s.x - sub_s * Em.x - sup_s * E.x) / diag_s,
                                 (rhs_s.y - sub_s * Em.y - sup_s * E.y) / diag_s);
  // interior: x = back substitution of g' + F p' (+ E q' on the last row)
  B[sj * r0] = F;
  B[sj * (r0 + M - 1)] = E;
  double2 xn = make_double2(dv[M - 2].x + F.x * pp[M - 2] + E.x * qL,
                            dv[M - 2].y + F.y * pp[M - 2] + E.y * qL);
  B[sj * (r0 + M - 2)] = xn;
#pragma unroll
  for (int t = M - 3; t >= 1; --t) {
    xn = make_double2(dv[t].x + F.x * pp[t] - cp[t] * xn.x, dv[t].y + F.y * pp[t] - cp[t] * xn.y);
    B[sj * (r0 + t)] = xn;
  }
}

// ------------------------------------------- SPN + SP0B through TMA tiles
// The spectrum as a real array [kz][J][2 Hp] (re, im interleaved): a tile is
// 32 reals (16 kx columns) x the ny rows of one kz, brought into shared memory
// by one TMA copy (box at x = 32 t, 16-byte aligned), next tile in flight on a
// second buffer.  Thread (lane, k): lane = real column (kx = 16 t + lane/2,
// re or im), k = partition (warp) of m = ny/16 rows; the re and im columns
// of a system run the same coefficient recurrence.  Each partition is
// eliminated in registers as in k_spn_part; the reduced system (F eliminated
// with the next partition's first row, then cyclic reduction over the 16
// partitions) goes through shared memory, one column per lane, so every
// shared-memory access of a warp is 32 consecutive reals.  The mean mode's
// two columns are skipped by the partitioned solve and marched by SP0B
// (mkp.f:263-290) afterwards, from the tile.  The solved tile leaves by one
// TMA store (columns past NX/2 are carried along unchanged).
__device__ int g_spn_wait_err = 0;

template <int M>
__global__ void __launch_bounds__(512, 1)
    k_spn_tma(const __grid_constant__ CUtensorMap tm, int H, int ny, int nz, int ntx,
              const double* __restrict__ AC, const double* __restrict__ KXZ) {
  constexpr int NL = 32;  // real columns per tile
  extern __shared__ __align__(128) unsigned char ssm[];
  const size_t tb_bytes = (((size_t)ny * NL * 8) + 127) & ~(size_t)127;
  double* buf0 = reinterpret_cast<double*>(ssm);
  double* buf1 = reinterpret_cast<double*>(ssm + tb_bytes);
  double* acs = reinterpret_cast<double*>(ssm + 2 * tb_bytes);  // AC1, AC2, AC3 [ny] each
  double* rs = acs + 3 * ny;          // [4][16][NL] first-row values of each partition
  double* pc = rs + 4 * 16 * NL;      // [4][16][NL] cyclic-reduction rows
  uint64_t* bar = reinterpret_cast<uint64_t*>(pc + 4 * 16 * NL);
  const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
  const long ntiles = (long)ntx * nz;
  const unsigned tile_tx = (unsigned)ny * NL * 8;
  for (int r = threadIdx.x; r < 3 * ny; r += blockDim.x)
    acs[r] = AC[r];
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  // the copies need the tensor map 64-byte aligned and the tile buffers
  // 128-byte aligned in shared memory; a launch that finds otherwise records
  // the error and copies nothing
  const bool aligned = ((reinterpret_cast<uintptr_t>(&tm) & 63) == 0) &&
                       ((smem_u32(buf0) & 127) == 0) && ((smem_u32(buf1) & 127) == 0) &&
                       ((smem_u32(bar) & 7) == 0);
  if (!aligned) {
    if (threadIdx.x == 0) atomicExch(&g_spn_wait_err, 2);
    return;
  }
  __syncthreads();
  long q = blockIdx.x;
  if (threadIdx.x == 0 && q < ntiles) {
    mbar_expect_tx(&bar[0], tile_tx);
    tma_load_3d(buf0, &tm, (int)(q % ntx) * NL, 0, (int)(q / ntx), &bar[0]);
  }
  const int r0 = k * M;
  auto RS = [&](int v, int kk) -> double& { return rs[(v * 16 + kk) * NL + lane]; };
  auto PC = [&](int v, int kk) -> double& { return pc[(v * 16 + kk) * NL + lane]; };
  for (int it = 0; q < ntiles; q += gridDim.x, ++it) {
    double* cur = (it & 1) ? buf1 : buf0;
    double* nxt = (it & 1) ? buf0 : buf1;
    const long qn = q + gridDim.x;
    if (threadIdx.x == 0 && qn < ntiles) {
      tma_store_wait_read();
      uint64_t* nb = &bar[(it + 1) & 1];
      mbar_expect_tx(nb, tile_tx);
      tma_load_3d(nxt, &tm, (int)(qn % ntx) * NL, 0, (int)(qn / ntx), nb);
    }
    if (!tma_wait(&bar[it & 1], (unsigned)((it >> 1) & 1)) && threadIdx.x == 0)
      atomicExch(&g_spn_wait_err, 1);
    const int kx = (int)(q % ntx) * (NL / 2) + (lane >> 1);
    const int kz = (int)(q / ntx);
    const bool mean = kx == 0 && kz == 0;
    const bool valid = kx < H && !mean;
    const double kxz = valid ? KXZ[kx + (long)H * kz] : 1.0;
    auto coef = [&](int r, double& a, double& b, double& c) {
      a = acs[r];
      b = acs[ny + r] - kxz;
      c = acs[2 * ny + r];
      if (r == 0) { b = b + a; a = 0.0; }
      if (r == ny - 1) { b = b + c; c = 0.0; }
    };
    double dv[M], cp[M], pp[M];
    const double* col = cur + (size_t)r0 * NL + lane;
#pragma unroll
    for (int t = 0; t < M; ++t) dv[t] = col[(size_t)t * NL];
    {
      double cprev = 0.0, pprev = 0.0, gprev = 0.0;
#pragma unroll
      for (int t = 1; t <= M - 2; ++t) {
        double a, b, c;
        coef(r0 + t, a, b, c);
        const double inv = 1.0 / (b - a * cprev);
        const double g = (dv[t] - a * gprev) * inv;
        const double p = (t == 1 ? -a : -a * pprev) * inv;
        cp[t] = c * inv;
        pp[t] = p;
        dv[t] = g;
        gprev = g;
        pprev = p;
        cprev = cp[t];
      }
    }
    const double gL = dv[M - 2], pL = pp[M - 2], qL = -cp[M - 2];
    double g1 = gL, p1 = pL, q1 = qL;
#pragma unroll
    for (int t = M - 3; t >= 1; --t) {
      g1 = dv[t] - cp[t] * g1;
      p1 = pp[t] - cp[t] * p1;
      q1 = -cp[t] * q1;
    }
    double as, bs, cs, ae, be, ce;
    coef(r0, as, bs, cs);
    coef(r0 + M - 1, ae, be, ce);
    const double sub_s = as, diag_s = bs + cs * p1, sup_s = cs * q1, rhs_s = dv[0] - cs * g1;
    const double sub_e = ae * pL, diag_e = be + ae * qL, sup_e = ce, rhs_e = dv[M - 1] - ae * gL;
    RS(0, k) = sub_s;
    RS(1, k) = diag_s;
    RS(2, k) = sup_s;
    RS(3, k) = rhs_s;
    __syncthreads();
    // F eliminated: al E(k-1) + be E(k) + ga E(k+1) = rho
    const double f = sub_e / diag_s;
    double al = -f * sub_s, bb = diag_e - f * sup_s, ga = 0.0, rho = rhs_e - f * rhs_s;
    if (k < 15) {
      const double hh = sup_e / RS(1, k + 1);
      bb -= hh * RS(0, k + 1);
      ga = -hh * RS(2, k + 1);
      rho -= hh * RS(3, k + 1);
    }
#pragma unroll
    for (int st = 1; st < 16; st <<= 1) {
      PC(0, k) = al;
      PC(1, k) = bb;
      PC(2, k) = ga;
      PC(3, k) = rho;
      __syncthreads();
      double nal = 0.0, nga = 0.0, nbb = bb, nrho = rho;
      if (k >= st) {
        const double k1 = al / PC(1, k - st);
        nal = -k1 * PC(0, k - st);
        nbb -= k1 * PC(2, k - st);
        nrho -= k1 * PC(3, k - st);
      }
      if (k + st < 16) {
        const double k2 = ga / PC(1, k + st);
        nga = -k2 * PC(2, k + st);
        nbb -= k2 * PC(0, k + st);
        nrho -= k2 * PC(3, k + st);
      }
      __syncthreads();
      al = nal;
      ga = nga;
      bb = nbb;
      rho = nrho;
    }
    const double E = rho / bb;
    PC(0, k) = E;
    __syncthreads();
    const double Em = k > 0 ? PC(0, k - 1) : 0.0;
    const double F = (rhs_s - sub_s * Em - sup_s * E) / diag_s;
    double* dst = cur + (size_t)r0 * NL + lane;
    if (valid) {
      dst[0] = F;
      dst[(size_t)(M - 1) * NL] = E;
      double xn = dv[M - 2] + F * pp[M - 2] + E * qL;
      dst[(size_t)(M - 2) * NL] = xn;
#pragma unroll
      for (int t = M - 3; t >= 1; --t) {
        xn = dv[t] + F * pp[t] - cp[t] * xn;
        dst[(size_t)t * NL] = xn;
      }
    }
    __syncthreads();
    if (kz == 0 && k == 0 && lane < 2 && (q % ntx) == 0) {
      // SP0B on column `lane` (re | im) of the mean mode, from the tile
      double* m0 = cur + lane;
      double pm = 0.0, pcur = 0.0, Dj = m0[0];
      m0[0] = 0.0;
      for (int J = 1; J <= ny - 1; ++J) {
        const double Dn = m0[(size_t)J * NL];
        const double pn = (Dj - acs[J - 1] * pm - acs[ny + J - 1] * pcur) / acs[2 * ny + J - 1];
        m0[(size_t)J * NL] = pn;
        pm = pcur;
        pcur = pn;
        Dj = Dn;
      }
    }
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tma_store_3d(&tm, (int)(q % ntx) * NL, 0, kz, cur);
      tma_store_commit();
    }
  }
  if (threadIdx.x == 0) tma_store_wait_all();
}

template <int M>
bool spn_tma_launch(const PoissonPlan& pp, cudaStream_t s) {
  CUtensorMap tm;
  const long e0 = 2L * pp.Hp, p1 = e0 * 8, p2 = p1 * pp.ny;
  if (p1 % 16 != 0 || ((uintptr_t)pp.spec & 15) != 0 || pp.ny > 256) return false;
  if (!tma_encode_3d(&tm, pp.spec, true, e0, pp.ny, pp.nz, p1, p2, 32, pp.ny, 1)) return false;
  const int ntx = (2 * pp.H + 31) / 32;
  const long ntiles = (long)ntx * pp.nz;
  const size_t tb = (((size_t)pp.ny * 32 * 8) + 127) & ~(size_t)127;
  const size_t smem = 2 * tb + (3 * (size_t)pp.ny + 8 * 16 * 32) * 8 + 16;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute((const void*)k_spn_tma<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  count_launch();
  k_spn_tma<M><<<(int)std::min<long>(ntiles, sms), 512, smem, s>>>(tm, pp.H, pp.ny, pp.nz, ntx,
                                                                  pp.AC, pp.KXZ);
  return true;
}

template <int M>
void spn_part_launch(const PoissonPlan& pp, cudaStream_t s) {
  const int nsys = pp.H * pp.nz;
  count_launch();
  k_spn_part<M><<<(nsys + 15) / 16, 256, 0, s>>>(
      pp.H, pp.ny, nsys, reinterpret_cast<double2*>(pp.spec), pp.Hp, (long)pp.Hp * pp.ny,
      pp.AC, pp.KXZ);
}

// dynamic shared memory above 48 KB needs the per-kernel opt-in (per device:
// set on every launch, as the other transform launches do)
void plane_smem_optin() {
  cudaFuncSetAttribute((const void*)k_p2s256, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmem);
  cudaFuncSetAttribute((const void*)k_s2p256, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmem);
}

}  // namespace

bool spn_part_ok(const PoissonPlan& pp) {
  return pp.ny % 16 == 0 && pp.ny / 16 >= 3 && pp.ny / 16 <= 16;
}

bool poisson3_ok(const PoissonPlan& pp) {
  return pp.nx == kN && pp.nz == kN && spn_part_ok(pp);
}

void launch_spn_part(const PoissonPlan& pp, cudaStream_t s) {
  switch (pp.ny / 16) {
    case 3: spn_part_launch<3>(pp, s); break;
    case 4: spn_part_launch<4>(pp, s); break;
    case 5: spn_part_launch<5>(pp, s); break;
    case 6: spn_part_launch<6>(pp, s); break;
    case 7: spn_part_launch<7>(pp, s); break;
    case 8: spn_part_launch<8>(pp, s); break;
    case 9: spn_part_launch<9>(pp, s); break;
    case 10: spn_part_launch<10>(pp, s); break;
    case 11: spn_part_launch<11>(pp, s); break;
    case 12: spn_part_launch<12>(pp, s); break;
    case 13: spn_part_launch<13>(pp, s); break;
    case 14: spn_part_launch<14>(pp, s); break;
    case 15: spn_part_launch<15>(pp, s); break;
    default: spn_part_launch<16>(pp, s); break;
  }
}

bool launch_spn_tma(const PoissonPlan& pp, cudaStream_t s) {
  if (!spn_part_ok(pp)) return false;
  switch (pp.ny / 16) {
    case 3: return spn_tma_launch<3>(pp, s);
    case 4: return spn_tma_launch<4>(pp, s);
    case 5: return spn_tma_launch<5>(pp, s);
    case 6: return spn_tma_launch<6>(pp, s);
    case 7: return spn_tma_launch<7>(pp, s);
    case 8: return spn_tma_launch<8>(pp, s);
    case 9: return spn_tma_launch<9>(pp, s);
    case 10: return spn_tma_launch<10>(pp, s);
    case 11: return spn_tma_launch<11>(pp, s);
    case 12: return spn_tma_launch<12>(pp, s);
    case 13: return spn_tma_launch<13>(pp, s);
    case 14: return spn_tma_launch<14>(pp, s);
    case 15: return spn_tma_launch<15>(pp, s);
    default: return spn_tma_launch<16>(pp, s);
  }
}

int spn2_wait_error();  // k_spn_babe_tma (k_fft.cu)
int spn_wait_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_spn_wait_err, sizeof(int)) != cudaSuccess) return 0;
  if (v) {
    const int z = 0;
    cudaMemcpyToSymbol(g_spn_wait_err, &z, sizeof(int));
  }
  const int b = spn2_wait_error();
  return v ? v : b;
}

void launch_p2s256(const PoissonPlan& pp, const Dims& d, const double* FP, cudaStream_t s) {
  plane_smem_optin();
  count_launch();
  k_p2s256<<<dim3(kCl, pp.ny), 256, kPlaneSmem, s>>>(
      d, reinterpret_cast<double2*>(pp.spec), pp.Hp, (long)pp.Hp * pp.ny, FP,
      reinterpret_cast<const double2*>(pp.twx), reinterpret_cast<const double2*>(pp.twz));
}

void launch_s2p256_phibc(const PoissonPlan& pp, const Dims& d, double* FP, cudaStream_t s) {
  plane_smem_optin();
  count_launch();
  k_s2p256<<<dim3(kCl, pp.ny), 256, kPlaneSmem, s>>>(
      d, reinterpret_cast<const double2*>(pp.spec), pp.Hp, (long)pp.Hp * pp.ny, FP,
      reinterpret_cast<const double2*>(pp.twx), reinterpret_cast<const double2*>(pp.twz));
}

}  // namespace nse
