// k_fft.cu -- FFT Poisson solve and projection of MKP (mkp.f:9-320,
// p2s_fftw2d.f:5-223) on the GPU with the library's own FFT kernels.
//
// Transform: per y-plane J the reference computes FFTW's r2c 2-D DFT of the
// samples FP(0:NX-1,J,0:NZ-1) (unnormalised, sign -1), keeps kx = 0..NX/2
// and divides by NX*NZ; the inverse is the unnormalised c2r.  Here:
//  * x pass: two real rows are packed into one complex row (a + i b), one
//    complex FFT of length NX is run in shared memory and the two half
//    spectra are separated with the Hermitian identities;
//  * z pass: a CTA holds W adjacent kx columns of one plane (W x NZ complex)
//    and runs W complex FFTs of length NZ;
//  * both use a Stockham autosort FFT (radix 4, 2, 3, 5 stages; Govindaraju
//    et al., SC'08 formulation) with twiddles exp(-2 pi i k/N) taken from a
//    table computed on the host in extended precision.
// Spectral solve (SPN/SP0B): one thread per (kx,kz) wavenumber runs CTRIDIAG
// (tridiag.f:43-58) along y, coalesced over kx; the mean mode runs SP0B's
// forward marching.  This file keeps FMA contraction enabled (the transform
// is a different algorithm from FFTW's in any case).
#include <math.h>

#include "common.cuh"
#include "fft_core.cuh"
#include "tma.cuh"

namespace nse {

struct FFTShape {
  int n;
  int nst;
  int rad[16];
};

static FFTShape make_shape(int n) {
  FFTShape s;
  s.n = n;
  s.nst = 0;
  int m = n;
  while (m % 4 == 0) { s.rad[s.nst++] = 4; m /= 4; }
  while (m % 2 == 0) { s.rad[s.nst++] = 2; m /= 2; }
  while (m % 3 == 0) { s.rad[s.nst++] = 3; m /= 3; }
  while (m % 5 == 0) { s.rad[s.nst++] = 5; m /= 5; }
  if (m != 1) s.nst = -1;  // unsupported prime factor
  return s;
}

bool fft_size_ok(int n) { return n >= 2 && make_shape(n).nst > 0; }

// one Stockham stage over `nb` independent FFTs of length N (fft f at
// src + f*fs); all threads of the block cooperate
template <int R, class CT>
__device__ __forceinline__ void stockham_stage(const CT* __restrict__ src, CT* __restrict__ dst,
                                               int N, int nb, int Ns,
                                               const CT* __restrict__ tw, bool inv, int fs) {
  int nbf = N / R;
  int total = nbf * nb;
  int tstep = N / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int f = t / nbf, j = t - f * nbf;
    const CT* in = src + (long)f * fs;
    CT* out = dst + (long)f * fs;
    CT v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[j + r * nbf];
    int kj = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        CT w = __ldg(tw + r * kj * tstep);
        if (inv) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    DftSmall<R, CT>::run(v, inv);
    int idxD = (j / Ns) * Ns * R + kj;
#pragma unroll
    for (int r = 0; r < R; ++r) out[idxD + r * Ns] = v[r];
  }
}

// runs the full FFT; data starts in a, returns the buffer holding the result;
// FFT f occupies [f*fs, f*fs + N) (fs >= N; fs = N+1 keeps column-wise tiles
// free of shared-memory bank conflicts)
template <class CT>
__device__ CT* fft_block(CT* a, CT* b, const FFTShape& sh, int nb, const CT* tw, bool inv,
                         int fs) {
  int Ns = 1;
  for (int s = 0; s < sh.nst; ++s) {
    int R = sh.rad[s];
    __syncthreads();
    if (R == 4) stockham_stage<4>(a, b, sh.n, nb, Ns, tw, inv, fs);
    else if (R == 2) stockham_stage<2>(a, b, sh.n, nb, Ns, tw, inv, fs);
    else if (R == 3) stockham_stage<3>(a, b, sh.n, nb, Ns, tw, inv, fs);
    else stockham_stage<5>(a, b, sh.n, nb, Ns, tw, inv, fs);
    Ns *= R;
    CT* t = a; a = b; b = t;
  }
  __syncthreads();
  return a;
}

// spectral array view: complex element (kx, J, kz) at base[kx + sj*J + sk*kz]
// (J counted from the first stored plane)
template <class CT>
struct SpecViewT {
  CT* base;
  long sj, sk;
  int j0 = 0;  // first plane (0-based) of a launch over a window of planes
};
using SpecView = SpecViewT<double2>;

// inputs of the forward x pass: src_mode 0 reads samples of FP; 1 forms the
// divergence right-hand side of mkp.f:90-97 from ut, vt, wt; 2 forms the
// residual of that right-hand side against the 7-point operator applied to
// phi (the iterative-refinement step of the mixed-precision form)
template <class S>
struct FwdSrc {
  const S *FP, *ut, *vt, *wt;
  const double* phi;
  GridDev g;
  GridRcp rg;
  int use_rcp;
  double dt;
  const double* AC;   // [3][ny]
  double rdx2, rdz2;  // 1/dx^2, 1/dz^2 of the uniform x, z spacings
};

// FP64 divergence right-hand side at cell (I, J, K) (all three >= 1)
template <class S>
__device__ __forceinline__ double div_rhs(const Dims& d, const FwdSrc<S>& q, int I, int J, int K) {
  long c = d.P(I, J, K);
  const double du = (double)q.ut[c] - (double)q.ut[c - 1];
  const double dv = (double)q.vt[c] - (double)q.vt[c - d.sx];
  const double dw = (double)q.wt[c] - (double)q.wt[c - d.sy];
  if (q.use_rcp)
    return (du * q.rg.rdx[I] + dv * q.rg.rdy[J] + dw * q.rg.rdz[K]) * (1.0 / q.dt);
  return (du / q.g.dx[I] + dv / q.g.dy[J] + dw / q.g.dz[K]) / q.dt;
}

// The divergence right-hand side on its own, written in the sample layout
// the forward x pass reads in src_mode 0: out(i, J, k) for i = 0..nx-1,
// J = 1..ny, k = 0..nz-1, with i = 0 standing for I = nx and k = 0 for
// K = nz (the periodic wrap of P2S, p2s_fftw2d.f:5-30).  Split from the
// transform because the fused pass holds six loads per sample in flight
// for two rows at once and stays latency-bound (0.180 ms at 256x192x256);
// this streaming kernel plus the plain transform take 0.145 ms, with
// identical values (the same expression, evaluated once per cell).
template <class S>
__global__ void __launch_bounds__(128) k_div_src(Dims d, FwdSrc<S> q, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = 1 + blockIdx.y;
  const int k = blockIdx.z;
  if (i >= d.nx) return;
  const int I = (i == 0) ? d.nx : i, K = (k == 0) ? d.nz : k;
  out[d.P(i, J, k)] = div_rhs(d, q, I, J, K);
}

// ------------------------------------------------------------- x forward --
// CTA: plane J (1..ny) and `npair` row pairs starting at row 2*npair*blockIdx.y
template <class CT, class S>
__global__ void k_fft_fwd_x(FFTShape sh, int npair, Dims d, SpecViewT<CT> sv, FwdSrc<S> q,
                            int src_mode, const CT* __restrict__ tw) {
  using RT = typename CReal<CT>::T;
  extern __shared__ __align__(16) char fsm[];
  CT* smem = reinterpret_cast<CT*>(fsm);
  const int N = sh.n;
  CT* a = smem;
  CT* b = smem + (long)npair * N;
  const int J = 1 + sv.j0 + blockIdx.x;
  const int kk0 = 2 * npair * blockIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  for (int t = threadIdx.x; t < npair * N; t += blockDim.x) {
    int pr = t / N, i = t - pr * N;
    int ka = kk0 + 2 * pr, kb = ka + 1;
    double va = 0.0, vb = 0.0;
    if (src_mode == 0) {
      if (ka < nz) va = (double)q.FP[d.P(i, J, ka)];
      if (kb < nz) vb = (double)q.FP[d.P(i, J, kb)];
    } else {
      // right-hand side at the periodic image of sample (i,k)
      int I = (i == 0) ? nx : i;
      for (int h = 0; h < 2; ++h) {
        int kq = h ? kb : ka;
        if (kq >= nz) continue;
        int K = (kq == 0) ? nz : kq;
        double val = div_rhs(d, q, I, J, K);
        if (src_mode == 2) {
          // minus the operator the spectral solve inverts (mkp.f:56-84):
          // periodic second differences in x and z, AC rows in y with the
          // Neumann ghosts of PHIBC
          const double* ph = q.phi;
          long c = d.P(I, J, K);
          const double p0 = ph[c];
          const double lx = (ph[c + 1] - 2.0 * p0 + ph[c - 1]) * q.rdx2;
          const double lz = (ph[c + d.sy] - 2.0 * p0 + ph[c - d.sy]) * q.rdz2;
          const double ly = q.AC[J - 1] * ph[c - d.sx] + q.AC[J - 1 + ny] * p0 +
                            q.AC[J - 1 + 2 * ny] * ph[c + d.sx];
          val = val - (lx + ly + lz);
        }
        if (h) vb = val; else va = val;
      }
    }
    a[t] = mkc<CT>((RT)va, (RT)vb);
  }
  CT* r = fft_block(a, b, sh, npair, tw, false, N);
  const int H = N / 2 + 1;
  for (int t = threadIdx.x; t < npair * H; t += blockDim.x) {
    int pr = t / H, kx = t - pr * H;
    int ka = kk0 + 2 * pr, kb = ka + 1;
    CT Z = r[pr * N + kx];
    CT Zr = r[pr * N + ((N - kx) % N)];
    CT A = mkc<CT>((Z.x + Zr.x) * RT(0.5), (Z.y - Zr.y) * RT(0.5));
    CT B = mkc<CT>((Z.y + Zr.y) * RT(0.5), (Zr.x - Z.x) * RT(0.5));
    if (ka < nz) sv.base[kx + sv.sj * (J - 1) + sv.sk * ka] = A;
    if (kb < nz) sv.base[kx + sv.sj * (J - 1) + sv.sk * kb] = B;
  }
}

// -------------------------------------------------------------- z passes --
// CTA: plane index jj (0..ny-1) and columns kx0..kx0+W-1
template <class CT>
__global__ void k_fft_z(FFTShape sh, int W, int H, SpecViewT<CT> sv, const CT* __restrict__ tw,
                        int inv, double nrm, int rmul) {
  using RT = typename CReal<CT>::T;
  extern __shared__ __align__(16) char fsm[];
  CT* smem = reinterpret_cast<CT*>(fsm);
  const int N = sh.n;
  const int FS = N + 1;
  CT* a = smem;
  CT* b = smem + (long)W * FS;
  const int jj = sv.j0 + blockIdx.y;
  const int kx0 = blockIdx.x * W;
  for (int t = threadIdx.x; t < W * N; t += blockDim.x) {
    int c = t % W, kz = t / W;
    int kx = kx0 + c;
    CT v = mkc<CT>(RT(0), RT(0));
    if (kx < H) v = sv.base[kx + sv.sj * jj + sv.sk * kz];
    a[c * FS + kz] = v;
  }
  CT* r = fft_block(a, b, sh, W, tw, inv != 0, FS);
  const RT rn = (RT)nrm;
  for (int t = threadIdx.x; t < W * N; t += blockDim.x) {
    int c = t % W, kz = t / W;
    int kx = kx0 + c;
    if (kx >= H) continue;
    CT v = r[c * FS + kz];
    // rmul: nrm is the exact reciprocal of a power of two (the same bits)
    if (!inv && rmul) { v.x = v.x * rn; v.y = v.y * rn; }
    if (!inv && !rmul) { v.x = v.x / rn; v.y = v.y / rn; }
    sv.base[kx + sv.sj * jj + sv.sk * kz] = v;
  }
}

// ------------------------------------------------------------- x inverse --
// c2r per row pair with the S2P wrap: FP(i,J,k) = s(i mod NX, k mod NZ) for
// i = 0..NX, k = 0..NZ (p2s_fftw2d.f:205-216); with `accumulate` the
// transform is added to FP (refinement step) instead of stored
template <class CT>
__global__ void k_fft_inv_x(FFTShape sh, int npair, Dims d, SpecViewT<CT> sv, double* FP,
                            const CT* __restrict__ tw, int accumulate) {
  using RT = typename CReal<CT>::T;
  extern __shared__ __align__(16) char fsm[];
  CT* smem = reinterpret_cast<CT*>(fsm);
  const int N = sh.n;
  CT* a = smem;
  CT* b = smem + (long)npair * N;
  const int J = 1 + sv.j0 + blockIdx.x;
  const int kk0 = 2 * npair * blockIdx.y;
  const int nz = d.nz;
  const int H = N / 2 + 1;
  for (int t = threadIdx.x; t < npair * H; t += blockDim.x) {
    int pr = t / H, kx = t - pr * H;
    int ka = kk0 + 2 * pr, kb = ka + 1;
    CT A = mkc<CT>(RT(0), RT(0)), B = mkc<CT>(RT(0), RT(0));
    if (ka < nz) A = sv.base[kx + sv.sj * (J - 1) + sv.sk * ka];
    if (kb < nz) B = sv.base[kx + sv.sj * (J - 1) + sv.sk * kb];
    if (kx == 0 || 2 * kx == N) { A.y = RT(0); B.y = RT(0); }
    // Z = A + iB at kx, conj(A) + i conj(B) at N - kx
    a[pr * N + kx] = mkc<CT>(A.x - B.y, A.y + B.x);
    if (kx > 0 && 2 * kx < N) a[pr * N + (N - kx)] = mkc<CT>(A.x + B.y, B.x - A.y);
  }
  CT* r = fft_block(a, b, sh, npair, tw, true, N);
  for (int t = threadIdx.x; t < npair * (N + 1); t += blockDim.x) {
    int pr = t / (N + 1), i = t - pr * (N + 1);
    int ka = kk0 + 2 * pr, kb = ka + 1;
    CT z = r[pr * N + (i % N)];
    if (ka < nz) {
      long c = d.P(i, J, ka);
      double v = accumulate ? FP[c] + (double)z.x : (double)z.x;
      FP[c] = v;
      if (ka == 0) FP[d.P(i, J, nz)] = v;
    }
    if (kb < nz) {
      long c = d.P(i, J, kb);
      FP[c] = accumulate ? FP[c] + (double)z.y : (double)z.y;
    }
  }
}

// x forward, N = 256: a half-warp transforms one row pair (two real rows
// packed as a + ib) of plane J; 8 pairs per 128-thread CTA.  SRC is the
// source mode (0 padded samples, 1 divergence, 2 refinement residual) as a
// template parameter, so the plain-sample pass of the resident step carries
// none of the other modes' registers: 96 of them, so five CTAs fit an SM.
template <class CT, class S, int SRC>
__global__ void __launch_bounds__(128, SRC == 0 ? 5 : 4) k_fft256_fwd_x(Dims d, SpecViewT<CT> sv, FwdSrc<S> q,
                                                      const CT* __restrict__ tw) {
  constexpr int src_mode = SRC;
  using RT = typename CReal<CT>::T;
  constexpr int N = 256, FS = 17;
  __shared__ CT sbuf[8][16 * FS];
  const int h = threadIdx.x >> 4, b = threadIdx.x & 15;
  CT* S_ = sbuf[h];
  const int J = 1 + sv.j0 + blockIdx.x;
  const int ka = 2 * (blockIdx.y * 8 + h), kb = ka + 1;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  CT v[16];
#pragma unroll
  for (int a = 0; a < 16; ++a) {
    const int i = 16 * a + b;
    double va = 0.0, vb = 0.0;
    if (src_mode == 0) {
      if (ka < nz) va = (double)q.FP[d.P(i, J, ka)];
      if (kb < nz) vb = (double)q.FP[d.P(i, J, kb)];
    } else {
      const int I = (i == 0) ? nx : i;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int kq = hh ? kb : ka;
        if (kq >= nz) continue;
        const int K = (kq == 0) ? nz : kq;
        double val = div_rhs(d, q, I, J, K);
        if (src_mode == 2) {
          const double* ph = q.phi;
          const long c = d.P(I, J, K);
          const double p0 = ph[c];
          const double lx = (ph[c + 1] - 2.0 * p0 + ph[c - 1]) * q.rdx2;
          const double lz = (ph[c + d.sy] - 2.0 * p0 + ph[c - d.sy]) * q.rdz2;
          const double ly = q.AC[J - 1] * ph[c - d.sx] + q.AC[J - 1 + ny] * p0 +
                            q.AC[J - 1 + 2 * ny] * ph[c + d.sx];
          val = val - (lx + ly + lz);
        }
        if (hh) vb = val; else va = val;
      }
    }
    v[a] = mkc<CT>((RT)va, (RT)vb);
  }
  fft256_inner(v, b, tw, false);
#pragma unroll
  for (int c = 0; c < 16; ++c) S_[b * FS + c] = v[c];
  __syncwarp();
#pragma unroll
  for (int bb = 0; bb < 16; ++bb) v[bb] = S_[bb * FS + b];  // this thread is now c = b
  __syncwarp();
  dft16(v, false);
  // X[b + 16e] in natural order for the Hermitian split
#pragma unroll
  for (int e = 0; e < 16; ++e) S_[b + 16 * e] = v[e];
  __syncwarp();
#pragma unroll
  for (int qq = 0; qq <= 8; ++qq) {
    const int kx = b + 16 * qq;
    if (kx > N / 2) break;
    const CT Z = S_[kx], Zr = S_[(N - kx) & (N - 1)];
    const CT A = mkc<CT>((Z.x + Zr.x) * RT(0.5), (Z.y - Zr.y) * RT(0.5));
    const CT B = mkc<CT>((Z.y + Zr.y) * RT(0.5), (Zr.x - Z.x) * RT(0.5));
    if (ka < nz) sv.base[kx + sv.sj * (J - 1) + sv.sk * ka] = A;
    if (kb < nz) sv.base[kx + sv.sj * (J - 1) + sv.sk * kb] = B;
  }
}

// x inverse, N = 256, with the S2P wrap (and `accumulate` as k_fft_inv_x).
// Five CTAs per SM (96 registers, a few spilled): 0.059 -> 0.054 ms per pass
// at 256x192x256 against four CTAs at 124 registers; the forward x pass
// measured slower with the same cap and keeps four.
template <class CT>
__global__ void __launch_bounds__(128, 5) k_fft256_inv_x(Dims d, SpecViewT<CT> sv, double* FP,
                                                      const CT* __restrict__ tw, int accumulate) {
  using RT = typename CReal<CT>::T;
  constexpr int N = 256, FS = 17;
  __shared__ CT sbuf[8][16 * FS];
  const int h = threadIdx.x >> 4, b = threadIdx.x & 15;
  CT* S_ = sbuf[h];
  const int J = 1 + sv.j0 + blockIdx.x;
  const int ka = 2 * (blockIdx.y * 8 + h), kb = ka + 1;
  const int nz = d.nz;
#pragma unroll
  for (int qq = 0; qq <= 8; ++qq) {
    const int kx = b + 16 * qq;
    if (kx > N / 2) break;
    CT A = mkc<CT>(RT(0), RT(0)), B = mkc<CT>(RT(0), RT(0));
    if (ka < nz) A = sv.base[kx + sv.sj * (J - 1) + sv.sk * ka];
    if (kb < nz) B = sv.base[kx + sv.sj * (J - 1) + sv.sk * kb];
    if (kx == 0 || 2 * kx == N) { A.y = RT(0); B.y = RT(0); }
    // Z = A + iB at kx, conj(A) + i conj(B) at N - kx
    S_[kx] = mkc<CT>(A.x - B.y, A.y + B.x);
    if (kx > 0 && 2 * kx < N) S_[N - kx] = mkc<CT>(A.x + B.y, B.x - A.y);
  }
  __syncwarp();
  CT v[16];
#pragma unroll
  for (int a = 0; a < 16; ++a) v[a] = S_[16 * a + b];
  __syncwarp();
  fft256_inner(v, b, tw, true);
#pragma unroll
  for (int c = 0; c < 16; ++c) S_[b * FS + c] = v[c];
  __syncwarp();
#pragma unroll
  for (int bb = 0; bb < 16; ++bb) v[bb] = S_[bb * FS + b];
  dft16(v, true);
  // thread b holds z(i = b + 16e)
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int i = b + 16 * e;
    const CT z = v[e];
    if (ka < nz) {
      const long c = d.P(i, J, ka);
      const double val = accumulate ? FP[c] + (double)z.x : (double)z.x;
      FP[c] = val;
      if (i == 0) FP[d.P(N, J, ka)] = val;
      if (ka == 0) {
        FP[d.P(i, J, nz)] = val;
        if (i == 0) FP[d.P(N, J, nz)] = val;
      }
    }
    if (kb < nz) {
      const long c = d.P(i, J, kb);
      const double val = accumulate ? FP[c] + (double)z.y : (double)z.y;
      FP[c] = val;
      if (i == 0) FP[d.P(N, J, kb)] = val;
    }
  }
}

// z pass, N = 256: a CTA transforms 16 adjacent kx columns of one plane
// (column group g0 + blockIdx.x); thread (col, b) holds x[16a + b] of its
// column (loads coalesced over col).  NORM, the forward pass's division by
// NX*NZ: 2 divides; 1 multiplies by the reciprocal, which the host passes
// only when NX*NZ is a power of two (then the product is the correctly
// rounded quotient, the same bits without a division sequence per value);
// 0 none (the inverse pass).
template <class CT, int NORM>
__global__ void __launch_bounds__(256) k_fft256_z(int H, SpecViewT<CT> sv,
                                                  const CT* __restrict__ tw, double nrm,
                                                  int g0) {
  constexpr bool inv = NORM == 0;
  using RT = typename CReal<CT>::T;
  constexpr int FS = 17;
  extern __shared__ __align__(16) char fsm[];
  CT* S_ = reinterpret_cast<CT*>(fsm);  // [c][b][col], col stride 1, b stride 17
  const int col = threadIdx.x & 15, b = threadIdx.x >> 4;
  const int jj = sv.j0 + blockIdx.y;
  const int kx = (g0 + blockIdx.x) * 16 + col;
  const bool ok = kx < H;
  CT* base = sv.base + kx + sv.sj * jj;
  CT v[16];
#pragma unroll
  for (int a = 0; a < 16; ++a) v[a] = ok ? base[sv.sk * (16 * a + b)] : mkc<CT>(RT(0), RT(0));
  fft256_inner(v, b, tw, inv != 0);
#pragma unroll
  for (int c = 0; c < 16; ++c) S_[(c * 16 + b) * FS + col] = v[c];
  __syncthreads();
  const int c = b;  // this thread now runs the outer DFT of index c
#pragma unroll
  for (int bb = 0; bb < 16; ++bb) v[bb] = S_[(c * 16 + bb) * FS + col];
  dft16(v, inv != 0);
  if (!ok) return;
  const RT rn = (RT)nrm;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    CT w = v[e];
    if (NORM == 2) { w.x = w.x / rn; w.y = w.y / rn; }
    if (NORM == 1) { w.x = w.x * rn; w.y = w.y * rn; }
    base[sv.sk * (c + 16 * e)] = w;
  }
}

// ------------------------------------------------------ SPN / SP0B (y) --
// Two threads per (kx, kz) system, on adjacent lanes: one runs the real part
// of the right-hand side and one the imaginary part (CTRIDIAG's matrix is
// real, tridiag.f:43-58, so both run the same coefficient recurrence and
// write the same value of A(I,3) to the scratch).  base points at plane
// J = 1 (svj, svk: complex strides); scratch sc holds A(I,3)/A(I,2) at
// [kx + scj*(J-1) + sck*kz].  RT is the storage type of the spectrum; the
// recurrences always run in FP64 (the low wavenumbers are nearly singular
// Neumann systems, where FP32 pivots would amplify rounding by the condition
// number) and the scratch is FP64.
template <class RT>
__global__ void k_spn(int H, int ny, int nz, RT* base, long svj, long svk, double* sc, long scj,
                      long sck, const double* __restrict__ AC, const double* __restrict__ KXZ,
                      int do_spn, int do_sp0b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int kx = t >> 1, comp = t & 1;
  const int kz = blockIdx.y;
  if (kx >= H || kz >= nz) return;
  const double* AC1 = AC;
  const double* AC2 = AC + ny;
  const double* AC3 = AC + 2 * ny;
  RT* B = base + 2 * (kx + svk * kz) + comp;
  const long sj = 2 * svj;  // reals between planes
  if (kx == 0 && kz == 0) {
    if (!do_sp0b) return;
    // SP0B mkp.f:271-288; the ghost PHIT(0,NY+1,0) is set by the caller.
    // Row J reads D(J) and overwrites the slot of D(J+1) after reading it;
    // the D values are read in double-buffered batches (this single thread
    // would otherwise wait one memory latency per row, longer than all the
    // other systems together)
    constexpr int SB = 16;
    double pm = 0.0, pc = 0.0;
    double Dj = (double)B[0];  // D(1)
    B[0] = (RT)pc;             // PHIT(0,1,0) = 0
    auto load0 = [&](double (&v)[SB], int J0) {
#pragma unroll
      for (int q = 0; q < SB; ++q)
        if (J0 + q <= ny - 1) v[q] = (double)B[sj * (J0 + q)];  // D(J+1)
    };
    auto march = [&](const double (&v)[SB], int J0) {
#pragma unroll
      for (int q = 0; q < SB; ++q) {
        const int J = J0 + q;
        if (J <= ny - 1) {
          double a1 = AC1[J - 1], a2 = AC2[J - 1], a3 = AC3[J - 1];
          double pn = (Dj - a1 * pm - a2 * pc) / a3;
          B[sj * J] = (RT)pn;  // PHIT(0,J+1,0)
          pm = pc;
          pc = pn;
          Dj = v[q];
        }
      }
    };
    double va[SB], vb[SB];
    load0(va, 1);
    for (int J0 = 1; J0 <= ny - 1; J0 += 2 * SB) {
      load0(vb, J0 + SB);
      march(va, J0);
      load0(va, J0 + 2 * SB);
      march(vb, J0 + SB);
    }
    return;
  }
  if (!do_spn) return;
  // SPN mkp.f:239-254 + CTRIDIAG tridiag.f:47-56, with one reciprocal of the
  // pivot per row.  The right-hand side is read in batches, double-buffered
  // so the loads of the next batch are in flight while this one is
  // eliminated.
  const double kxz = KXZ[kx + (long)H * kz];
  double* s3 = sc + kx + sck * kz;
  const int NN = ny;
  double a2 = AC2[0] - kxz;
  if (NN == 1) { a2 = a2 + AC1[0]; a2 = a2 + AC3[0]; }
  else a2 = a2 + AC1[0];  // AA(1,2) += AA(1,1)
  double b = (double)B[0];
  constexpr int FB = 16;
  auto load_f = [&](double (&v)[FB], int I0) {
#pragma unroll
    for (int q = 0; q < FB; ++q)
      if (I0 + q <= NN - 1) v[q] = (double)B[sj * (I0 + q)];
  };
  auto elim = [&](const double (&v)[FB], int I0) {
#pragma unroll
    for (int q = 0; q < FB; ++q) {
      const int I = I0 + q;
      if (I <= NN - 1) {
        const double r = 1.0 / a2;
        const double a3 = AC3[I - 1] * r;
        b = b * r;
        B[sj * (I - 1)] = (RT)b;
        s3[scj * (I - 1)] = a3;
        const double a1n = AC1[I];
        double a2n = AC2[I] - kxz;
        if (I + 1 == NN) a2n = a2n + AC3[NN - 1];  // AA(NY,2) += AA(NY,3)
        a2 = a2n - a1n * a3;
        b = v[q] - a1n * b;
      }
    }
  };
  {
    double va[FB], vb[FB];
    load_f(va, 1);
    for (int I0 = 1; I0 <= NN - 1; I0 += 2 * FB) {
      load_f(vb, I0 + FB);
      elim(va, I0);
      load_f(va, I0 + 2 * FB);
      elim(vb, I0 + FB);
    }
  }
  b = b / a2;
  B[sj * (NN - 1)] = (RT)b;
  constexpr int BB = 8;
  auto load_b = [&](double (&bi)[BB], double (&av)[BB], int I0) {
#pragma unroll
    for (int q = 0; q < BB; ++q)
      if (I0 - q >= 1) {
        bi[q] = (double)B[sj * (I0 - q - 1)];
        av[q] = s3[scj * (I0 - q - 1)];
      }
  };
  auto back = [&](const double (&bi)[BB], const double (&av)[BB], int I0) {
#pragma unroll
    for (int q = 0; q < BB; ++q) {
      const int I = I0 - q;
      if (I >= 1) {
        b = bi[q] - av[q] * b;
        B[sj * (I - 1)] = (RT)b;
      }
    }
  };
  {
    double ba[BB], aa[BB], bb[BB], ab[BB];
    load_b(ba, aa, NN - 1);
    for (int I0 = NN - 1; I0 >= 1; I0 -= 2 * BB) {
      load_b(bb, ab, I0 - BB);
      back(ba, aa, I0);
      load_b(ba, aa, I0 - 2 * BB);
      back(bb, ab, I0 - BB);
    }
  }
}

// ------------------------------------- SPN: two-ended Thomas (fast form) --
// The Neumann-folded SPN matrix of wavenumber (kx, kz) (mkp.f:239-254)
// depends only on the grid (AC) and KXZ.  Its rows are split at m = ny/2:
// rows 0..m-1 are eliminated downwards, x(r) = y(r) - cT(r) x(r+1), and rows
// m..ny-1 upwards, x(r) = z(r) - cB(r) x(r-1); the two meet in a 2x2 system
// for x(m-1), x(m).  The pivot reciprocals im(r) (top pivots above m, bottom
// pivots from m on) are tabulated once per context, real [kz][r][kx] with
// pitch Hp; cT(r) = AC3(r) im(r), cB(r) = AC1(r) im(r).  The mean mode keeps
// SP0B's forward marching (mkp.f:263-290).
__global__ void k_spn_tables(int H, int Hp, int ny, int nz, int m, const double* __restrict__ AC,
                             const double* __restrict__ KXZ, double* im) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int kz = blockIdx.y;
  if (kx >= H) return;
  const double* AC1 = AC;
  const double* AC2 = AC + ny;
  const double* AC3 = AC + 2 * ny;
  const long sr = Hp, base = kx + (long)Hp * ny * kz;
  if (kx == 0 && kz == 0) {
    for (int r = 0; r < ny; ++r) im[base + sr * r] = 0.0;
    return;
  }
  const double kxz = KXZ[kx + (long)H * kz];
  auto diag = [&](int r) {
    double b = AC2[r] - kxz;
    if (r == 0) b = b + AC1[0];
    if (r == ny - 1) b = b + AC3[ny - 1];
    return b;
  };
  double cp = 0.0;
  for (int r = 0; r < m; ++r) {
    const double mm = (r == 0) ? diag(0) : diag(r) - AC1[r] * cp;
    const double w = 1.0 / mm;
    im[base + sr * r] = w;
    cp = AC3[r] * w;
  }
  cp = 0.0;
  for (int r = ny - 1; r >= m; --r) {
    const double mm = (r == ny - 1) ? diag(r) : diag(r) - AC3[r] * cp;
    const double w = 1.0 / mm;
    im[base + sr * r] = w;
    cp = AC1[r] * w;
  }
}

// asynchronous global -> shared copies of 4 or 8 bytes (cp.async, waited
// for by the issuing thread with cp.async.wait_all: no spin loop)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(BYTES)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
}

// The recurrences of the two-ended solve with one explicit rounding per
// operation, shared by k_spn_babe and k_spn_babe_tma so the two give the same
// bits: elimination y(q) = (d(q) - cf y(q-1)) im(q), back substitution
// x(r) = y(r) - (cf im) x(r+-1), the 2x2 meeting of the halves and SP0B's
// marching row (mkp.f:271-288).  The marching row multiplies by the
// reciprocal ra3 = 1/AC3 instead of dividing by AC3: the reciprocals do not
// depend on the recurrence, so they leave its serial chain (one lane marches
// all ny rows of the mean mode, the longest chain of the solve).
__device__ __forceinline__ double spn_down(bool first, double d, double cf, double y, double w) {
  return __dmul_rn(first ? d : __fma_rn(-cf, y, d), w);
}
__device__ __forceinline__ double spn_up(double y, double cf, double w, double x) {
  return __fma_rn(-__dmul_rn(cf, w), x, y);
}
__device__ __forceinline__ double spn_meet(double ytop, double zbot, double cT, double cB) {
  return __ddiv_rn(__fma_rn(-cB, ytop, zbot), __fma_rn(-cB, cT, 1.0));
}
__device__ __forceinline__ double sp0b_row(double Dj, double pm, double pc, double a1, double a2,
                                           double ra3) {
  return __dmul_rn(__fma_rn(-a2, pc, __fma_rn(-a1, pm, Dj)), ra3);
}

// Four threads per (kx, kz): (re | im) x (top | bottom half), 16 systems per
// 64-thread CTA.  Each thread first issues cp.async copies of all the rows of
// its half (the spectrum values; the comp-0 thread of each half also the
// pivot reciprocals) into shared memory, so every row is in flight at once,
// then runs its recurrence from shared memory; the back substitution writes
// the solution to global memory.  Shared memory: values [q][thread],
// pivots [q][half].
//
// Transposed use (the discrete adjoint): the SPN matrix is diag(dy)^-1 S with
// S symmetric (AC1(j) = 1/(dy12(j-1) dy(j)), AC3(j) = 1/(dy12(j) dy(j))), so
// its transposed solve is the same solve between the scalings 1/dy (pre, on
// load) and dy (post, on store); the mean mode then runs SP0B's transpose,
// a backward marching.  pre, post: null for the forward solve.
template <class RT>
__global__ void __launch_bounds__(64) k_spn_babe(int H, int ny, int nz, int m, RT* base,
                                                 long svj, long svk,
                                                 const double* __restrict__ im, long tj,
                                                 long tk, const double* __restrict__ AC,
                                                 const double* __restrict__ rAC3,
                                                 const double* __restrict__ pre,
                                                 const double* __restrict__ post, int g0) {
  extern __shared__ __align__(16) unsigned char spn_sm[];
  const int rmax = ny - m;  // rows of the longer (bottom) half
  RT* vs = reinterpret_cast<RT*>(spn_sm);                                  // [rmax][64]
  double* ws = reinterpret_cast<double*>(spn_sm + (((size_t)rmax * 64 * sizeof(RT) + 15) & ~(size_t)15));  // [rmax][32]
  double* acs = ws + (size_t)rmax * 32;  // AC1 (ny), AC3 (ny)
  const int lt = threadIdx.x;
  for (int r = lt; r < ny; r += 64) {
    acs[r] = AC[r];
    acs[ny + r] = AC[2 * ny + r];
  }
  __syncthreads();
  const int comp = lt & 1, part = (lt >> 1) & 1, hs = lt >> 1;
  const int kx = (g0 + blockIdx.x) * 16 + (lt >> 2);
  const int kz = blockIdx.y;
  const bool mean = (kx == 0 && kz == 0);
  const bool valid = kx < H && !mean;
  const double* AC1 = AC;
  const double* AC3 = AC + 2 * ny;
  const long sj = 2 * svj;
  RT* B = base + 2 * ((long)(kx < H ? kx : 0) + svk * kz) + comp;
  const double* IM = im + (kx < H ? kx : 0) + tk * kz;
  const int cnt = part ? ny - m : m;
  auto row = [&](int q) { return part ? ny - 1 - q : q; };
  // the mean mode's column (all ny rows) is staged in the columns of its
  // top and bottom threads: row q at vs[q][lt] for q < rmax, else at
  // vs[q - rmax][lt + 2]
  auto mean_slot = [&](int q) -> RT& {
    return q < rmax ? vs[q * 64 + lt] : vs[(q - rmax) * 64 + lt + 2];
  };
  if (valid) {
    for (int q = 0; q < cnt; ++q) {
      const int r = row(q);
      cp_async<sizeof(RT)>(&vs[q * 64 + lt], &B[sj * r]);
      if (comp == 0) cp_async<8>(&ws[q * 32 + hs], &IM[tj * r]);
    }
  } else if (mean && part == 0) {
    for (int q = 0; q < ny; ++q) cp_async<sizeof(RT)>(&mean_slot(q), &B[sj * q]);
  }
  cp_async_wait_all();
  __syncwarp();
  if (mean && part == 0 && !pre) {
    // SP0B mkp.f:271-288 (phi(1) = 0, forward marching; see k_spn) from the
    // staged column
    const double* AC2 = AC + ny;
    double pm = 0.0, pc = 0.0;
    double Dj = (double)mean_slot(0);
    B[0] = (RT)0.0;
#pragma unroll 4
    for (int J = 1; J <= ny - 1; ++J) {
      const double Dn = (double)mean_slot(J);
      const double pn = sp0b_row(Dj, pm, pc, AC1[J - 1], AC2[J - 1],
                                 rAC3 ? rAC3[J - 1] : 1.0 / AC3[J - 1]);
      B[sj * J] = (RT)pn;
      pm = pc;
      pc = pn;
      Dj = Dn;
    }
  } else if (mean && part == 0) {
    // SP0B transposed: t(J) = (phibar(J+1) - AC2(J+1) t(J+1) - AC1(J+2) t(J+2)) / AC3(J),
    // Dbar(J) = t(J) for J = ny-1..1, Dbar(ny) = 0
    const double* AC2 = AC + ny;
    double t1 = 0.0, t2 = 0.0;
    B[sj * (ny - 1)] = (RT)0.0;
    for (int J = ny - 1; J >= 1; --J) {
      double v = (double)mean_slot(J) - AC2[J] * t1;  // phibar(J+1) is row J
      if (J + 1 <= ny - 1) v -= AC1[J + 1] * t2;
      const double tj = __dmul_rn(v, rAC3 ? rAC3[J - 1] : 1.0 / AC3[J - 1]);
      B[sj * (J - 1)] = (RT)tj;
      t2 = t1;
      t1 = tj;
    }
  }
  // elimination: top rows 0..m-1 downwards, bottom rows ny-1..m upwards;
  // the eliminated values stay in double in place of the loaded ones when RT
  // is double, in a register-free second pass otherwise
  double y = 0.0;
  double* ys = reinterpret_cast<double*>(vs);  // used only when RT is double
  const double* cfe = acs + (part ? ny : 0);   // elimination coefficient by row
  const double* cfb = acs + (part ? 0 : ny);   // back-substitution coefficient by row
  if (valid) {
#pragma unroll 4
    for (int q = 0; q < cnt; ++q) {
      const int r = row(q);
      const double cf = cfe[r];
      const double d = pre ? (double)vs[q * 64 + lt] * pre[r + 1] : (double)vs[q * 64 + lt];
      y = spn_down(q == 0, d, cf, y, ws[q * 32 + hs]);
      if (sizeof(RT) == sizeof(double)) ys[q * 64 + lt] = y;
      else vs[q * 64 + lt] = (RT)0;  // FP32 storage: recomputed below
    }
  }
  // y(m-1) of the top thread, z(m) of the bottom thread
  const double other = __shfl_xor_sync(0xffffffffu, y, 2);
  if (!valid) return;
  const double ytop = part ? other : y;
  const double zbot = part ? y : other;
  const double cT = __dmul_rn(AC3[m - 1], part ? IM[tj * (m - 1)] : ws[(m - 1) * 32 + hs]);
  const double cB = __dmul_rn(AC1[m], part ? ws[(ny - 1 - m) * 32 + hs] : IM[tj * m]);
  const double xm = spn_meet(ytop, zbot, cT, cB);
  double x = part ? xm : __fma_rn(-cT, xm, ytop);
  B[sj * row(cnt - 1)] = (RT)(post ? x * post[row(cnt - 1) + 1] : x);
#pragma unroll 4
  for (int q = cnt - 2; q >= 0; --q) {
    const int r = row(q);
    x = spn_up(ys[q * 64 + lt], cfb[r], ws[q * 32 + hs], x);
    B[sj * r] = (RT)(post ? x * post[r + 1] : x);
  }
}

// The same two-ended solve on one tile of SPN_KT = 12 kx columns x one kz
// plane, moved by TMA: the tile's spectrum rows (box 24 reals x ny rows) and
// pivot reciprocals (box 12 x ny) arrive on one mbarrier, one warp solves it
// in shared memory and the solved values overwrite the tile in place and
// leave by one TMA store.  Lane = 16 half + kxl (kxl < 12): each lane runs the
// re and im recurrences of its half (half 0: rows 0..m-1 downwards, half 1:
// rows ny-1..m upwards), which share the pivots; a half-warp's accesses to a
// row are contiguous (no bank conflicts).  The row loads run one block of
// SPN_U rows ahead of the recurrence (register double buffering), so the
// shared-memory and L1 latencies overlap the dependent FMA chain.  Four
// 54 KB tiles fit an SM at ny = 192.  Columns kx >= H are outside both tensor
// maps (zero-filled on load, not stored); columns kx0 + ... >= kx1 (the end of
// a kx slice) are not solved and go back unchanged.  The mean mode's lane
// marches SP0B on the tile's kx = 0 column.  Forward solve only (the
// transposed solve keeps k_spn_babe).  Bounded waits: a TMA copy that does
// not arrive sets g_spn2_wait_err and the tile is not stored.
constexpr int SPN_KT = 12, SPN_U = 8;
// One sweep of the two-ended recurrence over n rows of a lane's half: row j
// of the sweep is v[j sv], w[j sv], c[j sc].  DOWN: elimination y(j) =
// (d(j) - c(j) y(j-1)) w(j); else back substitution x(j) = y(j) - c(j) w(j)
// x(j-1); each result replaces the row's value.  Loads run one block of
// SPN_U rows ahead of the recurrence (two register buffers), so their
// shared-memory and L1 latencies overlap the dependent chain.
template <bool DOWN>
__device__ __forceinline__ void spn_sweep(double2* v, const double* w, const double* c, int sv,
                                          int sc, int n, double2& y) {
  constexpr int U = SPN_U;
  double2 dA[U], dB[U];
  double wA[U], wB[U], cA[U], cB[U];
  const int nb = n / U;
  auto load = [&](int b, double2* dd, double* ww, double* cc) {
    const double2* pv = v + b * U * sv;
    const double* pw = w + b * U * sv;
    const double* pc = c + b * U * sc;
#pragma unroll
    for (int k = 0; k < U; ++k) {
      dd[k] = pv[k * sv];
      ww[k] = pw[k * sv];
      cc[k] = __ldg(pc + k * sc);
    }
  };
  auto row = [&](double2 d, double cf, double wr) {
    if (DOWN) {
      y.x = spn_down(false, d.x, cf, y.x, wr);
      y.y = spn_down(false, d.y, cf, y.y, wr);
    } else {
      y.x = spn_up(d.x, cf, wr, y.x);
      y.y = spn_up(d.y, cf, wr, y.y);
    }
  };
  auto step = [&](int b, const double2* dd, const double* ww, const double* cc) {
    double2* pv = v + b * U * sv;
#pragma unroll
    for (int k = 0; k < U; ++k) {
      row(dd[k], cc[k], ww[k]);
      pv[k * sv] = y;
    }
  };
  if (nb > 0) load(0, dA, wA, cA);
  int b = 0;
  for (; b + 2 <= nb; b += 2) {
    load(b + 1, dB, wB, cB);
    step(b, dA, wA, cA);
    if (b + 2 < nb) load(b + 2, dA, wA, cA);
    step(b + 1, dB, wB, cB);
  }
  if (b < nb) step(b, dA, wA, cA);
  for (int j = nb * U; j < n; ++j) {
    row(v[j * sv], __ldg(c + j * sc), w[j * sv]);
    v[j * sv] = y;
  }
}

__device__ int g_spn2_wait_err = 0;

__host__ __device__ inline size_t spn_tile_piv_off(int ny) {
  return ((size_t)ny * 2 * SPN_KT * sizeof(double) + 127) & ~(size_t)127;
}
__host__ __device__ inline size_t spn_tile_smem(int ny) {
  return spn_tile_piv_off(ny) + (size_t)ny * SPN_KT * sizeof(double) + 16;
}

__global__ void __launch_bounds__(32) k_spn_babe_tma(const __grid_constant__ CUtensorMap tv,
                                                     const __grid_constant__ CUtensorMap tp,
                                                     int H, int ny, int m,
                                                     const double* __restrict__ AC,
                                                     const double* __restrict__ rAC3, int kx0,
                                                     int kx1) {
  constexpr int KT = SPN_KT;
  extern __shared__ __align__(128) unsigned char sbt_sm[];
  double* vs = reinterpret_cast<double*>(sbt_sm);                        // [ny][2 KT]
  double* ws = reinterpret_cast<double*>(sbt_sm + spn_tile_piv_off(ny));  // [ny][KT]
  uint64_t* bar = reinterpret_cast<uint64_t*>(ws + (size_t)ny * KT);
  const int lane = threadIdx.x;
  const int kb = kx0 + KT * blockIdx.x, kz = blockIdx.y;
  const bool aligned = ((reinterpret_cast<uintptr_t>(&tv) & 63) == 0) &&
                       ((reinterpret_cast<uintptr_t>(&tp) & 63) == 0) &&
                       ((smem_u32(vs) & 127) == 0) && ((smem_u32(ws) & 127) == 0);
  if (!aligned) {
    if (lane == 0) atomicExch(&g_spn2_wait_err, 2);
    return;
  }
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
    mbar_expect_tx(bar, (unsigned)ny * 3u * KT * 8u);
    tma_load_3d(vs, &tv, 2 * kb, 0, kz, bar);
    tma_load_3d(ws, &tp, kb, 0, kz, bar);
  }
  __syncwarp();
  if (!tma_wait(bar, 0)) {
    // the copies of this tile did not arrive: record it, give them one more
    // bounded wait (the CTA's shared memory must outlive them) and store nothing
    if (lane == 0) atomicExch(&g_spn2_wait_err, 1);
    tma_wait(bar, 0);
    return;
  }
  const int kxl = lane & 15, part = lane >> 4;
  const int kx = kb + kxl;
  const bool mean = (kx == 0 && kz == 0);
  const bool valid = kxl < KT && kx < kx1 && kx < H && !mean;
  const double* AC1 = AC;
  const double* AC2 = AC + ny;
  const double* AC3 = AC + 2 * ny;
  double2* v2 = reinterpret_cast<double2*>(vs) + (kxl < KT ? kxl : 0);  // row r at v2[KT r]
  const double* w = ws + (kxl < KT ? kxl : 0);                           // row r at w[KT r]
  if (mean && part == 0) {
    // SP0B (mkp.f:271-288) on the re and im columns of kx = 0
    double2 pm = make_double2(0.0, 0.0), pc = pm, Dj = v2[0];
    v2[0] = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int J = 1; J <= ny - 1; ++J) {
      const double2 Dn = v2[KT * J];
      const double a1 = __ldg(AC1 + J - 1), a2 = __ldg(AC2 + J - 1);
      const double a3 = rAC3 ? __ldg(rAC3 + J - 1) : 1.0 / __ldg(AC3 + J - 1);
      const double2 pn = make_double2(sp0b_row(Dj.x, pm.x, pc.x, a1, a2, a3),
                                      sp0b_row(Dj.y, pm.y, pc.y, a1, a2, a3));
      v2[KT * J] = pn;
      pm = pc;
      pc = pn;
      Dj = Dn;
    }
  }
  // this lane's rows: q = 0 .. cnt-1 is row r0 + dr q
  const int cnt = part ? ny - m : m;
  const int r0 = part ? ny - 1 : 0, dr = part ? -1 : 1;
  const int sv = KT * dr;
  double2 y = make_double2(0.0, 0.0);
  if (valid) {
    // elimination (coefficient AC1 downwards, AC3 upwards): row q = 0, then
    // the sweep over q = 1 .. cnt-1
    const double* cfe = (part ? AC3 : AC1) + r0;
    double2* vb = v2 + KT * r0;
    const double* wb = w + KT * r0;
    const double2 d0 = vb[0];
    const double w0 = wb[0];
    y = make_double2(spn_down(true, d0.x, 0.0, 0.0, w0), spn_down(true, d0.y, 0.0, 0.0, w0));
    vb[0] = y;
    spn_sweep<true>(vb + sv, wb + sv, cfe + dr, sv, dr, cnt - 1, y);
  }
  // y(m-1) of the top lane, z(m) of the bottom lane
  double2 o;
  o.x = __shfl_xor_sync(0xffffffffu, y.x, 16);
  o.y = __shfl_xor_sync(0xffffffffu, y.y, 16);
  if (valid) {
    const double2 ytop = part ? o : y, zbot = part ? y : o;
    const double cT = __dmul_rn(__ldg(AC3 + m - 1), w[KT * (m - 1)]);
    const double cBm = __dmul_rn(__ldg(AC1 + m), w[KT * m]);
    const double2 xm = make_double2(spn_meet(ytop.x, zbot.x, cT, cBm),
                                    spn_meet(ytop.y, zbot.y, cT, cBm));
    double2 x = part ? xm : make_double2(__fma_rn(-cT, xm.x, ytop.x),
                                         __fma_rn(-cT, xm.y, ytop.y));
    v2[KT * (part ? m : m - 1)] = x;
    // back substitution (coefficient AC3 in the top half, AC1 in the bottom
    // half) over q = cnt-2 .. 0, from the meeting point outwards
    const int qs = r0 + dr * (cnt - 2);
    const double* cfb = (part ? AC1 : AC3) + qs;
    spn_sweep<false>(v2 + KT * qs, w + KT * qs, cfb, -sv, -dr, cnt - 1, x);
  }
  fence_async_smem();
  __syncwarp();
  if (lane == 0) {
    tma_store_3d(&tv, 2 * kb, 0, kz, vs);
    tma_store_commit();
    tma_store_wait_read();
  }
}

// ------------------------------------------------------------------ PHIBC --
// mkp.f:293-320.  Phase 0 is the first loop (y ghosts (I,0|NY+1,K), I=0..NX,
// K=1..NZ, copied from J=1|NY as they are on entry).  Phase 1 is the rest in
// closed form: for J=1..NY every x/z ghost (I,J,K) ends up equal to the
// interior cell (1+(I-1) mod NX, J, 1+(K-1) mod NZ).  Cells outside these
// sets keep their value, as in the reference.
__global__ void k_phibc(Dims d, double* PHI, int phase) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (phase == 0) {
    long nC = 2L * (nx + 1) * nz;
    if (t >= nC) return;
    int J = (t & 1) ? ny + 1 : 0;
    long r = t >> 1;
    int I = (int)(r % (nx + 1));
    int K = 1 + (int)(r / (nx + 1));
    PHI[d.P(I, J, K)] = PHI[d.P(I, J == 0 ? 1 : ny, K)];
    return;
  }
  long nA = 2L * ny * (nz + 2);  // I in {0, nx+1}, J 1..ny, K 0..nz+1
  long nB = 2L * nx * ny;        // I 1..nx, J 1..ny, K in {0, nz+1}
  int I, J, K;
  if (t < nA) {
    I = (t & 1) ? nx + 1 : 0;
    long r = t >> 1;
    J = 1 + (int)(r % ny);
    K = (int)(r / ny);
  } else if (t < nA + nB) {
    long r = t - nA;
    I = 1 + (int)(r % nx);
    r /= nx;
    J = 1 + (int)(r % ny);
    K = (r / ny) ? nz + 1 : 0;
  } else {
    return;
  }
  int mI = 1 + (I - 1 + nx) % nx;
  int mK = 1 + (K - 1 + nz) % nz;
  PHI[d.P(I, J, K)] = PHI[d.P(mI, J, mK)];
}

// --------------------------------------------------------------- launchers --
static int fft_threads(int nb_times_n) { return nb_times_n >= 2048 ? 512 : 256; }

// dynamic shared memory above 48 KB needs the per-kernel opt-in
static void smem_optin(const void* kernel, size_t bytes) {
  if (bytes > 48 * 1024)
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <class CT>
static SpecViewT<CT> spec_internal_t(const PoissonPlan& pp) {
  SpecViewT<CT> sv;
  sv.base = reinterpret_cast<CT*>(pp.spec);
  sv.sj = pp.Hp;
  sv.sk = (long)pp.Hp * pp.ny;
  return sv;
}

template <class CT> static const CT* twx_of(const PoissonPlan& pp);
template <> const double2* twx_of<double2>(const PoissonPlan& pp) {
  return reinterpret_cast<const double2*>(pp.twx);
}
template <> const float2* twx_of<float2>(const PoissonPlan& pp) {
  return reinterpret_cast<const float2*>(pp.twx_f);
}
template <class CT> static const CT* twz_of(const PoissonPlan& pp);
template <> const double2* twz_of<double2>(const PoissonPlan& pp) {
  return reinterpret_cast<const double2*>(pp.twz);
}
template <> const float2* twz_of<float2>(const PoissonPlan& pp) {
  return reinterpret_cast<const float2*>(pp.twz_f);
}

static int row_pairs(const PoissonPlan& pp) {
  int npair = 1024 / pp.nx;
  if (npair < 1) npair = 1;
  if (npair > (pp.nz + 1) / 2) npair = (pp.nz + 1) / 2;
  return npair;
}

template <class CT, class S>
static void fwd_x(const PoissonPlan& pp, const Dims& d, const FwdSrc<S>& q, int src_mode,
                  cudaStream_t s, int j0 = 0, int nj = 0) {
  if (nj <= 0) { j0 = 0; nj = pp.ny; }
  SpecViewT<CT> sv = spec_internal_t<CT>(pp);
  sv.j0 = j0;
  if (pp.nx == 256 && pp.nz % 16 == 0) {
    dim3 grid(nj, pp.nz / 16);
    count_launch();
    if (src_mode == 0)
      k_fft256_fwd_x<CT, S, 0><<<grid, 128, 0, s>>>(d, sv, q, twx_of<CT>(pp));
    else if (src_mode == 1)
      k_fft256_fwd_x<CT, S, 1><<<grid, 128, 0, s>>>(d, sv, q, twx_of<CT>(pp));
    else
      k_fft256_fwd_x<CT, S, 2><<<grid, 128, 0, s>>>(d, sv, q, twx_of<CT>(pp));
    return;
  }
  FFTShape sh = make_shape(pp.nx);
  int npair = row_pairs(pp);
  dim3 grid(nj, (pp.nz + 2 * npair - 1) / (2 * npair));
  size_t sm = 2 * (size_t)npair * pp.nx * sizeof(CT);
  smem_optin((const void*)k_fft_fwd_x<CT, S>, sm);
  count_launch();
  k_fft_fwd_x<CT, S><<<grid, fft_threads(npair * pp.nx), sm, s>>>(sh, npair, d, sv, q, src_mode,
                                                                   twx_of<CT>(pp));
}

void launch_fft_fwd_x(const PoissonPlan& pp, const Dims& d, const double* FP,
                      const double* ut, const double* vt, const double* wt,
                      const GridDev& g, double dt, int src_mode, cudaStream_t s,
                      const GridRcp* rg, int j0, int nj) {
  FwdSrc<double> q{};
  q.FP = FP; q.ut = ut; q.vt = vt; q.wt = wt; q.g = g; q.dt = dt;
  if (rg) { q.rg = *rg; q.use_rcp = 1; }
  fwd_x<double2, double>(pp, d, q, src_mode, s, j0, nj);
}

template <class S>
static void div_src(const Dims& d, const GridRcp& rg, const S* ut, const S* vt, const S* wt,
                    double dt, double* out, cudaStream_t s) {
  FwdSrc<S> q{};
  q.ut = ut; q.vt = vt; q.wt = wt; q.rg = rg; q.use_rcp = 1; q.dt = dt;
  dim3 grid((d.nx + 127) / 128, d.ny, d.nz);
  count_launch();
  k_div_src<S><<<grid, 128, 0, s>>>(d, q, out);
}
void launch_div_src(const Dims& d, const GridRcp& rg, const double* ut, const double* vt,
                    const double* wt, double dt, double* out, cudaStream_t s) {
  div_src<double>(d, rg, ut, vt, wt, dt, out, s);
}
void launch_div_src32(const Dims& d, const GridRcp& rg, const float* ut, const float* vt,
                      const float* wt, double dt, double* out, cudaStream_t s) {
  div_src<float>(d, rg, ut, vt, wt, dt, out, s);
}

// g0, ng: the groups of 16 kx columns to transform (ng = 0: all; only the
// NZ = 256 kernel takes a subset)
template <class CT>
static void fft_z(const PoissonPlan& pp, bool inverse, cudaStream_t s, int j0 = 0, int nj = 0,
                  int g0 = 0, int ng = 0) {
  if (nj <= 0) { j0 = 0; nj = pp.ny; }
  SpecViewT<CT> sv = spec_internal_t<CT>(pp);
  sv.j0 = j0;
  if (pp.nz == 256) {
    if (ng <= 0) { g0 = 0; ng = (pp.H + 15) / 16; }
    dim3 grid(ng, nj);
    size_t sm = 16 * 16 * 17 * sizeof(CT);
    const double nrm = (double)pp.nx * (double)pp.nz;
    int e2 = 0;
    const bool pow2 = frexp(nrm, &e2) == 0.5;  // nrm = 2^(e2-1)
    count_launch();
    if (inverse) {
      smem_optin((const void*)k_fft256_z<CT, 0>, sm);
      k_fft256_z<CT, 0><<<grid, 256, sm, s>>>(pp.H, sv, twz_of<CT>(pp), nrm, g0);
    } else if (pow2) {
      smem_optin((const void*)k_fft256_z<CT, 1>, sm);
      k_fft256_z<CT, 1><<<grid, 256, sm, s>>>(pp.H, sv, twz_of<CT>(pp), 1.0 / nrm, g0);
    } else {
      smem_optin((const void*)k_fft256_z<CT, 2>, sm);
      k_fft256_z<CT, 2><<<grid, 256, sm, s>>>(pp.H, sv, twz_of<CT>(pp), nrm, g0);
    }
    return;
  }
  FFTShape sh = make_shape(pp.nz);
  int W = 2048 / pp.nz;
  if (W < 1) W = 1;
  if (W > 16) W = 16;
  dim3 grid((pp.H + W - 1) / W, nj);
  size_t sm = 2 * (size_t)W * (pp.nz + 1) * sizeof(CT);
  smem_optin((const void*)k_fft_z<CT>, sm);
  count_launch();
  const double nrm = (double)pp.nx * (double)pp.nz;
  int e2 = 0;
  const bool pow2 = !inverse && frexp(nrm, &e2) == 0.5;
  k_fft_z<CT><<<grid, fft_threads(W * pp.nz), sm, s>>>(sh, W, pp.H, sv, twz_of<CT>(pp),
                                                       inverse ? 1 : 0, pow2 ? 1.0 / nrm : nrm,
                                                       pow2 ? 1 : 0);
}
void launch_fft_z(const PoissonPlan& pp, bool inverse, cudaStream_t s, int j0, int nj) {
  fft_z<double2>(pp, inverse, s, j0, nj);
}

// split row of the two-ended SPN and its shared-memory footprint (the rows
// of the longer half for 128 threads); 0 when the plan cannot use it
static size_t spn_smem(int ny, int m);
int spn_split(const PoissonPlan& pp) {
  if (pp.ny < 4) return 0;
  const int m = pp.ny / 2;
  return spn_smem(pp.ny, m) <= 200 * 1024 ? m : 0;
}

void launch_spn_tables(const PoissonPlan& pp, double* im, cudaStream_t s) {
  dim3 grid((pp.H + 63) / 64, pp.nz);
  count_launch();
  k_spn_tables<<<grid, 64, 0, s>>>(pp.H, pp.Hp, pp.ny, pp.nz, spn_split(pp), pp.AC, pp.KXZ, im);
}

static size_t spn_smem(int ny, int m) {
  const size_t r = (size_t)(ny - m);
  return ((r * 64 * sizeof(double) + 15) & ~(size_t)15) + r * 32 * sizeof(double) +
         2 * (size_t)ny * sizeof(double);
}

// g0, ng: the groups of 16 kx columns to solve (ng = 0: all)
template <class RT>
static void spn_babe(const PoissonPlan& pp, RT* spec, cudaStream_t s, int g0 = 0, int ng = 0) {
  const int m = spn_split(pp);
  const size_t sm = spn_smem(pp.ny, m);
  smem_optin((const void*)k_spn_babe<RT>, sm);
  if (ng <= 0) { g0 = 0; ng = (pp.H + 15) / 16; }
  dim3 grid(ng, pp.nz);
  count_launch();
  k_spn_babe<RT><<<grid, 64, sm, s>>>(pp.H, pp.ny, pp.nz, m, spec, pp.Hp, (long)pp.Hp * pp.ny,
                                      pp.spn_im, pp.Hp, (long)pp.Hp * pp.ny, pp.AC, pp.rAC3,
                                      nullptr, nullptr, g0);
}

// the TMA tile form of the two-ended SPN (k_spn_babe_tma) on the kx columns
// of groups g0 .. g0+ng-1 of 16 (ng = 0: all); false when the plan cannot use
// it (no pivot tables, the cp.async form asked for, more than 256 rows for
// one box, or a tensor map the driver refuses), and nothing is launched then
static bool spn_babe_tma(const PoissonPlan& pp, cudaStream_t s, int g0 = 0, int ng = 0) {
  if (!pp.spn_im || pp.spn_cp || pp.ny > 256) return false;
  const int m = spn_split(pp);
  if (m == 0) return false;
  const long sv1 = 16L * pp.Hp, sv2 = sv1 * pp.ny;  // complex rows, planes (bytes)
  const long sp1 = 8L * pp.Hp, sp2 = sp1 * pp.ny;   // pivot rows, planes
  if ((sp1 & 15) != 0 || ((uintptr_t)pp.spec & 15) != 0 || ((uintptr_t)pp.spn_im & 15) != 0)
    return false;
  CUtensorMap tv, tp;
  if (!tma_encode_3d(&tv, pp.spec, true, 2L * pp.H, pp.ny, pp.nz, sv1, sv2, 2 * SPN_KT, pp.ny,
                     1) ||
      !tma_encode_3d(&tp, pp.spn_im, true, pp.H, pp.ny, pp.nz, sp1, sp2, SPN_KT, pp.ny, 1))
    return false;
  const size_t sm = spn_tile_smem(pp.ny);
  smem_optin((const void*)k_spn_babe_tma, sm);
  const int kx0 = ng > 0 ? 16 * g0 : 0;
  const int kx1 = ng > 0 ? std::min(16 * (g0 + ng), pp.H) : pp.H;
  if (kx1 <= kx0) return true;
  count_launch();
  k_spn_babe_tma<<<dim3((kx1 - kx0 + SPN_KT - 1) / SPN_KT, pp.nz), 32, sm, s>>>(
      tv, tp, pp.H, pp.ny, m, pp.AC, pp.rAC3, kx0, kx1);
  return true;
}

int spn2_wait_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_spn2_wait_err, sizeof(int)) != cudaSuccess) return 0;
  if (v) {
    const int z = 0;
    cudaMemcpyToSymbol(g_spn2_wait_err, &z, sizeof(int));
  }
  return v;
}

// transposed SPN + SP0B (the discrete adjoint) on the FP64 spectrum: rdy, dy
// are the reciprocal and plain y spacings (index 0..ny+1); false when the plan
// has no pivot tables
bool launch_spn_transposed(const PoissonPlan& pp, const double* rdy, const double* dy,
                           cudaStream_t s) {
  if (!pp.spn_im) return false;
  const int m = spn_split(pp);
  const size_t sm = spn_smem(pp.ny, m);
  smem_optin((const void*)k_spn_babe<double>, sm);
  dim3 grid((pp.H + 15) / 16, pp.nz);
  count_launch();
  k_spn_babe<double><<<grid, 64, sm, s>>>(pp.H, pp.ny, pp.nz, m, pp.spec, pp.Hp,
                                          (long)pp.Hp * pp.ny, pp.spn_im, pp.Hp,
                                          (long)pp.Hp * pp.ny, pp.AC, pp.rAC3, rdy, dy, 0);
  return true;
}

// SPN + SP0B with the tabulated pivots (fast form); k_spn when the plan has
// no tables
void launch_spn_fast(const PoissonPlan& pp, cudaStream_t s) {
  if (!pp.spn_im) {
    launch_spn(pp, true, true, s);
    return;
  }
  if (!spn_babe_tma(pp, s)) spn_babe<double>(pp, pp.spec, s);
}

// The z transforms and the SPN between them, in nchunk slices of the kx
// column groups: z forward, SPN and z inverse of one slice run back to back,
// so the slice's spectrum (107 MB / nchunk at 256x192x256) is re-read from
// L2 instead of HBM by the second and third pass.  Every column sees the
// same operations as in the unsliced order (the passes act on disjoint
// columns), so the result is bit-identical.  Slicing needs the N = 256 z
// kernel and the tabulated SPN; otherwise the three passes run whole.
int poisson_mid_groups(const PoissonPlan& pp) {
  return (pp.nz == 256 && pp.spn_im) ? (pp.H + 15) / 16 : 0;
}
void launch_poisson_mid(const PoissonPlan& pp, int nchunk, cudaStream_t s) {
  const int G = poisson_mid_groups(pp);
  if (G == 0 || nchunk <= 1) {
    fft_z<double2>(pp, false, s);
    launch_spn_fast(pp, s);
    fft_z<double2>(pp, true, s);
    return;
  }
  if (nchunk > G) nchunk = G;
  for (int c = 0; c < nchunk; ++c) {
    const int ga = (int)((long)c * G / nchunk), gb = (int)((long)(c + 1) * G / nchunk);
    fft_z<double2>(pp, false, s, 0, 0, ga, gb - ga);
    if (!spn_babe_tma(pp, s, ga, gb - ga)) spn_babe<double>(pp, pp.spec, s, ga, gb - ga);
    fft_z<double2>(pp, true, s, 0, 0, ga, gb - ga);
  }
}

void launch_spn_f32(const PoissonPlan& pp, cudaStream_t s);
void launch_spn_fast_f32(const PoissonPlan& pp, cudaStream_t s) {
  // the FP32 spectrum keeps k_spn (FP64 recurrence); the two-ended kernel
  // keeps its eliminated values in place of FP64 loads
  launch_spn_f32(pp, s);
}

void launch_spn(const PoissonPlan& pp, bool do_spn, bool do_sp0b, cudaStream_t s) {
  dim3 grid((2 * pp.H + 63) / 64, pp.nz);
  count_launch();
  k_spn<double><<<grid, 64, 0, s>>>(pp.H, pp.ny, pp.nz, pp.spec, pp.Hp, (long)pp.Hp * pp.ny,
                                    pp.scr, pp.Hp, (long)pp.Hp * pp.ny, pp.AC, pp.KXZ,
                                    do_spn ? 1 : 0, do_sp0b ? 1 : 0);
}

// k_spn on an arbitrary spectrum view: base points at (kx=0, J=1, kz=0),
// complex strides sj, sk; the scratch sc is indexed kx + scj*(J-1) + sck*kz
void launch_spn_view(int H, int ny, int nz, double* base, long sj, long sk, double* sc,
                     long scj, long sck, const double* AC, const double* KXZ, bool do_spn,
                     bool do_sp0b, cudaStream_t s) {
  dim3 grid((2 * H + 63) / 64, nz);
  count_launch();
  k_spn<double><<<grid, 64, 0, s>>>(H, ny, nz, base, sj, sk, sc, scj, sck, AC, KXZ,
                                    do_spn ? 1 : 0, do_sp0b ? 1 : 0);
}

template <class CT>
static void inv_x(const PoissonPlan& pp, const Dims& d, double* FP, bool accumulate,
                  cudaStream_t s, int j0 = 0, int nj = 0) {
  if (nj <= 0) { j0 = 0; nj = pp.ny; }
  SpecViewT<CT> sv = spec_internal_t<CT>(pp);
  sv.j0 = j0;
  if (pp.nx == 256 && pp.nz % 16 == 0) {
    dim3 grid(nj, pp.nz / 16);
    count_launch();
    k_fft256_inv_x<CT><<<grid, 128, 0, s>>>(d, sv, FP, twx_of<CT>(pp), accumulate ? 1 : 0);
    return;
  }
  FFTShape sh = make_shape(pp.nx);
  int npair = row_pairs(pp);
  dim3 grid(nj, (pp.nz + 2 * npair - 1) / (2 * npair));
  size_t sm = 2 * (size_t)npair * pp.nx * sizeof(CT);
  smem_optin((const void*)k_fft_inv_x<CT>, sm);
  count_launch();
  k_fft_inv_x<CT><<<grid, fft_threads(npair * pp.nx), sm, s>>>(sh, npair, d, sv, FP,
                                                               twx_of<CT>(pp),
                                                               accumulate ? 1 : 0);
}
void launch_fft_inv_x(const PoissonPlan& pp, const Dims& d, double* FP, cudaStream_t s, int j0,
                      int nj) {
  inv_x<double2>(pp, d, FP, false, s, j0, nj);
}

// ---------------------------------------- mixed-precision Poisson solve --
// FP32 transforms and spectrum, FP64 SPN/SP0B recurrences, and FP64 residual
// refinement:  phi0 = S(D);  phi = phi0 + S(D - L phi0)  where S is the
// FP32-stored spectral solve and L the discrete operator it inverts.  D is
// formed in FP64 from the FP32 fields u*, v*, w*.  mode 1: D; mode 2: the
// residual D - L phi (phi with PHIBC ghosts).
void launch_fft_fwd_x_f32(const PoissonPlan& pp, const Dims& d, const GridDev& g,
                          const GridRcp& rg, const float* ut, const float* vt, const float* wt,
                          double dt, const double* phi, double dx, double dz, int mode,
                          cudaStream_t s) {
  FwdSrc<float> q{};
  q.ut = ut; q.vt = vt; q.wt = wt; q.g = g; q.rg = rg; q.use_rcp = 1; q.dt = dt;
  q.phi = phi; q.AC = pp.AC; q.rdx2 = 1.0 / (dx * dx); q.rdz2 = 1.0 / (dz * dz);
  fwd_x<float2, float>(pp, d, q, mode, s);
}
void launch_fft_z_f32(const PoissonPlan& pp, bool inverse, cudaStream_t s) {
  fft_z<float2>(pp, inverse, s);
}
void launch_spn_f32(const PoissonPlan& pp, cudaStream_t s) {
  dim3 grid((2 * pp.H + 63) / 64, pp.nz);
  count_launch();
  k_spn<float><<<grid, 64, 0, s>>>(pp.H, pp.ny, pp.nz, reinterpret_cast<float*>(pp.spec), pp.Hp,
                                   (long)pp.Hp * pp.ny, pp.scr, pp.Hp, (long)pp.Hp * pp.ny,
                                   pp.AC, pp.KXZ, 1, 1);
}
void launch_fft_inv_x_f32(const PoissonPlan& pp, const Dims& d, double* phi, bool accumulate,
                          cudaStream_t s) {
  inv_x<float2>(pp, d, phi, accumulate, s);
}

void launch_phibc(const Dims& d, double* PHI, cudaStream_t s) {
  long n0 = 2L * (d.nx + 1) * d.nz;
  long n1 = 2L * d.ny * (d.nz + 2) + 2L * d.nx * d.ny;
  count_launch();
  k_phibc<<<(unsigned)((n0 + 255) / 256), 256, 0, s>>>(d, PHI, 0);
  count_launch();
  k_phibc<<<(unsigned)((n1 + 255) / 256), 256, 0, s>>>(d, PHI, 1);
}

// internal spectrum <-> reference PHIT(0:nx/2,0:ny+1,0:nz+1) for J=1..NY,
// K=0..NZ-1
__global__ void k_spec_phit(int H, int Hp, int ny, int nz, double2* spec, double2* phit,
                            int to_phit) {
  int kx = blockIdx.x * blockDim.x + threadIdx.x;
  int jj = blockIdx.y, kz = blockIdx.z;
  if (kx >= H) return;
  long si = kx + (long)Hp * (jj + (long)ny * kz);
  long pi = kx + (long)H * ((jj + 1) + (long)(ny + 2) * kz);
  if (to_phit) phit[pi] = spec[si];
  else spec[si] = phit[pi];
}
void launch_spec_to_phit(const PoissonPlan& pp, double* phit, cudaStream_t s) {
  dim3 grid((pp.H + 63) / 64, pp.ny, pp.nz);
  count_launch();
  k_spec_phit<<<grid, 64, 0, s>>>(pp.H, pp.Hp, pp.ny, pp.nz,
                                  reinterpret_cast<double2*>(pp.spec),
                                  reinterpret_cast<double2*>(phit), 1);
}
void launch_phit_to_spec(const PoissonPlan& pp, const double* phit, cudaStream_t s) {
  dim3 grid((pp.H + 63) / 64, pp.ny, pp.nz);
  count_launch();
  k_spec_phit<<<grid, 64, 0, s>>>(pp.H, pp.Hp, pp.ny, pp.nz,
                                  reinterpret_cast<double2*>(pp.spec),
                                  const_cast<double2*>(reinterpret_cast<const double2*>(phit)),
                                  0);
}

// AC, KXZ (mkp.f:54-84) and the twiddle tables, on the host
bool poisson_plan_tables(int nx, int ny, int nz, const double* dx, const double* dy,
                         const double* dz, const double* dy12, double xl, double zl,
                         double* AC, double* KXZ, double* twx, double* twz) {
  if (!fft_size_ok(nx) || !fft_size_ok(nz)) return false;
  const double PI = 3.14159265358979312;
  int H = nx / 2 + 1;
  for (int K = 0; K <= nz; ++K) {
    double KZ = (K <= nz / 2) ? (double)K : (double)(K - nz);
    if (K <= nz - 1) KZ = KZ / zl * PI * 2.0;
    for (int I = 0; I <= nx / 2; ++I) {
      double KX = (double)I / xl * PI * 2.0;
      KXZ[I + (long)H * K] = 2.0 * (1.0 - cos(KX * dx[I])) / dx[I] / dx[I] +
                             2.0 * (1.0 - cos(KZ * dz[K])) / dz[K] / dz[K];
    }
  }
  for (int J = 1; J <= ny; ++J) {
    AC[J - 1] = 1.0 / dy12[J - 1] / dy[J];
    AC[J - 1 + 2 * ny] = 1.0 / dy12[J] / dy[J];
    AC[J - 1 + ny] = -AC[J - 1] - AC[J - 1 + 2 * ny];
  }
  const long double tp = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < nx; ++k) {
    long double a = tp * (long double)k / (long double)nx;
    twx[2 * k] = (double)cosl(a);
    twx[2 * k + 1] = (double)(-sinl(a));
  }
  for (int k = 0; k < nz; ++k) {
    long double a = tp * (long double)k / (long double)nz;
    twz[2 * k] = (double)cosl(a);
    twz[2 * k + 1] = (double)(-sinl(a));
  }
  return true;
}

}  // namespace nse
