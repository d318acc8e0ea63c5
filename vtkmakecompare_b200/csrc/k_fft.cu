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

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ double2 mul_mi(double2 a, bool inv) {
  return inv ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <int R>
__device__ __forceinline__ void dft_small(double2* v, bool inv);

template <>
__device__ __forceinline__ void dft_small<2>(double2* v, bool) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
template <>
__device__ __forceinline__ void dft_small<4>(double2* v, bool inv) {
  double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  double2 t2 = cadd(v[1], v[3]), t3 = mul_mi(csub(v[1], v[3]), inv);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}
template <>
__device__ __forceinline__ void dft_small<3>(double2* v, bool inv) {
  const double s = 0.86602540378443864676;  // sin(2 pi/3)
  double2 t = cadd(v[1], v[2]);
  double2 d = csub(v[1], v[2]);
  double2 m = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
  double2 r = mul_mi(make_double2(s * d.x, s * d.y), inv);  // -i s (v1 - v2)
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, r);
  v[2] = csub(m, r);
}
template <>
__device__ __forceinline__ void dft_small<5>(double2* v, bool inv) {
  const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
  const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
  double2 a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
  double2 b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
  double2 x0 = v[0];
  double2 p1 = make_double2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  double2 p2 = make_double2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  double2 q1 = mul_mi(make_double2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), inv);
  double2 q2 = mul_mi(make_double2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), inv);
  v[0] = make_double2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
  v[1] = cadd(p1, q1);
  v[4] = csub(p1, q1);
  v[2] = cadd(p2, q2);
  v[3] = csub(p2, q2);
}

// one Stockham stage over `nb` independent FFTs of length N stored
// contiguously (fft f at src + f*N); all threads of the block cooperate
template <int R>
__device__ __forceinline__ void stockham_stage(const double2* __restrict__ src,
                                               double2* __restrict__ dst, int N, int nb,
                                               int Ns, const double2* __restrict__ tw,
                                               bool inv, int fs) {
  int nbf = N / R;
  int total = nbf * nb;
  int tstep = N / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int f = t / nbf, j = t - f * nbf;
    const double2* in = src + (long)f * fs;
    double2* out = dst + (long)f * fs;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[j + r * nbf];
    int kj = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        double2 w = __ldg(tw + r * kj * tstep);
        if (inv) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dft_small<R>(v, inv);
    int idxD = (j / Ns) * Ns * R + kj;
#pragma unroll
    for (int r = 0; r < R; ++r) out[idxD + r * Ns] = v[r];
  }
}

// runs the full FFT; data starts in a, returns the buffer holding the result;
// FFT f occupies [f*fs, f*fs + N) (fs >= N; fs = N+1 keeps column-wise tiles
// free of shared-memory bank conflicts)
__device__ double2* fft_block(double2* a, double2* b, const FFTShape& sh, int nb,
                              const double2* tw, bool inv, int fs) {
  int Ns = 1;
  for (int s = 0; s < sh.nst; ++s) {
    int R = sh.rad[s];
    __syncthreads();
    if (R == 4) stockham_stage<4>(a, b, sh.n, nb, Ns, tw, inv, fs);
    else if (R == 2) stockham_stage<2>(a, b, sh.n, nb, Ns, tw, inv, fs);
    else if (R == 3) stockham_stage<3>(a, b, sh.n, nb, Ns, tw, inv, fs);
    else stockham_stage<5>(a, b, sh.n, nb, Ns, tw, inv, fs);
    Ns *= R;
    double2* t = a; a = b; b = t;
  }
  __syncthreads();
  return a;
}

// spectral array view: complex element (kx, J, kz) at base[kx + sj*J + sk*kz]
// (J counted from the first stored plane)
struct SpecView {
  double2* base;
  long sj, sk;
};

// ------------------------------------------------------------- x forward --
// CTA: plane J (1..ny) and `npair` row pairs starting at row 2*npair*blockIdx.y
__global__ void k_fft_fwd_x(FFTShape sh, int npair, Dims d, SpecView sv, const double* FP,
                            const double* ut, const double* vt, const double* wt, GridDev g,
                            GridRcp rg, int use_rcp, double dt, int src_mode,
                            const double2* __restrict__ tw) {
  extern __shared__ double2 smem[];
  const int N = sh.n;
  double2* a = smem;
  double2* b = smem + (long)npair * N;
  const int J = 1 + blockIdx.x;
  const int kk0 = 2 * npair * blockIdx.y;
  const int nx = d.nx, nz = d.nz;
  for (int t = threadIdx.x; t < npair * N; t += blockDim.x) {
    int pr = t / N, i = t - pr * N;
    int ka = kk0 + 2 * pr, kb = ka + 1;
    double va = 0.0, vb = 0.0;
    if (src_mode == 0) {
      if (ka < nz) va = FP[d.P(i, J, ka)];
      if (kb < nz) vb = FP[d.P(i, J, kb)];
    } else {
      // divergence RHS of mkp.f:90-97 at the periodic image of sample (i,k)
      int I = (i == 0) ? nx : i;
      for (int q = 0; q < 2; ++q) {
        int kq = q ? kb : ka;
        if (kq >= nz) continue;
        int K = (kq == 0) ? nz : kq;
        long c = d.P(I, J, K);
        double val;
        if (use_rcp)
          val = ((ut[c] - ut[c - 1]) * rg.rdx[I] + (vt[c] - vt[c - d.sx]) * rg.rdy[J] +
                 (wt[c] - wt[c - d.sy]) * rg.rdz[K]) *
                (1.0 / dt);
        else
          val = ((ut[c] - ut[c - 1]) / g.dx[I] + (vt[c] - vt[c - d.sx]) / g.dy[J] +
                 (wt[c] - wt[c - d.sy]) / g.dz[K]) /
                dt;
        if (q) vb = val; else va = val;
      }
    }
    a[t] = make_double2(va, vb);
  }
  double2* r = fft_block(a, b, sh, npair, tw, false, N);
  const int H = N / 2 + 1;
  for (int t = threadIdx.x; t < npair * H; t += blockDim.x) {
    int pr = t / H, kx = t - pr * H;
    int ka = kk0 + 2 * pr, kb = ka + 1;
    double2 Z = r[pr * N + kx];
    double2 Zr = r[pr * N + ((N - kx) % N)];
    double2 A = make_double2((Z.x + Zr.x) * 0.5, (Z.y - Zr.y) * 0.5);
    double2 B = make_double2((Z.y + Zr.y) * 0.5, (Zr.x - Z.x) * 0.5);
    if (ka < nz) sv.base[kx + sv.sj * (J - 1) + sv.sk * ka] = A;
    if (kb < nz) sv.base[kx + sv.sj * (J - 1) + sv.sk * kb] = B;
  }
}

// -------------------------------------------------------------- z passes --
// CTA: plane index jj (0..ny-1) and columns kx0..kx0+W-1
__global__ void k_fft_z(FFTShape sh, int W, int H, SpecView sv, const double2* __restrict__ tw,
                        int inv, double nrm) {
  extern __shared__ double2 smem[];
  const int N = sh.n;
  const int FS = N + 1;
  double2* a = smem;
  double2* b = smem + (long)W * FS;
  const int jj = blockIdx.y;
  const int kx0 = blockIdx.x * W;
  for (int t = threadIdx.x; t < W * N; t += blockDim.x) {
    int c = t % W, kz = t / W;
    int kx = kx0 + c;
    double2 v = make_double2(0.0, 0.0);
    if (kx < H) v = sv.base[kx + sv.sj * jj + sv.sk * kz];
    a[c * FS + kz] = v;
  }
  double2* r = fft_block(a, b, sh, W, tw, inv != 0, FS);
  for (int t = threadIdx.x; t < W * N; t += blockDim.x) {
    int c = t % W, kz = t / W;
    int kx = kx0 + c;
    if (kx >= H) continue;
    double2 v = r[c * FS + kz];
    if (!inv) { v.x = v.x / nrm; v.y = v.y / nrm; }
    sv.base[kx + sv.sj * jj + sv.sk * kz] = v;
  }
}

// ------------------------------------------------------------- x inverse --
// c2r per row pair with the S2P wrap: FP(i,J,k) = s(i mod NX, k mod NZ) for
// i = 0..NX, k = 0..NZ (p2s_fftw2d.f:205-216)
__global__ void k_fft_inv_x(FFTShape sh, int npair, Dims d, SpecView sv, double* FP,
                            const double2* __restrict__ tw) {
  extern __shared__ double2 smem[];
  const int N = sh.n;
  double2* a = smem;
  double2* b = smem + (long)npair * N;
  const int J = 1 + blockIdx.x;
  const int kk0 = 2 * npair * blockIdx.y;
  const int nz = d.nz;
  const int H = N / 2 + 1;
  for (int t = threadIdx.x; t < npair * H; t += blockDim.x) {
    int pr = t / H, kx = t - pr * H;
    int ka = kk0 + 2 * pr, kb = ka + 1;
    double2 A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
    if (ka < nz) A = sv.base[kx + sv.sj * (J - 1) + sv.sk * ka];
    if (kb < nz) B = sv.base[kx + sv.sj * (J - 1) + sv.sk * kb];
    if (kx == 0 || 2 * kx == N) { A.y = 0.0; B.y = 0.0; }
    // Z = A + iB at kx, conj(A) + i conj(B) at N - kx
    a[pr * N + kx] = make_double2(A.x - B.y, A.y + B.x);
    if (kx > 0 && 2 * kx < N) a[pr * N + (N - kx)] = make_double2(A.x + B.y, B.x - A.y);
  }
  double2* r = fft_block(a, b, sh, npair, tw, true, N);
  for (int t = threadIdx.x; t < npair * (N + 1); t += blockDim.x) {
    int pr = t / (N + 1), i = t - pr * (N + 1);
    int ka = kk0 + 2 * pr, kb = ka + 1;
    double2 z = r[pr * N + (i % N)];
    if (ka < nz) {
      FP[d.P(i, J, ka)] = z.x;
      if (ka == 0) FP[d.P(i, J, nz)] = z.x;
    }
    if (kb < nz) FP[d.P(i, J, kb)] = z.y;
  }
}

// ------------------------------------------------------ SPN / SP0B (y) --
// Two threads per (kx, kz) system, on adjacent lanes: one runs the real part
// of the right-hand side and one the imaginary part (CTRIDIAG's matrix is
// real, tridiag.f:43-58, so both run the same coefficient recurrence and
// write the same value of A(I,3) to the scratch).  sv points at plane J = 1;
// scratch sc holds A(I,3)/A(I,2) at [kx + scj*(J-1) + sck*kz].
__global__ void k_spn(int H, int ny, int nz, SpecView sv, double* sc, long scj, long sck,
                      const double* __restrict__ AC, const double* __restrict__ KXZ,
                      int do_spn, int do_sp0b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int kx = t >> 1, comp = t & 1;
  const int kz = blockIdx.y;
  if (kx >= H || kz >= nz) return;
  const double* AC1 = AC;
  const double* AC2 = AC + ny;
  const double* AC3 = AC + 2 * ny;
  double* B = reinterpret_cast<double*>(sv.base + kx + sv.sk * kz) + comp;
  const long sj = 2 * sv.sj;  // doubles between planes
  if (kx == 0 && kz == 0) {
    if (!do_sp0b) return;
    // SP0B mkp.f:271-288; the ghost PHIT(0,NY+1,0) is set by the caller
    double pm = 0.0, pc = 0.0;
    double Dn = B[0];  // D(1)
    B[0] = pc;         // PHIT(0,1,0) = 0
    for (int J = 1; J <= ny - 1; ++J) {
      double Dj = Dn;
      Dn = B[sj * J];  // D(J+1), read before it is overwritten
      double a1 = AC1[J - 1], a2 = AC2[J - 1], a3 = AC3[J - 1];
      double pn = (Dj - a1 * pm - a2 * pc) / a3;
      B[sj * J] = pn;  // PHIT(0,J+1,0)
      pm = pc;
      pc = pn;
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
  double b = B[0];
  constexpr int FB = 16;
  auto load_f = [&](double (&v)[FB], int I0) {
#pragma unroll
    for (int q = 0; q < FB; ++q)
      if (I0 + q <= NN - 1) v[q] = B[sj * (I0 + q)];
  };
  auto elim = [&](const double (&v)[FB], int I0) {
#pragma unroll
    for (int q = 0; q < FB; ++q) {
      const int I = I0 + q;
      if (I <= NN - 1) {
        const double r = 1.0 / a2;
        const double a3 = AC3[I - 1] * r;
        b = b * r;
        B[sj * (I - 1)] = b;
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
  B[sj * (NN - 1)] = b;
  constexpr int BB = 8;
  auto load_b = [&](double (&bi)[BB], double (&av)[BB], int I0) {
#pragma unroll
    for (int q = 0; q < BB; ++q)
      if (I0 - q >= 1) {
        bi[q] = B[sj * (I0 - q - 1)];
        av[q] = s3[scj * (I0 - q - 1)];
      }
  };
  auto back = [&](const double (&bi)[BB], const double (&av)[BB], int I0) {
#pragma unroll
    for (int q = 0; q < BB; ++q) {
      const int I = I0 - q;
      if (I >= 1) {
        b = bi[q] - av[q] * b;
        B[sj * (I - 1)] = b;
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

static SpecView spec_internal(const PoissonPlan& pp) {
  SpecView sv;
  sv.base = reinterpret_cast<double2*>(pp.spec);
  sv.sj = pp.Hp;
  sv.sk = (long)pp.Hp * pp.ny;
  return sv;
}

void launch_fft_fwd_x(const PoissonPlan& pp, const Dims& d, const double* FP,
                      const double* ut, const double* vt, const double* wt,
                      const GridDev& g, double dt, int src_mode, cudaStream_t s,
                      const GridRcp* rg) {
  GridRcp r{};
  if (rg) r = *rg;
  FFTShape sh = make_shape(pp.nx);
  int npair = 1024 / pp.nx;
  if (npair < 1) npair = 1;
  if (npair > (pp.nz + 1) / 2) npair = (pp.nz + 1) / 2;
  dim3 grid(pp.ny, (pp.nz + 2 * npair - 1) / (2 * npair));
  size_t sm = 2 * (size_t)npair * pp.nx * sizeof(double2);
  smem_optin((const void*)k_fft_fwd_x, sm);
  count_launch();
  k_fft_fwd_x<<<grid, fft_threads(npair * pp.nx), sm, s>>>(
      sh, npair, d, spec_internal(pp), FP, ut, vt, wt, g, r, rg ? 1 : 0, dt, src_mode,
      reinterpret_cast<const double2*>(pp.twx));
}

void launch_fft_z(const PoissonPlan& pp, bool inverse, cudaStream_t s) {
  FFTShape sh = make_shape(pp.nz);
  int W = 2048 / pp.nz;
  if (W < 1) W = 1;
  if (W > 16) W = 16;
  dim3 grid((pp.H + W - 1) / W, pp.ny);
  size_t sm = 2 * (size_t)W * (pp.nz + 1) * sizeof(double2);
  smem_optin((const void*)k_fft_z, sm);
  count_launch();
  k_fft_z<<<grid, fft_threads(W * pp.nz), sm, s>>>(sh, W, pp.H, spec_internal(pp),
                                                 reinterpret_cast<const double2*>(pp.twz),
                                                 inverse ? 1 : 0,
                                                 (double)pp.nx * (double)pp.nz);
}

void launch_spn(const PoissonPlan& pp, bool do_spn, bool do_sp0b, cudaStream_t s) {
  dim3 grid((2 * pp.H + 63) / 64, pp.nz);
  count_launch();
  k_spn<<<grid, 64, 0, s>>>(pp.H, pp.ny, pp.nz, spec_internal(pp), pp.scr, pp.Hp,
                            (long)pp.Hp * pp.ny, pp.AC, pp.KXZ, do_spn ? 1 : 0,
                            do_sp0b ? 1 : 0);
}

// k_spn on an arbitrary spectrum view: base points at (kx=0, J=1, kz=0),
// complex strides sj, sk; the scratch sc is indexed kx + scj*(J-1) + sck*kz
void launch_spn_view(int H, int ny, int nz, double* base, long sj, long sk, double* sc,
                     long scj, long sck, const double* AC, const double* KXZ, bool do_spn,
                     bool do_sp0b, cudaStream_t s) {
  SpecView sv;
  sv.base = reinterpret_cast<double2*>(base);
  sv.sj = sj;
  sv.sk = sk;
  dim3 grid((2 * H + 63) / 64, nz);
  count_launch();
  k_spn<<<grid, 64, 0, s>>>(H, ny, nz, sv, sc, scj, sck, AC, KXZ, do_spn ? 1 : 0,
                            do_sp0b ? 1 : 0);
}

void launch_fft_inv_x(const PoissonPlan& pp, const Dims& d, double* FP, cudaStream_t s) {
  FFTShape sh = make_shape(pp.nx);
  int npair = 1024 / pp.nx;
  if (npair < 1) npair = 1;
  if (npair > (pp.nz + 1) / 2) npair = (pp.nz + 1) / 2;
  dim3 grid(pp.ny, (pp.nz + 2 * npair - 1) / (2 * npair));
  size_t sm = 2 * (size_t)npair * pp.nx * sizeof(double2);
  smem_optin((const void*)k_fft_inv_x, sm);
  count_launch();
  k_fft_inv_x<<<grid, fft_threads(npair * pp.nx), sm, s>>>(
      sh, npair, d, spec_internal(pp), FP, reinterpret_cast<const double2*>(pp.twx));
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
