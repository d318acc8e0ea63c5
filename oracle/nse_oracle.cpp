/*
 * nse_oracle.cpp -- CPU oracle (test infrastructure only; see nse_oracle.h).
 *
 * A restatement of the reference routines with their operation order.  Each
 * function names the reference file:line it follows.  Build with
 *   g++ -O2 -fopenmp -ffp-contract=off -fno-fast-math -fPIC -shared
 * so that every a*b+c stays two rounded operations, like the x86-64 Fortran
 * build of the reference.
 */
#include "nse_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

int g_faithful = 0;

/* padded (0:nx+1,0:ny+1,0:nz+1) column-major index */
struct Pad {
  long sx, sy;
  Pad(int nx, int ny) : sx(nx + 2), sy((long)(nx + 2) * (ny + 2)) {}
  long operator()(long i, long j, long k) const { return i + sx * j + sy * k; }
};
/* cellvalue(1:nx,1:ny,1:nz,1:4) */
struct Cell {
  long nx, nxy, nxyz;
  Cell(int nx_, int ny_, int nz_)
      : nx(nx_), nxy((long)nx_ * ny_), nxyz((long)nx_ * ny_ * nz_) {}
  long operator()(long i, long j, long k, long n) const {
    return (i - 1) + nx * (j - 1) + nxy * (k - 1) + nxyz * (n - 1);
  }
};

/* dense scratch that models the reference's per-line a(0:n+1,0:n+1) zeroing */
void touch_dense(int n) {
  if (!g_faithful) return;
  thread_local std::vector<double> a;
  size_t m = (size_t)(n + 2) * (size_t)(n + 2);
  if (a.size() < m) a.resize(m);
  std::memset(a.data(), 0, m * sizeof(double));
  asm volatile("" ::"r"(a.data()) : "memory");
}

/* UL elimination used by implicit_uy / implicit_Ty (nse_dominik.f:1549-1570,
 * 1844-1864) on a tridiagonal matrix over rows 0..m: lo[j]=a(j,j-1),
 * di[j]=a(j,j), up[j]=a(j,j+1).  The dense matrix of the reference only ever
 * has these three diagonals touched, so banded storage gives the same
 * arithmetic. */
void ul_eliminate(int m, double* lo, double* di, double* up, double* u) {
  for (int j = m; j >= 1; --j) {  /* "from lower" */
    double aa = di[j];
    di[j] = di[j] / aa;
    lo[j] = lo[j] / aa;
    double bb = up[j - 1];
    up[j - 1] = up[j - 1] - bb * di[j];
    di[j - 1] = di[j - 1] - bb * lo[j];
    u[j] = u[j] / aa;
    u[j - 1] = u[j - 1] - bb * u[j];
  }
  for (int j = 0; j <= m - 1; ++j) {
    double aa = di[j];
    di[j] = di[j] / aa;
    double bb = lo[j + 1];
    lo[j + 1] = lo[j + 1] - bb * di[j];
    u[j] = u[j] / aa;
    u[j + 1] = u[j + 1] - bb * u[j];
  }
}

/* ---------------------------------------------------------------- FFT ---- */
/* Mixed-radix recursive decimation-in-time FFT (Cooley-Tukey, any factor; the
 * factor-p butterfly is a direct p-point DFT).  Twiddles exp(-2 pi i k/n) are
 * evaluated in long double and rounded once. */
struct FFTPlan {
  int n;
  std::vector<int> fac;
  std::vector<cplx> w;
  explicit FFTPlan(int n_) : n(n_), w(n_) {
    int m = n;
    for (int p : {4, 2, 3, 5}) {
      while (m % p == 0) { fac.push_back(p); m /= p; }
    }
    for (int p = 7; m > 1; p += 2) {
      while (m % p == 0) { fac.push_back(p); m /= p; }
    }
    const long double tp = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < n; ++k) {
      long double a = tp * (long double)k / (long double)n;
      w[k] = cplx((double)cosl(a), (double)(-sinl(a)));
    }
  }
};

void fft_rec(const cplx* in, long istride, cplx* out, int n, const FFTPlan& P,
             int wstride, int fi, bool inv) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = P.fac[fi];
  int m = n / p;
  for (int q = 0; q < p; ++q)
    fft_rec(in + q * istride, istride * p, out + (long)q * m, m, P, wstride * p, fi + 1, inv);
  cplx tmp[64];
  std::vector<cplx> big;
  cplx* t = tmp;
  if (p > 64) { big.resize(p); t = big.data(); }
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) t[q] = out[(long)q * m + k];
    for (int s = 0; s < p; ++s) {
      cplx acc = t[0];
      for (int q = 1; q < p; ++q) {
        long e = ((long)q * (k + (long)m * s)) % n;
        cplx tw = P.w[(e * wstride) % P.n];
        if (inv) tw = std::conj(tw);
        acc += t[q] * tw;
      }
      out[k + (long)m * s] = acc;
    }
  }
}

void fft(const FFTPlan& P, const cplx* in, cplx* out, bool inv) {
  fft_rec(in, 1, out, P.n, P, 1, 0, inv);
}

}  // namespace

extern "C" {

void or_set_faithful(int on) { g_faithful = on; }
int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* SET_C nse_dominik.f:553-607 */
static void set_c_dir(int n, double L, double* X, double* X12, double* D, double* D12) {
  for (int i = 0; i <= n + 1; ++i) {
    X12[i] = L * (double)i / (double)n;
    X[i] = L * ((double)i - 0.50) / (double)n;
  }
  for (int i = 0; i <= n; ++i) D12[i] = X[i + 1] - X[i];
  D12[n + 1] = 2.0 * (X12[n + 1] - X[n + 1]);
  for (int i = 1; i <= n + 1; ++i) D[i] = X12[i] - X12[i - 1];
  D[0] = D[1];
  D[n + 1] = D[n];
}

void or_set_c(int nx, int ny, int nz, double* x, double* x12, double* y, double* y12,
              double* z, double* z12, double* dx, double* dx12, double* dy, double* dy12,
              double* dz, double* dz12, double xl, double yl, double zl) {
  set_c_dir(nx, xl, x, x12, dx, dx12);
  set_c_dir(ny, yl, y, y12, dy, dy12);
  set_c_dir(nz, zl, z, z12, dz, dz12);
}

/* SET_C variant with y faces y12(j) = y0 + yl/2 (1 + tanh(g(2j/ny-1))/tanh g),
 * j=0..ny; ghost faces and centres mirror the wall spacing; the spacing
 * formulas are those of nse_dominik.f:586-594. */
void or_set_c_stretched(int nx, int ny, int nz, double* x, double* x12, double* y,
                        double* y12, double* z, double* z12, double* dx, double* dx12,
                        double* dy, double* dy12, double* dz, double* dz12, double xl,
                        double yl, double zl, double y0, double gamma) {
  set_c_dir(nx, xl, x, x12, dx, dx12);
  set_c_dir(nz, zl, z, z12, dz, dz12);
  if (gamma == 0.0) {
    set_c_dir(ny, yl, y, y12, dy, dy12);
    for (int j = 0; j <= ny + 1; ++j) { y[j] += y0; y12[j] += y0; }
    return;
  }
  double tg = std::tanh(gamma);
  for (int j = 0; j <= ny; ++j)
    y12[j] = y0 + 0.5 * yl * (1.0 + std::tanh(gamma * (2.0 * j / ny - 1.0)) / tg);
  y12[ny + 1] = 2.0 * y12[ny] - y12[ny - 1];
  for (int j = 1; j <= ny; ++j) y[j] = 0.5 * (y12[j - 1] + y12[j]);
  y[0] = 2.0 * y12[0] - y[1];
  y[ny + 1] = 2.0 * y12[ny] - y[ny];
  for (int j = 0; j <= ny; ++j) dy12[j] = y[j + 1] - y[j];
  dy12[ny + 1] = 2.0 * (y12[ny + 1] - y[ny + 1]);
  for (int j = 1; j <= ny + 1; ++j) dy[j] = y12[j] - y12[j - 1];
  dy[0] = dy[1];
  dy[ny + 1] = dy[ny];
}

/* SET_BC nse_dominik.f:611-753.  Extension: the T wall ghosts become
 * 2*T_wall - T_interior when tbot/ttop are non-zero (the reference's
 * -1*T is the T_wall=0 case, nse_dominik.f:739-740). */
void or_set_bc(double* U, double* V, double* W, double* P, int nx, int ny, int nz,
               double* T, double tbot, double ttop) {
  Pad F(nx, ny);
  double* fl[5] = {U, V, W, P, T};
  for (int f = 0; f < 5; ++f) {
    double* A = fl[f];
    for (int k = 0; k <= nz + 1; ++k)
      for (int j = 0; j <= ny + 1; ++j) {
        A[F(0, j, k)] = A[F(nx, j, k)];
        A[F(nx + 1, j, k)] = A[F(1, j, k)];
      }
    for (int k = 0; k <= nz + 1; ++k)
      for (int i = 0; i <= nx + 1; ++i) {
        if (f == 0 || f == 2) {
          A[F(i, 0, k)] = -1.0 * A[F(i, 1, k)];
          A[F(i, ny + 1, k)] = -1.0 * A[F(i, ny, k)];
        } else if (f == 1) {
          A[F(i, 0, k)] = 0.0;
          A[F(i, ny, k)] = 0.0;
        } else if (f == 3) {
          A[F(i, 0, k)] = A[F(i, 1, k)];
          A[F(i, ny + 1, k)] = A[F(i, ny, k)];
        } else {
          A[F(i, 0, k)] = (tbot == 0.0) ? -1.0 * A[F(i, 1, k)] : 2.0 * tbot - A[F(i, 1, k)];
          A[F(i, ny + 1, k)] =
              (ttop == 0.0) ? -1.0 * A[F(i, ny, k)] : 2.0 * ttop - A[F(i, ny, k)];
        }
      }
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx + 1; ++i) {
        A[F(i, j, 0)] = A[F(i, j, nz)];
        A[F(i, j, nz + 1)] = A[F(i, j, 1)];
      }
  }
}

/* SET_CONVECT nse_dominik.f:757-831; the body force (1.0 at :785) is `force` */
void or_set_convect(const double* U, double* U_V, const double* V, double* V_V,
                    const double* W, double* W_V, double DT, int nx, int ny, int nz,
                    const double* DX, const double* DY, const double* DZ,
                    const double* DX12, const double* DY12, const double* DZ12,
                    double force) {
  Pad F(nx, ny);
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        double U1 = ((U[F(I, J, K)] + U[F(I + 1, J, K)]) * (U[F(I, J, K)] + U[F(I + 1, J, K)]) -
                     (U[F(I, J, K)] + U[F(I - 1, J, K)]) * (U[F(I, J, K)] + U[F(I - 1, J, K)])) /
                    DX12[I];
        double U2 = ((V[F(I + 1, J, K)] * DX[I + 1] + V[F(I, J, K)] * DX[I]) *
                         (U[F(I, J + 1, K)] + U[F(I, J, K)]) -
                     (V[F(I + 1, J - 1, K)] * DX[I + 1] + V[F(I, J - 1, K)] * DX[I]) *
                         (U[F(I, J, K)] + U[F(I, J - 1, K)])) /
                    DX12[I] / DY[J];
        double U3 = ((W[F(I + 1, J, K)] * DX[I + 1] + W[F(I, J, K)] * DX[I]) *
                         (U[F(I, J, K + 1)] + U[F(I, J, K)]) -
                     (W[F(I + 1, J, K - 1)] * DX[I + 1] + W[F(I, J, K - 1)] * DX[I]) *
                         (U[F(I, J, K)] + U[F(I, J, K - 1)])) /
                    DX12[I] / DZ[K];
        U_V[F(I, J, K)] = 0.25 * (-U1 - U2 - U3) * DT + force * DT;
      }
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        double V1 = ((U[F(I, J + 1, K)] * DY[J + 1] + U[F(I, J, K)] * DY[J]) *
                         (V[F(I + 1, J, K)] + V[F(I, J, K)]) -
                     (U[F(I - 1, J + 1, K)] * DY[J + 1] + U[F(I - 1, J, K)] * DY[J]) *
                         (V[F(I, J, K)] + V[F(I - 1, J, K)])) /
                    DY12[J] / DX[I];
        double V2 = ((V[F(I, J, K)] + V[F(I, J + 1, K)]) * (V[F(I, J, K)] + V[F(I, J + 1, K)]) -
                     (V[F(I, J, K)] + V[F(I, J - 1, K)]) * (V[F(I, J, K)] + V[F(I, J - 1, K)])) /
                    DY12[J];
        double V3 = ((W[F(I, J + 1, K)] * DY[J + 1] + W[F(I, J, K)] * DY[J]) *
                         (V[F(I, J, K + 1)] + V[F(I, J, K)]) -
                     (W[F(I, J + 1, K - 1)] * DY[J + 1] + W[F(I, J, K - 1)] * DY[J]) *
                         (V[F(I, J, K)] + V[F(I, J, K - 1)])) /
                    DY12[J] / DZ[K];
        V_V[F(I, J, K)] = 0.25 * (-V1 - V2 - V3) * DT;
      }
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        double W1 = ((U[F(I, J, K + 1)] * DZ[K + 1] + U[F(I, J, K)] * DZ[K]) *
                         (W[F(I + 1, J, K)] + W[F(I, J, K)]) -
                     (U[F(I - 1, J, K + 1)] * DZ[K + 1] + U[F(I - 1, J, K)] * DZ[K]) *
                         (W[F(I, J, K)] + W[F(I - 1, J, K)])) /
                    DZ12[K] / DX[I];
        double W2 = ((V[F(I, J, K + 1)] * DZ[K + 1] + V[F(I, J, K)] * DZ[K]) *
                         (W[F(I, J + 1, K)] + W[F(I, J, K)]) -
                     (V[F(I, J - 1, K + 1)] * DZ[K + 1] + V[F(I, J - 1, K)] * DZ[K]) *
                         (W[F(I, J, K)] + W[F(I, J - 1, K)])) /
                    DZ12[K] / DY[J];
        double W3 = ((W[F(I, J, K)] + W[F(I, J, K + 1)]) * (W[F(I, J, K)] + W[F(I, J, K + 1)]) -
                     (W[F(I, J, K)] + W[F(I, J, K - 1)]) * (W[F(I, J, K)] + W[F(I, J, K - 1)])) /
                    DZ12[K];
        W_V[F(I, J, K)] = 0.25 * (-W1 - W2 - W3) * DT;
      }
}

/* SET_CONVECTION_FOR_SCALAR nse_dominik.f:834-884; heat source (1.0 at :879) is `source` */
void or_set_convection_for_scalar(const double* U, const double* V, const double* W,
                                  double DT, int nx, int ny, int nz, const double* DX,
                                  const double* DY, const double* DZ, const double* DX12,
                                  const double* DY12, const double* DZ12, const double* T,
                                  double* U_VT, const double* R, double source) {
  Pad F(nx, ny);
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        long c = F(I, J, K);
        double UT = (-((R[F(I - 1, J, K)] * T[F(I - 1, J, K)] * DX[I] + R[c] * T[c] * DX[I - 1]) *
                       U[F(I - 1, J, K)]) / 2.0 / DX12[I - 1] +
                     ((R[c] * T[c] * DX[I + 1] + R[F(I + 1, J, K)] * T[F(I + 1, J, K)] * DX[I]) *
                      U[c]) / 2.0 / DX12[I]) /
                    DX[I];
        double VT = (-((R[F(I, J - 1, K)] * T[F(I, J - 1, K)] * DY[J] + R[c] * T[c] * DY[J - 1]) *
                       V[F(I, J - 1, K)]) / 2.0 / DY12[J - 1] +
                     ((R[c] * T[c] * DY[J + 1] + R[F(I, J + 1, K)] * T[F(I, J + 1, K)] * DY[J]) *
                      V[c]) / 2.0 / DY12[J]) /
                    DY[J];
        double WT = (-((R[F(I, J, K - 1)] * T[F(I, J, K - 1)] * DZ[K] + R[c] * T[c] * DZ[K - 1]) *
                       W[F(I, J, K - 1)]) / 2.0 / DZ12[K - 1] +
                     ((R[c] * T[c] * DZ[K + 1] + R[F(I, J, K + 1)] * T[F(I, J, K + 1)] * DZ[K]) *
                      W[c]) / 2.0 / DZ12[K]) /
                    DZ[K];
        U_VT[c] = (-UT - VT - WT) * DT / R[c] + source * DT;
      }
}

/* SET_CONDUCTION nse_dominik.f:888-945 */
void or_set_conduction(const double* U, double* U_D, const double* V, double* V_D,
                       const double* W, double* W_D, double RE, double DT, int nx, int ny,
                       int nz, const double* DX, const double* DY, const double* DZ,
                       const double* DX12, const double* DY12, const double* DZ12) {
  Pad F(nx, ny);
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        long c = F(I, J, K);
        double U1 = ((U[F(I + 1, J, K)] - U[c]) / DX[I + 1] - (U[c] - U[F(I - 1, J, K)]) / DX[I]) / DX12[I];
        double U2 = ((U[F(I, J + 1, K)] - U[c]) / DY12[J] - (U[c] - U[F(I, J - 1, K)]) / DY12[J - 1]) / DY[J];
        double U3 = ((U[F(I, J, K + 1)] - U[c]) / DZ12[K] - (U[c] - U[F(I, J, K - 1)]) / DZ12[K - 1]) / DZ[K];
        U_D[c] = DT / RE / 2.0 * (U1 + U2 + U3);
        double V1 = ((V[F(I + 1, J, K)] - V[c]) / DX12[I] - (V[c] - V[F(I - 1, J, K)]) / DX12[I - 1]) / DX[I];
        double V2 = ((V[F(I, J + 1, K)] - V[c]) / DY[J + 1] - (V[c] - V[F(I, J - 1, K)]) / DY[J]) / DY12[J];
        double V3 = ((V[F(I, J, K + 1)] - V[c]) / DZ12[K] - (V[c] - V[F(I, J, K - 1)]) / DZ12[K - 1]) / DZ[K];
        V_D[c] = DT / RE / 2.0 * (V1 + V2 + V3);
        double W1 = ((W[F(I + 1, J, K)] - W[c]) / DX12[I] - (W[c] - W[F(I - 1, J, K)]) / DX12[I - 1]) / DX[I];
        double W2 = ((W[F(I, J + 1, K)] - W[c]) / DY12[J] - (W[c] - W[F(I, J - 1, K)]) / DY12[J - 1]) / DY[J];
        double W3 = ((W[F(I, J, K + 1)] - W[c]) / DZ[K + 1] - (W[c] - W[F(I, J, K - 1)]) / DZ[K]) / DZ12[K];
        W_D[c] = DT / RE / 2.0 * (W1 + W2 + W3);
      }
}

/* SET_DIFFUSION_FOR_SCALAR nse_dominik.f:950-1004 */
void or_set_diffusion_for_scalar(double RE, double DT, int nx, int ny, int nz,
                                 const double* DX, const double* DY, const double* DZ,
                                 const double* DX12, const double* DY12,
                                 const double* DZ12, const double* T, double* U_DT,
                                 double SC, const double* L, const double* R) {
  Pad F(nx, ny);
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        long c = F(I, J, K);
        long xp = F(I + 1, J, K), xm = F(I - 1, J, K);
        long yp = F(I, J + 1, K), ym = F(I, J - 1, K);
        long zp = F(I, J, K + 1), zm = F(I, J, K - 1);
        double UT1 = ((DX[I + 1] + DX[I]) / (DX[I + 1] / L[xp] + DX[I] / L[c]) * (T[xp] - T[c]) / DX12[I] -
                      (DX[I - 1] + DX[I]) / (DX[I - 1] / L[xm] + DX[I] / L[c]) * (T[c] - T[xm]) / DX12[I - 1]) /
                     DX[I];
        double UT2 = ((DY[J + 1] + DY[J]) / (DY[J + 1] / L[yp] + DY[J] / L[c]) * (T[yp] - T[c]) / DY12[J] -
                      (DY[J - 1] + DY[J]) / (DY[J - 1] / L[ym] + DY[J] / L[c]) * (T[c] - T[ym]) / DY12[J - 1]) /
                     DY[J];
        double UT3 = ((DZ[K + 1] + DZ[K]) / (DZ[K + 1] / L[zp] + DZ[K] / L[c]) * (T[zp] - T[c]) / DZ12[K] -
                      (DZ[K - 1] + DZ[K]) / (DZ[K - 1] / L[zm] + DZ[K] / L[c]) * (T[c] - T[zm]) / DZ12[K - 1]) /
                     DZ[K];
        U_DT[c] = (UT1 + UT2 + UT3) / 2.0 / RE / SC / R[c] * DT;
      }
}

/* SET_IMMERSED_BOUNDARY nse_dominik.f:1011-1129 (the unused PHI_INT integral omitted) */
void or_set_immersed_boundary(double ETA, int nx, int ny, int nz, double DT, double* U_L,
                              double* V_L, double* W_L, double* T_L, double* CV,
                              const double* U_TA, const double* V_TA, const double* W_TA,
                              int L) {
  Pad F(nx, ny);
  Cell C(nx, ny, nz);
  if (L == 1) {
    for (int K = 1; K <= nz; ++K)
      for (int J = 1; J <= ny; ++J) {
        for (int I = 1; I <= nx - 1; ++I)
          CV[C(I, J, K, 2)] = (CV[C(I, J, K, 1)] + CV[C(I + 1, J, K, 1)]) * 0.50;
        CV[C(nx, J, K, 2)] = CV[C(nx, J, K, 1)];
      }
    for (int K = 1; K <= nz; ++K)
      for (int I = 1; I <= nx; ++I) {
        for (int J = 1; J <= ny - 1; ++J)
          CV[C(I, J, K, 3)] = (CV[C(I, J, K, 1)] + CV[C(I, J + 1, K, 1)]) * 0.50;
        CV[C(I, ny, K, 3)] = CV[C(I, ny, K, 1)];
      }
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        for (int K = 1; K <= nz - 1; ++K)
          CV[C(I, J, K, 4)] = (CV[C(I, J, K, 1)] + CV[C(I, J, K + 1, 1)]) * 0.50;
        CV[C(I, J, nz, 4)] = CV[C(I, J, nz, 1)];
      }
  }
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) {
        long c = F(I, J, K);
        U_L[c] = ETA * CV[C(I, J, K, 2)] * U_TA[c] * DT;
        V_L[c] = ETA * CV[C(I, J, K, 3)] * V_TA[c] * DT;
        W_L[c] = ETA * CV[C(I, J, K, 4)] * W_TA[c] * DT;
        T_L[c] = 0.0;
      }
}

/* SET_EXPLICIT nse_dominik.f:1132-1286 */
void or_set_explicit(const double* u_v, double* u_pre, const double* u_d, double* u_a,
                     const double* v_v, double* v_pre, const double* v_d, double* v_a,
                     const double* w_v, double* w_pre, const double* w_d, double* w_a,
                     const double* u_l, const double* v_l, const double* w_l, int nx,
                     int ny, int nz, int l) {
  Pad F(nx, ny);
  double a1, a2, b1;
  if (l == 1) { a1 = 1.0; a2 = 0.0; b1 = 1.0; }
  else { a1 = 1.5; a2 = -0.5; b1 = 1.0; }
  const double* vv[3] = {u_v, v_v, w_v};
  double* pre[3] = {u_pre, v_pre, w_pre};
  const double* dd[3] = {u_d, v_d, w_d};
  const double* ll[3] = {u_l, v_l, w_l};
  double* aa[3] = {u_a, v_a, w_a};
  for (int f = 0; f < 3; ++f) {
    double* A = aa[f];
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          long c = F(i, j, k);
          A[c] = a1 * vv[f][c] + a2 * pre[f][c] + b1 * dd[f][c] + b1 * ll[f][c];
        }
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j) {
        A[F(0, j, k)] = A[F(nx, j, k)];
        A[F(nx + 1, j, k)] = A[F(1, j, k)];
      }
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) {
        A[F(i, 0, k)] = -1.0 * A[F(i, 1, k)];
        A[F(i, ny + 1, k)] = -1.0 * A[F(i, ny, k)];
      }
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        A[F(i, j, 0)] = A[F(i, j, nz)];
        A[F(i, j, nz + 1)] = A[F(i, j, 1)];
      }
  }
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        long c = F(i, j, k);
        u_pre[c] = u_v[c];
        v_pre[c] = v_v[c];
        w_pre[c] = w_v[c];
      }
}

/* set_explicit_for_tempreture nse_dominik.f:1291-1341 (incl. the z ghost at :1328) */
void or_set_explicit_for_tempreture(const double* u_vT, const double* u_dT, double* u_T,
                                    double* T_pre, const double* T_l, int nx, int ny,
                                    int nz, int l) {
  Pad F(nx, ny);
  double a1, a2, b1;
  if (l == 1) { a1 = 1.0; a2 = 0.0; b1 = 1.0; }
  else { a1 = 1.5; a2 = -0.5; b1 = 1.0; }
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        long c = F(i, j, k);
        u_T[c] = a1 * u_vT[c] + a2 * T_pre[c] + b1 * u_dT[c] + b1 * T_l[c];
      }
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j) {
      u_T[F(0, j, k)] = u_T[F(nx, j, k)];
      u_T[F(nx + 1, j, k)] = u_T[F(1, j, k)];
    }
  for (int i = 0; i <= nx + 1; ++i)
    for (int j = 0; j <= ny + 1; ++j) {
      u_T[F(i, j, 0)] = u_T[F(i, j, nz)];
      u_T[F(i, j, nz + 1)] = u_T[F(i, j, 0)];
    }
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) T_pre[F(i, j, k)] = u_vT[F(i, j, k)];
}

/* implicit_uy nse_dominik.f:1505-1577 */
void or_implicit_uy(double* SUY, int ny, const double* dy, const double* dy12, double Re,
                    double dt, double ft, double fb, double eta, const double* CUY) {
  touch_dense(ny);
  std::vector<double> lo(ny + 2, 0.0), di(ny + 2, 0.0), up(ny + 2, 0.0), u(ny + 2);
  double beta = dt / Re / 2.0;
  for (int j = 1; j <= ny; ++j) {
    double alpha = dt * eta * CUY[j - 1] + 1.0;
    lo[j] = -beta / alpha / dy12[j - 1] / dy[j];
    di[j] = 1.0 + beta / alpha * (1.0 / dy12[j] + 1.0 / dy12[j - 1]) / dy[j];
    up[j] = -beta / alpha / dy12[j] / dy[j];
  }
  di[0] = 1.0; up[0] = 1.0;
  di[ny + 1] = 1.0; lo[ny + 1] = 1.0;
  for (int j = 1; j <= ny; ++j) u[j] = SUY[j];
  u[0] = ft;
  u[ny + 1] = fb;
  ul_eliminate(ny + 1, lo.data(), di.data(), up.data(), u.data());
  for (int j = 0; j <= ny + 1; ++j) SUY[j] = u[j];
}

/* implicit_vy nse_dominik.f:1583-1648 (system over 0..ny, Dirichlet rows 0 and ny) */
void or_implicit_vy(double* SVY, int ny, const double* dy, const double* dy12, double Re,
                    double dt, double ft, double fb, double eta, const double* CVY) {
  touch_dense(ny - 1);
  std::vector<double> lo(ny + 1, 0.0), di(ny + 1, 0.0), up(ny + 1, 0.0), u(ny + 1);
  double beta = dt / Re / 2.0;
  di[0] = 1.0;
  di[ny] = 1.0;
  for (int j = 1; j <= ny - 1; ++j) {
    double alpha = dt * eta * CVY[j - 1] + 1.0;
    lo[j] = -beta / alpha / dy[j] / dy12[j];
    di[j] = 1.0 + beta / alpha * (1.0 / dy[j + 1] + 1.0 / dy[j]) / dy12[j];
    up[j] = -beta / alpha / dy[j + 1] / dy12[j];
  }
  for (int j = 1; j <= ny - 1; ++j) u[j] = SVY[j];
  u[0] = ft;
  u[ny] = fb;
  ul_eliminate(ny, lo.data(), di.data(), up.data(), u.data());
  for (int j = 0; j <= ny; ++j) SVY[j] = u[j];
}

/* harmonic-mean conductance rows shared by implicit_Ty (nse_dominik.f:1811-1829)
 * and implicit_Tx (:1752-1770); ll/rr indexed 0..n+1 */
static void t_rows(int n, const double* d, const double* d12, double beta,
                   const double* alpha, const double* ll, const double* rr, double* lo,
                   double* di, double* up) {
  for (int i = 1; i <= n; ++i) {
    double Hm = (d[i] + d[i - 1]) / (d[i] / ll[i] + d[i - 1] / ll[i - 1]);
    double Hp = (d[i + 1] + d[i]) / (d[i + 1] / ll[i + 1] + d[i] / ll[i]);
    lo[i] = -beta / alpha[i] * Hm / d12[i - 1] / d[i] / rr[i];
    di[i] = 1.0 + beta / alpha[i] * (Hp / d12[i] / d[i] + Hm / d12[i - 1] / d[i]) / rr[i];
    up[i] = -beta / alpha[i] * Hp / d12[i] / d[i] / rr[i];
  }
}

/* implicit_Ty nse_dominik.f:1784-1870.  lly/rry/CUY are indexed 0..ny+1 as in
 * the reference; lly(0), lly(ny+1) are read although parallel_Ty never sets
 * them (nse_dominik.f:3005-3010): callers pass the thc ghost values there. */
void or_implicit_ty(double* STY, int ny, const double* dy, const double* dy12, double Re,
                    double Sc, double dt, const double* lly, const double* rry, double ft,
                    double fb, const double* CUY, double eta) {
  touch_dense(ny);
  std::vector<double> lo(ny + 2, 0.0), di(ny + 2, 0.0), up(ny + 2, 0.0), T(ny + 2),
      alpha(ny + 2);
  double beta = dt / Re / Sc / 2.0;
  for (int j = 1; j <= ny; ++j) alpha[j] = dt * eta * CUY[j] + 1.0;
  di[0] = 1.0; up[0] = 1.0;
  di[ny + 1] = 1.0; lo[ny + 1] = 1.0;
  t_rows(ny, dy, dy12, beta, alpha.data(), lly, rry, lo.data(), di.data(), up.data());
  for (int i = 1; i <= ny; ++i) T[i] = STY[i];
  T[0] = ft;
  T[ny + 1] = fb;
  ul_eliminate(ny + 1, lo.data(), di.data(), up.data(), T.data());
  for (int i = 1; i <= ny; ++i) STY[i] = T[i];
}

/* TDMA periodic_implicit.f:47-64 (Numerical Recipes tridag over 0..n+1) */
void or_tdma(const double* a, const double* b, const double* c, const double* r, double* u,
             int n) {
  std::vector<double> gam(n + 2);
  double bet = b[0];
  u[0] = r[0] / bet;
  for (int j = 1; j <= n + 1; ++j) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n; j >= 0; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
}

/* cyclic periodic_implicit.f:67-93 (Sherman-Morrison, gamma=1) */
void or_cyclic(const double* a, const double* b, const double* c, double alpha,
               double beta, const double* r, double* x, int n) {
  std::vector<double> bb(n + 2), u(n + 2), z(n + 2);
  double gamma = 1.0;
  bb[0] = b[0] - gamma;
  bb[n + 1] = b[n + 1] - alpha * beta / gamma;
  for (int i = 1; i <= n; ++i) bb[i] = b[i];
  or_tdma(a, bb.data(), c, r, x, n);
  u[0] = gamma;
  u[n + 1] = alpha;
  for (int i = 1; i <= n; ++i) u[i] = 0.0;
  or_tdma(a, bb.data(), c, u.data(), z.data(), n);
  double fact = (x[0] + beta * x[n + 1] / gamma) / (1.0 + z[0] + beta * z[n + 1] / gamma);
  for (int i = 0; i <= n + 1; ++i) x[i] = x[i] - fact * z[i];
}

/* implicit_solver periodic_implicit.f:1-44; SUX indexed 0..nx+1, CUX 1..nx (CUX[i-1]) */
void or_implicit_solver(double* SUX, int nx, const double* dx, const double* dx12,
                        double Re, double dt, double ft, double fb, double eta,
                        const double* CUX) {
  std::vector<double> u(nx + 2), aa(nx + 2, 0.0), bb(nx + 2, 0.0), cc(nx + 2, 0.0);
  double beta = dt / Re / 2.0;
  for (int i = 1; i <= nx; ++i) u[i] = SUX[i];
  u[0] = ft;
  u[nx + 1] = fb;
  for (int i = 1; i <= nx; ++i) {
    double alpha = dt * eta * CUX[i - 1] + 1.0;
    aa[i] = -beta / alpha / dx[i] / dx12[i];
    bb[i] = 1.0 + beta / alpha * (1.0 / dx[i + 1] + 1.0 / dx[i]) / dx12[i];
    cc[i] = -beta / alpha / dx[i + 1] / dx12[i];
  }
  aa[0] = 0.0; bb[0] = 0.0; cc[0] = 1.0;
  aa[nx + 1] = 1.0; bb[nx + 1] = 0.0; cc[nx + 1] = 0.0;
  or_cyclic(aa.data(), bb.data(), cc.data(), -1.0, -1.0, u.data(), SUX, nx);
}

/* implicit_Tx nse_dominik.f:1725-1781; llx/rrx/CUX indexed 0..nx+1 */
void or_implicit_tx(double* STX, int nx, const double* dx, const double* dx12, double Re,
                    double Sc, double dt, const double* llx, const double* rrx, double ft,
                    double fb, double eta, const double* CUX) {
  std::vector<double> T(nx + 2), aa(nx + 2, 0.0), bb(nx + 2, 0.0), cc(nx + 2, 0.0),
      alpha(nx + 2);
  double beta = dt / Re / Sc / 2.0;
  for (int i = 1; i <= nx; ++i) alpha[i] = dt * eta * CUX[i] + 1.0;
  for (int i = 1; i <= nx; ++i) T[i] = STX[i];
  T[0] = ft;
  T[nx + 1] = fb;
  t_rows(nx, dx, dx12, beta, alpha.data(), llx, rrx, aa.data(), bb.data(), cc.data());
  aa[0] = 0.0; bb[0] = 0.0; cc[0] = 1.0;
  aa[nx + 1] = 1.0; bb[nx + 1] = 0.0; cc[nx + 1] = 0.0;
  or_cyclic(aa.data(), bb.data(), cc.data(), -1.0, -1.0, T.data(), STX, nx);
}

/* solve_u_temp nse_dominik.f:1344-1461 with parallel_uy/z/x/vy :2893-2967 */
void or_solve_u_temp(double* u_a, double* v_a, double* w_a, int nx, int ny, int nz,
                     const double* dx, const double* dy, const double* dz,
                     const double* dx12, const double* dy12, const double* dz12, double Re,
                     double dt, double eta, const double* cv, const double* u,
                     const double* v, const double* w) {
  Pad F(nx, ny);
  Cell C(nx, ny, nz);
  double* fa[3] = {u_a, v_a, w_a};
  const double* fo[3] = {u, v, w};
  for (int comp = 0; comp < 3; ++comp) {
    double* A = fa[comp];
    int n = comp + 2;
    int jtop = (comp == 1) ? ny - 1 : ny;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          long c = F(i, j, k);
          A[c] = (fo[comp][c] + A[c]) / (1.0 + eta * cv[C(i, j, k, n)] * dt);
        }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i) {
      std::vector<double> S(ny + 2), Cc(ny + 1);
      for (int k = 1; k <= nz; ++k) {
        if (comp == 1) {
          for (int j = 1; j <= ny - 1; ++j) { S[j] = A[F(i, j, k)]; Cc[j - 1] = cv[C(i, j, k, n)]; }
          or_implicit_vy(S.data(), ny, dy, dy12, Re, dt, 0.0, 0.0, eta, Cc.data());
          for (int j = 0; j <= ny; ++j) A[F(i, j, k)] = S[j];
        } else {
          for (int j = 1; j <= ny; ++j) { S[j] = A[F(i, j, k)]; Cc[j - 1] = cv[C(i, j, k, n)]; }
          or_implicit_uy(S.data(), ny, dy, dy12, Re, dt, 0.0, 0.0, eta, Cc.data());
          for (int j = 0; j <= ny + 1; ++j) A[F(i, j, k)] = S[j];
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i) {
      std::vector<double> S(nz + 2), Cc(nz);
      for (int j = 1; j <= jtop; ++j) {
        for (int k = 1; k <= nz; ++k) { S[k] = A[F(i, j, k)]; Cc[k - 1] = cv[C(i, j, k, n)]; }
        or_implicit_solver(S.data(), nz, dz, dz12, Re, dt, 0.0, 0.0, eta, Cc.data());
        for (int k = 0; k <= nz + 1; ++k) A[F(i, j, k)] = S[k];
      }
    }
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= jtop; ++j) {
      std::vector<double> S(nx + 2), Cc(nx);
      for (int k = 1; k <= nz; ++k) {
        for (int i = 1; i <= nx; ++i) { S[i] = A[F(i, j, k)]; Cc[i - 1] = cv[C(i, j, k, n)]; }
        or_implicit_solver(S.data(), nx, dx, dx12, Re, dt, 0.0, 0.0, eta, Cc.data());
        for (int i = 0; i <= nx + 1; ++i) A[F(i, j, k)] = S[i];
      }
    }
  }
}

/* solve_t nse_dominik.f:1465-1501 with parallel_Tx/Ty/Tz :2969-3045.  The
 * uninitialised ll(0), ll(n+1) of the reference drivers are taken from the
 * thc ghost cells.  ft_y/fb_y are the y-wall ghost rows (0 in the reference,
 * nse_dominik.f:3011-3012). */
void or_solve_t(double* u_T, int nx, int ny, int nz, const double* dx, const double* dy,
                const double* dz, const double* dx12, const double* dy12,
                const double* dz12, double Re, double Sc, double dt, const double* rhoCp,
                const double* thc, const double* cv, double eta, double ft_y,
                double fb_y) {
  Pad F(nx, ny);
  Cell C(nx, ny, nz);
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= nx; ++i) {
    std::vector<double> S(ny + 2), cu(ny + 2), rr(ny + 2), ll(ny + 2);
    for (int k = 1; k <= nz; ++k) {
      for (int j = 1; j <= ny; ++j) {
        rr[j] = rhoCp[F(i, j, k)];
        ll[j] = thc[F(i, j, k)];
        S[j] = u_T[F(i, j, k)];
        cu[j] = cv[C(i, j, k, 1)];
      }
      ll[0] = thc[F(i, 0, k)];
      ll[ny + 1] = thc[F(i, ny + 1, k)];
      or_implicit_ty(S.data(), ny, dy, dy12, Re, Sc, dt, ll.data(), rr.data(), ft_y, fb_y,
                     cu.data(), eta);
      for (int j = 1; j <= ny; ++j) u_T[F(i, j, k)] = S[j];
    }
  }
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= ny; ++j) {
    std::vector<double> S(nx + 2), cu(nx + 2), rr(nx + 2), ll(nx + 2);
    for (int k = 1; k <= nz; ++k) {
      for (int i = 1; i <= nx; ++i) {
        rr[i] = rhoCp[F(i, j, k)];
        ll[i] = thc[F(i, j, k)];
        S[i] = u_T[F(i, j, k)];
        cu[i] = cv[C(i, j, k, 1)];
      }
      ll[0] = thc[F(0, j, k)];
      ll[nx + 1] = thc[F(nx + 1, j, k)];
      or_implicit_tx(S.data(), nx, dx, dx12, Re, Sc, dt, ll.data(), rr.data(), 0.0, 0.0,
                     eta, cu.data());
      for (int i = 1; i <= nx; ++i) u_T[F(i, j, k)] = S[i];
    }
  }
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= nx; ++i) {
    std::vector<double> S(nz + 2), cu(nz + 2), rr(nz + 2), ll(nz + 2);
    for (int j = 1; j <= ny; ++j) {
      for (int k = 1; k <= nz; ++k) {
        rr[k] = rhoCp[F(i, j, k)];
        ll[k] = thc[F(i, j, k)];
        S[k] = u_T[F(i, j, k)];
        cu[k] = cv[C(i, j, k, 1)];
      }
      ll[0] = thc[F(i, j, 0)];
      ll[nz + 1] = thc[F(i, j, nz + 1)];
      or_implicit_tx(S.data(), nz, dz, dz12, Re, Sc, dt, ll.data(), rr.data(), 0.0, 0.0,
                     eta, cu.data());
      for (int k = 1; k <= nz; ++k) u_T[F(i, j, k)] = S[k];
    }
  }
}

/* TRIDIAG tridiag.f:5-19 */
void or_tridiag(double* A, double* B, int NN) {
  double* A1 = A; double* A2 = A + NN; double* A3 = A + 2 * NN;
  for (int I = 0; I < NN - 1; ++I) {
    A3[I] = A3[I] / A2[I];
    B[I] = B[I] / A2[I];
    A2[I + 1] = A2[I + 1] - A1[I + 1] * A3[I];
    B[I + 1] = B[I + 1] - A1[I + 1] * B[I];
  }
  B[NN - 1] = B[NN - 1] / A2[NN - 1];
  for (int I = NN - 2; I >= 0; --I) B[I] = B[I] - A3[I] * B[I + 1];
}

/* TRID2 tridiag.f:21-41 (M right-hand sides, B(M,N)) */
void or_trid2(double* A, double* B, int M, int N) {
  double* A1 = A; double* A2 = A + N; double* A3 = A + 2 * N;
  for (int I = 0; I < N - 1; ++I) {
    A3[I] = A3[I] / A2[I];
    A2[I + 1] = A2[I + 1] - A1[I + 1] * A3[I];
    for (int J = 0; J < M; ++J) {
      B[J + (long)M * I] = B[J + (long)M * I] / A2[I];
      B[J + (long)M * (I + 1)] = B[J + (long)M * (I + 1)] - A1[I + 1] * B[J + (long)M * I];
    }
  }
  for (int J = 0; J < M; ++J) B[J + (long)M * (N - 1)] = B[J + (long)M * (N - 1)] / A2[N - 1];
  for (int I = N - 2; I >= 0; --I)
    for (int J = 0; J < M; ++J)
      B[J + (long)M * I] = B[J + (long)M * I] - A3[I] * B[J + (long)M * (I + 1)];
}

/* CTRIDIAG tridiag.f:43-58: real matrix, complex right-hand side; complex/real
 * and real*complex act component-wise */
void or_ctridiag(double* A, double* B, int NN) {
  double* A1 = A; double* A2 = A + NN; double* A3 = A + 2 * NN;
  for (int I = 0; I < NN - 1; ++I) {
    A3[I] = A3[I] / A2[I];
    B[2 * I] = B[2 * I] / A2[I];
    B[2 * I + 1] = B[2 * I + 1] / A2[I];
    A2[I + 1] = A2[I + 1] - A1[I + 1] * A3[I];
    B[2 * I + 2] = B[2 * I + 2] - A1[I + 1] * B[2 * I];
    B[2 * I + 3] = B[2 * I + 3] - A1[I + 1] * B[2 * I + 1];
  }
  B[2 * NN - 2] = B[2 * NN - 2] / A2[NN - 1];
  B[2 * NN - 1] = B[2 * NN - 1] / A2[NN - 1];
  for (int I = NN - 2; I >= 0; --I) {
    B[2 * I] = B[2 * I] - A3[I] * B[2 * I + 2];
    B[2 * I + 1] = B[2 * I + 1] - A3[I] * B[2 * I + 3];
  }
}

/* P2S p2s_fftw2d.f:5-114: for J=1..NY, r2c of FP(0:NX-1,J,0:NZ-1) (unnormalised,
 * FFTW sign -1), half spectrum kx=0..NX/2, divided by NX*NZ, into
 * FPT(0:NX/2,J,0:NZ-1).  Other FPT entries are left untouched. */
void or_p2s(const double* FP, double* FPT, int NX, int NY, int NZ) {
  Pad F(NX, NY);
  int H = NX / 2 + 1;
  long sj = H, sk = (long)H * (NY + 2);
  FFTPlan PX(NX), PZ(NZ);
  double nrm = (double)(NX * NZ);
#pragma omp parallel for schedule(static)
  for (int J = 1; J <= NY; ++J) {
    std::vector<cplx> in(NX > NZ ? NX : NZ), out(NX > NZ ? NX : NZ);
    std::vector<cplx> half((size_t)H * NZ);
    for (int K = 0; K < NZ; ++K) {
      for (int I = 0; I < NX; ++I) in[I] = cplx(FP[F(I, J, K)], 0.0);
      fft(PX, in.data(), out.data(), false);
      for (int I = 0; I < H; ++I) half[I + (size_t)H * K] = out[I];
    }
    for (int I = 0; I < H; ++I) {
      for (int K = 0; K < NZ; ++K) in[K] = half[I + (size_t)H * K];
      fft(PZ, in.data(), out.data(), false);
      for (int K = 0; K < NZ; ++K) {
        long o = 2 * (I + sj * J + sk * K);
        FPT[o] = out[K].real() / nrm;
        FPT[o + 1] = out[K].imag() / nrm;
      }
    }
  }
}

/* S2P p2s_fftw2d.f:116-223: for J=1..NY, c2r (unnormalised, sign +1) of
 * FPT(0:NX/2,J,0:NZ-1) into FP(0:NX-1,J,0:NZ-1), then FP(NX,J,0:NZ)=FP(0,J,.)
 * and FP(0:NX,J,NZ)=FP(.,J,0) (:211-216).  c2r semantics: the z-inverse is a
 * complex DFT per kx column; the x-inverse uses the Hermitian extension with
 * the imaginary parts of the kx=0 and kx=NX/2 terms dropped. */
void or_s2p(const double* FPT, double* FP, int NX, int NY, int NZ) {
  Pad F(NX, NY);
  int H = NX / 2 + 1;
  long sj = H, sk = (long)H * (NY + 2);
  FFTPlan PX(NX), PZ(NZ);
#pragma omp parallel for schedule(static)
  for (int J = 1; J <= NY; ++J) {
    std::vector<cplx> in(NX > NZ ? NX : NZ), out(NX > NZ ? NX : NZ);
    std::vector<cplx> half((size_t)H * NZ);
    for (int I = 0; I < H; ++I) {
      for (int K = 0; K < NZ; ++K) {
        long o = 2 * (I + sj * J + sk * K);
        in[K] = cplx(FPT[o], FPT[o + 1]);
      }
      fft(PZ, in.data(), out.data(), true);
      for (int K = 0; K < NZ; ++K) half[I + (size_t)H * K] = out[K];
    }
    for (int K = 0; K < NZ; ++K) {
      for (int I = 0; I < H; ++I) in[I] = half[I + (size_t)H * K];
      in[0] = cplx(in[0].real(), 0.0);
      if (NX % 2 == 0) in[NX / 2] = cplx(in[NX / 2].real(), 0.0);
      for (int I = H; I < NX; ++I) in[I] = std::conj(in[NX - I]);
      fft(PX, in.data(), out.data(), true);
      for (int I = 0; I < NX; ++I) FP[F(I, J, K)] = out[I].real();
    }
    for (int K = 0; K <= NZ; ++K) FP[F(NX, J, K)] = FP[F(0, J, K)];
    for (int I = 0; I <= NX; ++I) FP[F(I, J, NZ)] = FP[F(I, J, 0)];
  }
}

/* AC and KXZ of MKP mkp.f:54-84.  AC(1:ny,3) column-major; KXZ(0:nx/2,0:nz). */
void or_mkp_coeffs(int nx, int ny, int nz, const double* dx, const double* dy,
                   const double* dz, const double* dy12, double xl, double zl, double* AC,
                   double* KXZ) {
  const double PI = 3.14159265358979312;
  int H = nx / 2 + 1;
  std::vector<double> KX(H), KZ(nz + 1);
  for (int I = 0; I <= nx / 2; ++I) KX[I] = (double)I / xl * PI * 2.0;
  for (int K = 0; K <= nz; ++K) KZ[K] = (K <= nz / 2) ? (double)K : (double)(K - nz);
  for (int K = 0; K <= nz - 1; ++K) KZ[K] = KZ[K] / zl * PI * 2.0;
  for (int K = 0; K <= nz; ++K)
    for (int I = 0; I <= nx / 2; ++I)
      KXZ[I + (long)H * K] = 2.0 * (1.0 - std::cos(KX[I] * dx[I])) / dx[I] / dx[I] +
                             2.0 * (1.0 - std::cos(KZ[K] * dz[K])) / dz[K] / dz[K];
  for (int J = 1; J <= ny; ++J) {
    AC[(J - 1)] = 1.0 / dy12[J - 1] / dy[J];
    AC[(J - 1) + 2 * ny] = 1.0 / dy12[J] / dy[J];
    AC[(J - 1) + ny] = -AC[(J - 1)] - AC[(J - 1) + 2 * ny];
  }
}

/* SPN mkp.f:223-260 */
void or_spn(int NX, int NY, int NZ, const double* AC, const double* KXZ, double* PHIT) {
  int H = NX / 2 + 1;
  long sj = H, sk = (long)H * (NY + 2);
#pragma omp parallel for schedule(static)
  for (int K = 0; K <= NZ - 1; ++K) {
    std::vector<double> AA(3 * NY), B(2 * NY);
    for (int I = 0; I <= NX / 2; ++I) {
      if ((I + 1) * (K + 1) > 1) {
        for (int J = 1; J <= NY; ++J) {
          AA[J - 1] = AC[J - 1];
          AA[J - 1 + NY] = AC[J - 1 + NY] - KXZ[I + (long)H * K];
          AA[J - 1 + 2 * NY] = AC[J - 1 + 2 * NY];
          long o = 2 * (I + sj * J + sk * K);
          B[2 * (J - 1)] = PHIT[o];
          B[2 * (J - 1) + 1] = PHIT[o + 1];
        }
        AA[NY + 0] = AA[NY + 0] + AA[0];
        AA[0] = 0.0;
        AA[NY + NY - 1] = AA[NY + NY - 1] + AA[2 * NY + NY - 1];
        AA[2 * NY + NY - 1] = 0.0;
        or_ctridiag(AA.data(), B.data(), NY);
        for (int J = 1; J <= NY; ++J) {
          long o = 2 * (I + sj * J + sk * K);
          PHIT[o] = B[2 * (J - 1)];
          PHIT[o + 1] = B[2 * (J - 1) + 1];
        }
      }
    }
  }
}

/* SP0B mkp.f:263-290: mean mode by forward marching, phi(0)=phi(1)=0 */
void or_sp0b(int NX, int NY, int NZ, const double* AC, double* PHIT) {
  (void)NZ;
  int H = NX / 2 + 1;
  long sj = H;
  std::vector<double> Dr(NY + 1), Di(NY + 1);
  for (int J = 1; J <= NY; ++J) { Dr[J] = PHIT[2 * sj * J]; Di[J] = PHIT[2 * sj * J + 1]; }
  PHIT[0] = 0.0; PHIT[1] = 0.0;
  PHIT[2 * sj] = 0.0; PHIT[2 * sj + 1] = 0.0;
  for (int J = 1; J <= NY - 1; ++J) {
    double a1 = AC[J - 1], a2 = AC[J - 1 + NY], a3 = AC[J - 1 + 2 * NY];
    double pmr = PHIT[2 * sj * (J - 1)], pmi = PHIT[2 * sj * (J - 1) + 1];
    double pr = PHIT[2 * sj * J], pi = PHIT[2 * sj * J + 1];
    PHIT[2 * sj * (J + 1)] = (Dr[J] - a1 * pmr - a2 * pr) / a3;
    PHIT[2 * sj * (J + 1) + 1] = (Di[J] - a1 * pmi - a2 * pi) / a3;
  }
  PHIT[2 * sj * (NY + 1)] = PHIT[2 * sj * NY];
  PHIT[2 * sj * (NY + 1) + 1] = PHIT[2 * sj * NY + 1];
}

/* PHIBC mkp.f:293-320 */
void or_phibc(int NX, int NY, int NZ, double* PHI) {
  Pad F(NX, NY);
  for (int K = 1; K <= NZ; ++K)
    for (int I = 0; I <= NX; ++I) {
      PHI[F(I, 0, K)] = PHI[F(I, 1, K)];
      PHI[F(I, NY + 1, K)] = PHI[F(I, NY, K)];
    }
  for (int J = 1; J <= NY; ++J)
    for (int I = 0; I <= NX; ++I) {
      PHI[F(I, J, NZ + 1)] = PHI[F(I, J, 1)];
      PHI[F(I, J, 0)] = PHI[F(I, J, NZ)];
    }
  for (int K = 0; K <= NZ; ++K)
    for (int J = 1; J <= NY; ++J) {
      PHI[F(NX + 1, J, K)] = PHI[F(1, J, K)];
      PHI[F(0, J, K)] = PHI[F(NX, J, K)];
    }
  for (int J = 1; J <= NY; ++J) {
    PHI[F(0, J, 0)] = PHI[F(NX, J, NZ)];
    PHI[F(0, J, NZ + 1)] = PHI[F(NX, J, 1)];
    PHI[F(NX + 1, J, 0)] = PHI[F(1, J, NZ)];
    PHI[F(NX + 1, J, NZ + 1)] = PHI[F(1, J, 1)];
  }
}

/* MKP mkp.f:9-220.  PHI is the caller's padded work array (the reference's
 * automatic array): cells the reference never writes keep what the caller put
 * there (zero in every use of this oracle). */
void or_mkp(double* p, const double* u_temp, const double* v_temp, const double* w_temp,
            double dt, const double* dx, const double* dy, const double* dz,
            const double* dx12, const double* dy12, const double* dz12, double Re, int nx,
            int ny, int nz, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
            double* v_ep2, double* w_ep2, double* divu, double* u, double* v, double* w,
            double xl, double zl, double* PHI) {
  (void)Re;
  Pad F(nx, ny);
  int H = nx / 2 + 1;
  std::vector<double> AC(3 * ny), KXZ((size_t)H * (nz + 1));
  or_mkp_coeffs(nx, ny, nz, dx, dy, dz, dy12, xl, zl, AC.data(), KXZ.data());
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        PHI[F(i, j, k)] = ((u_temp[F(i, j, k)] - u_temp[F(i - 1, j, k)]) / dx[i] +
                           (v_temp[F(i, j, k)] - v_temp[F(i, j - 1, k)]) / dy[j] +
                           (w_temp[F(i, j, k)] - w_temp[F(i, j, k - 1)]) / dz[k]) /
                          dt;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) PHI[F(i, j, 0)] = PHI[F(i, j, nz)];
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) PHI[F(0, j, k)] = PHI[F(nx, j, k)];
  for (int j = 1; j <= ny; ++j) PHI[F(0, j, 0)] = PHI[F(nx, j, nz)];

  std::vector<double> PHIT(2 * (size_t)H * (ny + 2) * (nz + 2), 0.0);
  or_p2s(PHI, PHIT.data(), nx, ny, nz);
  or_spn(nx, ny, nz, AC.data(), KXZ.data(), PHIT.data());
  or_sp0b(nx, ny, nz, AC.data(), PHIT.data());
  or_s2p(PHIT.data(), PHI, nx, ny, nz);
  or_phibc(nx, ny, nz, PHI);

#pragma omp parallel for schedule(static)
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        long c = F(i, j, k);
        double gx = (PHI[F(i + 1, j, k)] - PHI[c]) / dx12[i];
        double gy = (PHI[F(i, j + 1, k)] - PHI[c]) / dy12[j];
        double gz = (PHI[F(i, j, k + 1)] - PHI[c]) / dz12[k];
        u[c] = u_temp[c] - dt * gx;
        v[c] = v_temp[c] - dt * gy;
        w[c] = w_temp[c] - dt * gz;
      }
#pragma omp parallel for schedule(static)
  for (int K = 1; K <= nz; ++K)
    for (int J = 1; J <= ny; ++J)
      for (int I = 1; I <= nx; ++I) p[F(I, J, K)] = PHI[F(I, J, K)];
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        long c = F(i, j, k);
        u_ep2[c] = -dt * (p[F(i + 1, j, k)] - p[c]) / dx12[i] + u_ta[c];
        v_ep2[c] = -dt * (p[F(i, j + 1, k)] - p[c]) / dy12[j] + v_ta[c];
        w_ep2[c] = -dt * (p[F(i, j, k + 1)] - p[c]) / dz12[k] + w_ta[c];
      }
#pragma omp parallel for schedule(static)
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        long c = F(i, j, k);
        u_ta[c] = dt * ((PHI[F(i + 1, j, k)] - PHI[c]) / dx12[i]);
        v_ta[c] = dt * ((PHI[F(i, j + 1, k)] - PHI[c]) / dy12[j]);
        w_ta[c] = dt * ((PHI[F(i, j, k + 1)] - PHI[c]) / dz12[k]);
      }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        divu[F(i, j, k)] = (u[F(i, j, k)] - u[F(i - 1, j, k)]) / dx[i] +
                           (v[F(i, j, k)] - v[F(i, j - 1, k)]) / dy[j] +
                           (w[F(i, j, k)] - w[F(i, j, k - 1)]) / dz[k];
}

/* set_levelset set_levelset.f:1-199 (iteration print-out and VTK files omitted).
 * nnn=2000, dt=1e-3 in the reference (:4-5); epsilon = 1.0d0-1 = 0 (:6) so
 * S(phi0) = phi0/|phi0| (NaN where phi0 == 0, as in the reference); the mask
 * transition half-width is width*dx(i) (width = 1 in the reference, :160-166). */
void or_set_levelset(int nx, int ny, int nz, const double* dx, const double* dx12,
                     const double* dy12, const double* dz12, const double* phi0,
                     double* phi, double* cellvalue, int nnn, double dtau, double width) {
  Pad F(nx, ny);
  Cell C(nx, ny, nz);
  const double epsilon = 1.0 - 1;
  const double pi = 3.1415926535;
  long ntot = (long)(nx + 2) * (ny + 2) * (nz + 2);
  std::vector<double> tmp(ntot, 0.0);
  for (long c = 0; c < ntot; ++c) phi[c] = phi0[c];
  for (int it = 0; it <= nnn; ++it) {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          long c = F(i, j, k);
          double a = (phi[c] - phi[F(i - 1, j, k)]) / dx12[i - 1];
          double b = (phi[F(i + 1, j, k)] - phi[c]) / dx[i];
          double cc = (phi[c] - phi[F(i, j - 1, k)]) / dy12[j - 1];
          double d = (phi[F(i, j + 1, k)] - phi[c]) / dy12[j];
          double e = (phi[c] - phi[F(i, j, k - 1)]) / dz12[k - 1];
          double f = (phi[F(i, j, k + 1)] - phi[c]) / dz12[k];
          double ap = a >= 0.0 ? a : 0.0, am = a >= 0.0 ? 0.0 : a;
          double bp = b >= 0.0 ? b : 0.0, bm = b >= 0.0 ? 0.0 : b;
          double cp = cc >= 0.0 ? cc : 0.0, cm = cc >= 0.0 ? 0.0 : cc;
          double dp = d >= 0.0 ? d : 0.0, dm = d >= 0.0 ? 0.0 : d;
          double ep = e >= 0.0 ? e : 0.0, em = e >= 0.0 ? 0.0 : e;
          double fp = f >= 0.0 ? f : 0.0, fm = f >= 0.0 ? 0.0 : f;
          double p0 = phi0[c];
          double sss = p0 / std::sqrt(p0 * p0 + epsilon * epsilon);
          double GGG;
          if (p0 > 0.0)
            GGG = std::sqrt(std::fmax(ap * ap, bm * bm) + std::fmax(cp * cp, dm * dm) +
                            std::fmax(ep * ep, fm * fm)) - 1.0;
          else if (p0 < 0.0)
            GGG = std::sqrt(std::fmax(am * am, bp * bp) + std::fmax(cm * cm, dp * dp) +
                            std::fmax(em * em, fp * fp)) - 1.0;
          else
            GGG = 0.0;
          tmp[c] = phi[c] - dtau * sss * GGG;
        }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) phi[F(i, j, k)] = tmp[F(i, j, k)];
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx + 1; ++i) {
        phi[F(i, j, 0)] = phi[F(i, j, 1)];
        phi[F(i, j, nz + 1)] = phi[F(i, j, nz)];
      }
    for (int k = 0; k <= nz + 1; ++k)
      for (int i = 0; i <= nx + 1; ++i) {
        phi[F(i, 0, k)] = phi[F(i, 1, k)];
        phi[F(i, ny + 1, k)] = phi[F(i, ny, k)];
      }
    for (int k = 0; k <= nz + 1; ++k)
      for (int j = 0; j <= ny + 1; ++j) {
        phi[F(0, j, k)] = phi[F(1, j, k)];
        phi[F(nx + 1, j, k)] = phi[F(nx, j, k)];
      }
  }
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double ph = phi[F(i, j, k)];
        double h = width * dx[i];
        double cv;
        if (ph >= h) cv = 1.0;
        else if (ph <= -1.0 * h) cv = 0.0;
        else cv = (std::sin(pi * ph / 2.0 / h) + 1.0) / 2.0;
        cellvalue[C(i, j, k, 1)] = cv;
      }
}

/* one time step: nse_dominik.f:290-446 */
void or_step(or_state* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
  Pad F(nx, ny);
  Cell C(nx, ny, nz);
  long ntot = (long)(nx + 2) * (ny + 2) * (nz + 2);
  or_set_bc(s->u, s->v, s->w, s->p, nx, ny, nz, s->T, s->tbot, s->ttop);
  or_set_convect(s->u, s->u_v, s->v, s->v_v, s->w, s->w_v, s->dt, nx, ny, nz, s->dx, s->dy,
                 s->dz, s->dx12, s->dy12, s->dz12, s->force);
  or_set_convection_for_scalar(s->u, s->v, s->w, s->dt, nx, ny, nz, s->dx, s->dy, s->dz,
                               s->dx12, s->dy12, s->dz12, s->T, s->u_vT, s->rhoCp,
                               s->source);
  or_set_conduction(s->u, s->u_d, s->v, s->v_d, s->w, s->w_d, s->Re, s->dt, nx, ny, nz,
                    s->dx, s->dy, s->dz, s->dx12, s->dy12, s->dz12);
  or_set_diffusion_for_scalar(s->Re, s->dt, nx, ny, nz, s->dx, s->dy, s->dz, s->dx12,
                              s->dy12, s->dz12, s->T, s->u_dT, s->Sc, s->thc, s->rhoCp);
  or_set_immersed_boundary(s->eta, nx, ny, nz, s->dt, s->u_l, s->v_l, s->w_l, s->T_l,
                           s->cellvalue, s->u_ta, s->v_ta, s->w_ta, s->l);
  or_set_explicit(s->u_v, s->u_pre, s->u_d, s->u_a, s->v_v, s->v_pre, s->v_d, s->v_a,
                  s->w_v, s->w_pre, s->w_d, s->w_a, s->u_l, s->v_l, s->w_l, nx, ny, nz,
                  s->l);
  or_set_explicit_for_tempreture(s->u_vT, s->u_dT, s->u_T, s->T_pre, s->T_l, nx, ny, nz,
                                 s->l);
  or_set_bc(s->u_a, s->v_a, s->w_a, s->p, nx, ny, nz, s->T, s->tbot, s->ttop);
  /* nse_dominik.f:387-396; extension: solid temperature tsolid (0 in the reference) */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        long c = F(i, j, k);
        double cv = s->cellvalue[C(i, j, k, 1)];
        if (s->tsolid == 0.0)
          s->u_T[c] = (s->T[c] + s->u_T[c]) / (1.0 + s->eta * cv * s->dt);
        else
          s->u_T[c] = (s->T[c] + s->u_T[c] + s->eta * cv * s->dt * s->tsolid) /
                      (1.0 + s->eta * cv * s->dt);
      }
  or_solve_u_temp(s->u_a, s->v_a, s->w_a, nx, ny, nz, s->dx, s->dy, s->dz, s->dx12,
                  s->dy12, s->dz12, s->Re, s->dt, s->eta, s->cellvalue, s->u, s->v, s->w);
  std::memcpy(s->u_temp, s->u_a, ntot * sizeof(double));
  std::memcpy(s->v_temp, s->v_a, ntot * sizeof(double));
  std::memcpy(s->w_temp, s->w_a, ntot * sizeof(double));
  or_solve_t(s->u_T, nx, ny, nz, s->dx, s->dy, s->dz, s->dx12, s->dy12, s->dz12, s->Re,
             s->Sc, s->dt, s->rhoCp, s->thc, s->cellvalue, s->eta, 2.0 * s->tbot,
             2.0 * s->ttop);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) s->T[F(i, j, k)] = s->u_T[F(i, j, k)];
  or_set_bc(s->u_temp, s->v_temp, s->w_temp, s->p, nx, ny, nz, s->T, s->tbot, s->ttop);
  or_mkp(s->p, s->u_temp, s->v_temp, s->w_temp, s->dt, s->dx, s->dy, s->dz, s->dx12,
         s->dy12, s->dz12, s->Re, nx, ny, nz, s->u_ta, s->v_ta, s->w_ta, s->u_ep2, s->v_ep2,
         s->w_ep2, s->divu, s->u, s->v, s->w, s->xl, s->zl, s->phi_work);
  s->l += 1;
}

}  // extern "C"
