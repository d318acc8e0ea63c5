// k_levelset.cu -- level-set reinitialisation and mask (set_levelset.f:1-199)
// and the FP64 monitor reductions.  Built with --fmad=false: the update
// phi - dt*S*G rounds like the reference.
#include "common.cuh"

namespace nse {

#define LD(p, i) __ldg((p) + (i))

// one sweep of set_levelset.f:32-96 into phi_new (interior cells)
__global__ void k_levelset_iter(Dims d, GridDev g, const double* __restrict__ phi0,
                                const double* __restrict__ phi, double* __restrict__ out,
                                double dtau) {
  int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  int k = 1 + blockIdx.z;
  if (i > d.nx || j > d.ny) return;
  const double epsilon = 1.0 - 1;  // the reference's PARAMETER(epsilon=1.0d0-1)
  long c = d.P(i, j, k);
  double pc = LD(phi, c);
  double a = (pc - LD(phi, c - 1)) / LD(g.dx12, i - 1);
  double b = (LD(phi, c + 1) - pc) / LD(g.dx, i);
  double cc = (pc - LD(phi, c - d.sx)) / LD(g.dy12, j - 1);
  double dd = (LD(phi, c + d.sx) - pc) / LD(g.dy12, j);
  double e = (pc - LD(phi, c - d.sy)) / LD(g.dz12, k - 1);
  double f = (LD(phi, c + d.sy) - pc) / LD(g.dz12, k);
  double ap = a >= 0.0 ? a : 0.0, am = a >= 0.0 ? 0.0 : a;
  double bp = b >= 0.0 ? b : 0.0, bm = b >= 0.0 ? 0.0 : b;
  double cp = cc >= 0.0 ? cc : 0.0, cm = cc >= 0.0 ? 0.0 : cc;
  double dp = dd >= 0.0 ? dd : 0.0, dm = dd >= 0.0 ? 0.0 : dd;
  double ep = e >= 0.0 ? e : 0.0, em = e >= 0.0 ? 0.0 : e;
  double fp = f >= 0.0 ? f : 0.0, fm = f >= 0.0 ? 0.0 : f;
  double p0 = LD(phi0, c);
  double sss = p0 / sqrt(p0 * p0 + epsilon * epsilon);
  double GGG;
  if (p0 > 0.0)
    GGG = sqrt(fmax(ap * ap, bm * bm) + fmax(cp * cp, dm * dm) + fmax(ep * ep, fm * fm)) - 1.0;
  else if (p0 < 0.0)
    GGG = sqrt(fmax(am * am, bp * bp) + fmax(cm * cm, dp * dp) + fmax(em * em, fp * fp)) - 1.0;
  else
    GGG = 0.0;
  out[c] = pc - dtau * sss * GGG;
}

// Neumann ghosts of set_levelset.f:107-124 (z, then y, then x passes): the
// composition gives every ghost the value of the nearest interior cell
__global__ void k_levelset_bc(Dims d, double* phi) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  long nA = 2L * (ny + 2) * (nz + 2);
  long nB = 2L * nx * (nz + 2);
  long nC = 2L * nx * ny;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (t < nA) {
    i = (t & 1) ? nx + 1 : 0;
    long r = t >> 1;
    j = (int)(r % (ny + 2));
    k = (int)(r / (ny + 2));
  } else if (t < nA + nB) {
    long r = t - nA;
    j = (r & 1) ? ny + 1 : 0;
    r >>= 1;
    i = 1 + (int)(r % nx);
    k = (int)(r / nx);
  } else if (t < nA + nB + nC) {
    long r = t - nA - nB;
    k = (r & 1) ? nz + 1 : 0;
    r >>= 1;
    i = 1 + (int)(r % nx);
    j = 1 + (int)(r / nx);
  } else {
    return;
  }
  int ci = i < 1 ? 1 : (i > nx ? nx : i);
  int cj = j < 1 ? 1 : (j > ny ? ny : j);
  int ck = k < 1 ? 1 : (k > nz ? nz : k);
  phi[d.P(i, j, k)] = phi[d.P(ci, cj, ck)];
}

// smoothed-Heaviside mask of set_levelset.f:157-170, transition half-width
// width*dx(i) (width = 1 in the reference)
__global__ void k_levelset_mask(Dims d, GridDev g, const double* __restrict__ phi,
                                double* __restrict__ cv, double width) {
  int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  int k = 1 + blockIdx.z;
  if (i > d.nx || j > d.ny) return;
  const double pi = 3.1415926535;
  double ph = LD(phi, d.P(i, j, k));
  double h = width * LD(g.dx, i);
  double v;
  if (ph >= h) v = 1.0;
  else if (ph <= -1.0 * h) v = 0.0;
  else v = (sin(pi * ph / 2.0 / h) + 1.0) / 2.0;
  cv[d.C(i, j, k)] = v;
}

static void interior_grid(const Dims& d, dim3& grid, dim3& block) {
  block = dim3(64, 4, 1);
  grid = dim3((d.nx + 63) / 64, (d.ny + 3) / 4, d.nz);
}

void launch_levelset_iter(const Dims& d, const GridDev& g, const double* phi0,
                          const double* phi, double* phi_new, double dtau, cudaStream_t s) {
  dim3 grid, block;
  interior_grid(d, grid, block);
  count_launch();
  k_levelset_iter<<<grid, block, 0, s>>>(d, g, phi0, phi, phi_new, dtau);
}
void launch_levelset_bc(const Dims& d, double* phi, cudaStream_t s) {
  long n = 2L * (d.ny + 2) * (d.nz + 2) + 2L * d.nx * (d.nz + 2) + 2L * d.nx * d.ny;
  count_launch();
  k_levelset_bc<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d, phi);
}
void launch_levelset_mask(const Dims& d, const GridDev& g, const double* phi,
                          double* cellvalue1, double width, cudaStream_t s) {
  dim3 grid, block;
  interior_grid(d, grid, block);
  count_launch();
  k_levelset_mask<<<grid, block, 0, s>>>(d, g, phi, cellvalue1, width);
}

// ---------------------------------------------------------------- monitor --
// FP64 reductions over interior cells: [0] max|divu|, [1] sum |u| dx,
// [2] sum |v| dy, [3] sum |w| dz, [4] sum T dx dy dz, [5] non-finite count of
// u, v, w, T.  Two passes (per-block partials, then one block) so the result
// does not depend on scheduling.
template <class DV>
__global__ void k_monitor_partial(Dims d, GridDev g, const double* u, const double* v,
                                  const double* w, const double* T, const DV* divu,
                                  double* part) {
  __shared__ double sh[6][256];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  long n = d.ncell;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    int i = 1 + (int)(t % d.nx);
    long r = t / d.nx;
    int j = 1 + (int)(r % d.ny);
    int k = 1 + (int)(r / d.ny);
    long c = d.P(i, j, k);
    double uu = u[c], vv = v[c], ww = w[c], tt = T[c];
    acc[0] = fmax(acc[0], fabs((double)divu[c]));
    acc[1] += fabs(uu) * g.dx[i];
    acc[2] += fabs(vv) * g.dy[j];
    acc[3] += fabs(ww) * g.dz[k];
    acc[4] += tt * g.dx[i] * g.dy[j] * g.dz[k];
    acc[5] += (isfinite(uu) && isfinite(vv) && isfinite(ww) && isfinite(tt)) ? 0.0 : 1.0;
  }
  for (int q = 0; q < 6; ++q) sh[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + s]);
      for (int q = 1; q < 6; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) part[q * gridDim.x + blockIdx.x] = sh[q][0];
}
__global__ void k_monitor_final(const double* part, int nb, double* out) {
  __shared__ double sh[6][256];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    acc[0] = fmax(acc[0], part[b]);
    for (int q = 1; q < 6; ++q) acc[q] += part[q * nb + b];
  }
  for (int q = 0; q < 6; ++q) sh[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + s]);
      for (int q = 1; q < 6; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) out[q] = sh[q][0];
}
// out6 must hold 6 + 6*592 doubles of device memory (partials follow)
template <class DV>
static void monitor(const Dims& d, const GridDev& g, const double* u, const double* v,
                    const double* w, const double* T, const DV* divu, double* out6,
                    cudaStream_t s) {
  const int nb = 592;  // 4 blocks per SM on a 148-SM part
  double* part = out6 + 6;
  count_launch();
  k_monitor_partial<DV><<<nb, 256, 0, s>>>(d, g, u, v, w, T, divu, part);
  count_launch();
  k_monitor_final<<<1, 256, 0, s>>>(part, nb, out6);
}
void launch_monitor(const Dims& d, const GridDev& g, const double* u, const double* v,
                    const double* w, const double* T, const double* divu, double* out6,
                    cudaStream_t s) {
  monitor<double>(d, g, u, v, w, T, divu, out6, s);
}
// mixed-precision form: divu stored in FP32 (the reductions stay FP64)
void launch_monitor_f32(const Dims& d, const GridDev& g, const double* u, const double* v,
                        const double* w, const double* T, const float* divu, double* out6,
                        cudaStream_t s) {
  monitor<float>(d, g, u, v, w, T, divu, out6, s);
}

}  // namespace nse
