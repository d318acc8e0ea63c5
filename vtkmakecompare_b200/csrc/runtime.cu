// runtime.cu -- host side of libnsegpu.so: error state, device work arena,
// the reference-named legacy entry points (host arrays in, host arrays out)
// and the resident context API (fields kept in HBM across steps).
#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "k_adjoint.cuh"
#include "k_lines.cuh"

namespace nse {

bool fft_size_ok(int n);  // k_fft.cu
void launch_line_table(int n, const double* D, const double* D12, const LineArgs& a, int kind,
                       double* base, cudaStream_t s);
void launch_line_flags(const Dims& d, const double* c1, int dir, int comp, int jtop,
                       unsigned char* flags, cudaStream_t s);
void launch_lines_exact(int dir, int kind, const Dims& d, double* f, const LineArgs& a,
                        const LineTab& tb, const int* slots, const double* ltab,
                        cudaStream_t s);
void launch_lines_fast(int dir, int kind, const Dims& d, double* f, const LineArgs& a,
                       const LineTab& tb, const int* slots, const double* ltab,
                       cudaStream_t s);
void launch_line_tables_masked(int dir, int kind, const Dims& d, const GridDev& g,
                               const double* c1, const LineArgs& a, const int* ids, int count,
                               double* out, cudaStream_t s);
// k_lines_part.cu
bool part_lines_supported(const Dims& d);
int line_wait_error();  // k_lines_part.cu: a TMA tile wait gave up since the last call
int x_rows_per_lane(int nx);  // k_lines_part.cu: rows per lane of the x solver (0: none)
size_t part_table_stride(int dir, int kind, const Dims& d);
void launch_part_tables(int dir, int kind, const Dims& d, const GridDev& g, const double* c1,
                        const LineArgs& a, const int* ids, int count, double* out,
                        cudaStream_t s);
void launch_lines_part(int dir, int kind, const Dims& d, double* f, const LineArgs& a,
                       const double* tab, const int* slots, const int* ids, int nmasked,
                       const double* mtab, cudaStream_t s);
void launch_lines_part_f32(int dir, int kind, const Dims& d, float* f, double* out,
                           const LineArgs& a, const float* tab, const int* slots,
                           const int* ids, int nmasked, const float* mtab,
                           const double* tab64, const double* mtab64, cudaStream_t s);
void launch_round_table(const double* in, float* out, long n, cudaStream_t s);
void launch_round_line_table(int dir, int kind, const Dims& d, const GridDev& g,
                             const double* c1, const LineArgs& a, const int* ids,
                             const double* in, float* out, long ntables, cudaStream_t s);
size_t part_table_stride32(int dir, int kind, const Dims& d);
// mixed-precision form (FP32 intermediates)
void launch_rhs_f32(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                    const double* u, const double* v, const double* w, const double* T,
                    const float* u_ta, const float* v_ta, const float* w_ta, float* u_pre,
                    float* v_pre, float* w_pre, float* T_pre, const double* c1, float* u_a,
                    float* v_a, float* w_a, float* u_T, bool math64, cudaStream_t s,
                    int shape = 0);
void launch_correct_f32(const Dims& d, const GridRcp& rg, const double* PHI, const float* ut,
                        const float* vt, const float* wt, double* p, double* u, double* v,
                        double* w, float* u_ta, float* v_ta, float* w_ta, float* u_ep2,
                        float* v_ep2, float* w_ep2, float* divu, double dt, cudaStream_t s,
                        int shape = 0);
void launch_set_bc_f32(const Dims& d, float* u, float* v, float* w, double* p, double* T,
                       double tbot, double ttop, int which, cudaStream_t s);
void launch_fft_fwd_x_f32(const PoissonPlan& pp, const Dims& d, const GridDev& g,
                          const GridRcp& rg, const float* ut, const float* vt, const float* wt,
                          double dt, const double* phi, double dx, double dz, int mode,
                          cudaStream_t s);

void launch_fft_z_f32(const PoissonPlan& pp, bool inverse, cudaStream_t s);
void launch_spn_f32(const PoissonPlan& pp, cudaStream_t s);
void launch_fft_inv_x_f32(const PoissonPlan& pp, const Dims& d, double* phi, bool accumulate,
                          cudaStream_t s);
void launch_monitor_f32(const Dims& d, const GridDev& g, const double* u, const double* v,
                        const double* w, const double* T, const float* divu, double* out6,
                        cudaStream_t s);

// ------------------------------------------------------------------ errors --
static thread_local int g_status = NSE_OK;
static thread_local char g_msg[512] = "";

void set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  g_status = status;
  fprintf(stderr, "nsegpu: %s\n", g_msg);
}

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(e == cudaErrorMemoryAllocation ? NSE_ERR_NOMEM : NSE_ERR_CUDA, "%s: %s", what,
            cudaGetErrorString(e));
  return false;
}

// device bytes the library holds (every allocation goes through DBuf) and
// the cap set by nse_set_alloc_limit (0: none)
static std::atomic<long long> g_alloc_bytes{0};
static std::atomic<long long> g_alloc_limit{0};

bool DBuf::ensure(size_t n) {
  if (n <= bytes && p) return true;
  release();
  if (n == 0) n = 16;
  const long long lim = g_alloc_limit.load();
  if (lim > 0 && g_alloc_bytes.load() + (long long)n > lim) {
    set_error(NSE_ERR_NOMEM, "device allocation of %zu bytes refused: the library holds %lld "
              "bytes and its limit is %lld (nse_set_alloc_limit)", n, g_alloc_bytes.load(), lim);
    return false;
  }
  if (!NSE_CUDA(cudaMalloc(&p, n))) {
    p = nullptr;
    bytes = 0;
    return false;
  }
  bytes = n;
  g_alloc_bytes.fetch_add((long long)n);
  return true;
}
void DBuf::release() {
  if (p) {
    cudaFree(p);
    g_alloc_bytes.fetch_sub((long long)bytes);
  }
  p = nullptr;
  bytes = 0;
}

bool ensure_device() {
  static int checked = 0;
  static bool ok = false;
  if (checked) {
    if (!ok) set_error(NSE_ERR_CUDA, "no usable CUDA device (sm_100 required)");
    return ok;
  }
  checked = 1;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error(NSE_ERR_CUDA, "no CUDA device available: %s", cudaGetErrorString(e));
    ok = false;
    return false;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) {
    set_error(NSE_ERR_CUDA, "device %d has compute capability %d.x; this library is built "
              "for sm_100a only", dev, major);
    ok = false;
    return false;
  }
  ok = true;
  return true;
}

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
// a graph replay launches the kernels its capture counted
static void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

DBuf& arena(int slot) {
  static DBuf slots[48];
  return slots[slot];
}

cudaStream_t legacy_stream() {
  static cudaStream_t s = nullptr;
  if (!s) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  return s;
}

static bool copy_box(double* dst, const double* src, const Dims& d, int i0, int i1, int j0,
                     int j1, int k0, int k1, cudaMemcpyKind kind, cudaStream_t s) {
  if (i0 == 0 && j0 == 0 && k0 == 0 && i1 == d.nx + 1 && j1 == d.ny + 1 && k1 == d.nz + 1)
    return NSE_CUDA(cudaMemcpyAsync(dst, src, d.ntot * sizeof(double), kind, s));
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  size_t pitch = (size_t)(d.nx + 2) * sizeof(double);
  p.srcPtr = make_cudaPitchedPtr((void*)src, pitch, d.nx + 2, d.ny + 2);
  p.dstPtr = make_cudaPitchedPtr((void*)dst, pitch, d.nx + 2, d.ny + 2);
  p.srcPos = make_cudaPos((size_t)i0 * sizeof(double), j0, k0);
  p.dstPos = p.srcPos;
  p.extent = make_cudaExtent((size_t)(i1 - i0 + 1) * sizeof(double), j1 - j0 + 1, k1 - k0 + 1);
  p.kind = kind;
  return NSE_CUDA(cudaMemcpy3DAsync(&p, s));
}
bool copy_box_d2h(double* host, const double* dev, const Dims& d, int i0, int i1, int j0,
                  int j1, int k0, int k1, cudaStream_t s) {
  return copy_box(host, dev, d, i0, i1, j0, j1, k0, k1, cudaMemcpyDeviceToHost, s);
}
bool copy_box_h2d(double* dev, const double* host, const Dims& d, int i0, int i1, int j0,
                  int j1, int k0, int k1, cudaStream_t s) {
  return copy_box(dev, host, d, i0, i1, j0, j1, k0, k1, cudaMemcpyHostToDevice, s);
}

// -------------------------------------------------------- legacy helpers --
// A legacy call stages its arrays in arena slots; `Stage` hands them out.
struct Stage {
  int next = 0;
  cudaStream_t s = legacy_stream();
  bool ok = true;
  double* alloc(size_t n) {
    if (!ok) return nullptr;
    DBuf& b = arena(next++);
    if (!b.ensure(n * sizeof(double))) { ok = false; return nullptr; }
    return b.as<double>();
  }
  double* up(const double* h, size_t n) {
    double* d = alloc(n);
    if (d && !NSE_CUDA(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, s)))
      ok = false;
    return ok ? d : nullptr;
  }
  bool down(double* h, const double* d, size_t n) {
    if (!ok) return false;
    if (!NSE_CUDA(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, s)))
      ok = false;
    return ok;
  }
  bool finish() {
    if (!ok) return false;
    if (!NSE_CUDA(cudaGetLastError())) return false;
    return NSE_CUDA(cudaStreamSynchronize(s));
  }
};

static bool dims_ok(int nx, int ny, int nz, const char* who) {
  if (nx < 1 || ny < 1 || nz < 1) {
    set_error(NSE_ERR_ARG, "%s: bad dimensions nx=%d ny=%d nz=%d", who, nx, ny, nz);
    return false;
  }
  return true;
}

}  // namespace nse

using namespace nse;

// =========================================================== C-ABI =========
extern "C" {

const char* nse_last_error(void) { return g_msg; }
void nse_set_alloc_limit(long long bytes) { g_alloc_limit.store(bytes > 0 ? bytes : 0); }
long long nse_alloc_bytes(void) { return g_alloc_bytes.load(); }
long long nse_launch_count(void) { return g_launches.load(); }
int nse_last_status(void) { return g_status; }
void nse_clear_error(void) {
  g_status = NSE_OK;
  g_msg[0] = 0;
}

// ------------------------------------------------------------ tridiag.f ----
void tridiag_(double* A, double* B, const int* NN) {
  if (!ensure_device()) return;
  int n = *NN;
  if (n < 1) { set_error(NSE_ERR_ARG, "tridiag: NN=%d", n); return; }
  Stage st;
  double* dA = st.up(A, 3 * (size_t)n);
  double* dB = st.up(B, n);
  if (!st.ok) return;
  launch_tridiag(dA, dB, n, 1, st.s);
  st.down(A, dA, 3 * (size_t)n);
  st.down(B, dB, n);
  st.finish();
}

void ctridiag_(double* A, double* B, const int* NN) {
  if (!ensure_device()) return;
  int n = *NN;
  if (n < 1) { set_error(NSE_ERR_ARG, "ctridiag: NN=%d", n); return; }
  Stage st;
  double* dA = st.up(A, 3 * (size_t)n);
  double* dB = st.up(B, 2 * (size_t)n);
  if (!st.ok) return;
  launch_tridiag(dA, dB, n, 2, st.s);
  st.down(A, dA, 3 * (size_t)n);
  st.down(B, dB, 2 * (size_t)n);
  st.finish();
}

void trid2_(double* A, double* B, const int* M, const int* N) {
  if (!ensure_device()) return;
  int m = *M, n = *N;
  if (m < 1 || n < 1) { set_error(NSE_ERR_ARG, "trid2: M=%d N=%d", m, n); return; }
  Stage st;
  double* dA = st.up(A, 3 * (size_t)n);
  double* dAm = st.up(A, 3 * (size_t)n);
  double* dB = st.up(B, (size_t)m * n);
  if (!st.ok) return;
  launch_trid2(dA, dAm, dB, m, n, st.s);
  st.down(A, dAm, 3 * (size_t)n);
  st.down(B, dB, (size_t)m * n);
  st.finish();
}

// -------------------------------------------------- periodic_implicit.f ----
void tdma_(const double* a, const double* b, const double* c, const double* r, double* u,
           const int* n) {
  if (!ensure_device()) return;
  int m = *n;
  if (m < 0) { set_error(NSE_ERR_ARG, "tdma: n=%d", m); return; }
  size_t L = m + 2;
  Stage st;
  double *da = st.up(a, L), *db = st.up(b, L), *dc = st.up(c, L), *dr = st.up(r, L);
  double *du = st.alloc(L), *dg = st.alloc(L);
  if (!st.ok) return;
  launch_tdma(da, db, dc, dr, du, dg, m, st.s);
  st.down(u, du, L);
  st.finish();
}

void cyclic_(const double* a, const double* b, const double* c, const double* alpha,
             const double* beta, const double* r, double* x, const int* n) {
  if (!ensure_device()) return;
  int m = *n;
  if (m < 0) { set_error(NSE_ERR_ARG, "cyclic: n=%d", m); return; }
  size_t L = m + 2;
  Stage st;
  double *da = st.up(a, L), *db = st.up(b, L), *dc = st.up(c, L), *dr = st.up(r, L);
  double *dx = st.alloc(L), *dbb = st.alloc(L), *dg = st.alloc(L), *dz = st.alloc(L);
  if (!st.ok) return;
  launch_cyclic_general(da, db, dc, *alpha, *beta, dr, dx, dbb, dg, dz, m, st.s);
  st.down(x, dx, L);
  st.finish();
}

// SUX is written on 0..nx+1 (cyclic writes x(0:n+1) although implicit_solver
// declares SUX(0:nx); every caller of the reference passes an (0:n+1) array)
void implicit_solver_(double* SUX, const int* nx, const double* dx, const double* dx12,
                      const double* Re, const double* dt, const double* ft,
                      const double* fb, const double* eta, const double* CUX) {
  if (!ensure_device()) return;
  int n = *nx;
  if (n < 1) { set_error(NSE_ERR_ARG, "implicit_solver: nx=%d", n); return; }
  size_t L = n + 2;
  Stage st;
  double* f = st.up(SUX, L);
  double *ddx = st.up(dx, L), *ddx12 = st.up(dx12, L), *dcu = st.up(CUX, n);
  double *g1 = st.alloc(L), *g2 = st.alloc(L);
  if (!st.ok) return;
  GridDev g{ddx, ddx, ddx, ddx12, ddx12, ddx12};
  launch_single_cyc(f, g1, g2, 0, n, g, *Re, 1.0, *dt, *eta, *ft, *fb, dcu, nullptr, nullptr,
                    st.s);
  st.down(SUX, f, L);
  st.finish();
}

// ----------------------------------------------- single y / T line solvers --
void implicit_uy_(double* SUY, const int* ny, const double* dy, const double* dy12,
                  const double* Re, const double* dt, const double* ft, const double* fb,
                  const double* eta, const double* CUY) {
  if (!ensure_device()) return;
  int n = *ny;
  if (n < 1) { set_error(NSE_ERR_ARG, "implicit_uy: ny=%d", n); return; }
  size_t L = n + 2;
  Stage st;
  double* f = st.up(SUY, L);
  double *ddy = st.up(dy, L), *ddy12 = st.up(dy12, L), *dcu = st.up(CUY, n);
  double* lsc = st.alloc(L);
  if (!st.ok) return;
  GridDev g{ddy, ddy, ddy, ddy12, ddy12, ddy12};
  launch_single_ul(f, lsc, 0, n, g, *Re, 1.0, *dt, *eta, *ft, *fb, dcu, nullptr, nullptr,
                   st.s);
  st.down(SUY, f, L);
  st.finish();
}

// SVY is written on 0..ny (nse_dominik.f:1643-1645)
void implicit_vy_(double* SVY, const int* ny, const double* dy, const double* dy12,
                  const double* Re, const double* dt, const double* ft, const double* fb,
                  const double* eta, const double* CVY) {
  if (!ensure_device()) return;
  int n = *ny;
  if (n < 2) { set_error(NSE_ERR_ARG, "implicit_vy: ny=%d", n); return; }
  size_t L = n + 2;
  Stage st;
  double* f = st.up(SVY, L);
  double *ddy = st.up(dy, L), *ddy12 = st.up(dy12, L), *dcu = st.up(CVY, n);
  double* lsc = st.alloc(L);
  if (!st.ok) return;
  GridDev g{ddy, ddy, ddy, ddy12, ddy12, ddy12};
  launch_single_ul(f, lsc, 1, n, g, *Re, 1.0, *dt, *eta, *ft, *fb, dcu, nullptr, nullptr,
                   st.s);
  st.down(SVY, f, n + 1);
  st.finish();
}

// STY is written on 1..ny (nse_dominik.f:1866-1868); lly/rry/CUY are (0:ny+1)
void implicit_ty_(double* STY, const int* ny, const double* dy, const double* dy12,
                  const double* Re, const double* Sc, const double* dt, const double* lly,
                  const double* rry, const double* ft, const double* fb, const double* CUY,
                  const double* eta) {
  if (!ensure_device()) return;
  int n = *ny;
  if (n < 1) { set_error(NSE_ERR_ARG, "implicit_ty: ny=%d", n); return; }
  size_t L = n + 2;
  Stage st;
  double* f = st.up(STY, L);
  double *ddy = st.up(dy, L), *ddy12 = st.up(dy12, L);
  double *dcu = st.up(CUY, L), *dll = st.up(lly, L), *drr = st.up(rry, L);
  double* lsc = st.alloc(L);
  if (!st.ok) return;
  GridDev g{ddy, ddy, ddy, ddy12, ddy12, ddy12};
  launch_single_ul(f, lsc, 2, n, g, *Re, *Sc, *dt, *eta, *ft, *fb, dcu, dll, drr, st.s);
  st.down(STY + 1, f + 1, n);
  st.finish();
}

// STX is written on 0..nx+1 by cyclic (nse_dominik.f:1779)
void implicit_tx_(double* STX, const int* nx, const double* dx, const double* dx12,
                  const double* Re, const double* Sc, const double* dt, const double* llx,
                  const double* rrx, const double* ft, const double* fb, const double* eta,
                  const double* CUX) {
  if (!ensure_device()) return;
  int n = *nx;
  if (n < 1) { set_error(NSE_ERR_ARG, "implicit_tx: nx=%d", n); return; }
  size_t L = n + 2;
  Stage st;
  double* f = st.up(STX, L);
  double *ddx = st.up(dx, L), *ddx12 = st.up(dx12, L);
  double *dcu = st.up(CUX, L), *dll = st.up(llx, L), *drr = st.up(rrx, L);
  double *g1 = st.alloc(L), *g2 = st.alloc(L);
  if (!st.ok) return;
  GridDev g{ddx, ddx, ddx, ddx12, ddx12, ddx12};
  launch_single_cyc(f, g1, g2, 1, n, g, *Re, *Sc, *dt, *eta, *ft, *fb, dcu, dll, drr, st.s);
  st.down(STX, f, L);
  st.finish();
}

// ------------------------------------- parallel_* line drivers (tier 2) ----
// nse_dominik.f:2893-3045: the reference's OpenMP loops in solve_u_temp and
// solve_t call one of these per line; each gathers the line of a padded
// field and its mask column into locals, calls the single-line solver and
// scatters the result.  Here the gather and scatter are host loops around
// the GPU single-line solvers above (one launch per call); solve_u_temp_,
// solve_t_ and the resident step solve all lines of a field in one launch,
// so these exist for a driver that calls them directly.
static long pad_at(int nx, int ny, int i, int j, int k) {
  return i + (long)(nx + 2) * (j + (long)(ny + 2) * k);
}
static long cell_at(int nx, int ny, int nz, int i, int j, int k, int n) {
  return (i - 1) + (long)nx * ((j - 1) + (long)ny * ((k - 1) + (long)nz * (n - 1)));
}
// a line index pair inside 1..na x 1..nb and a mask column 1..4
static bool line_ok(const char* who, int a, int na, int b, int nb, int n) {
  if (a < 1 || a > na || b < 1 || b > nb || n < 1 || n > 4) {
    set_error(NSE_ERR_ARG, "%s: line (%d, %d) or mask column %d out of range", who, a, b, n);
    return false;
  }
  return true;
}

// parallel_uy(i,k,u_a,cellvalue,nx,ny,nz,dy,dy12,Re,dt,eta,n) :2893;
// writes u_a(i,0:ny+1,k)
void parallel_uy_(const int* i, const int* k, double* u_a, const double* cellvalue,
                  const int* nx, const int* ny, const int* nz, const double* dy,
                  const double* dy12, const double* Re, const double* dt, const double* eta,
                  const int* n) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_uy") || !line_ok("parallel_uy", *i, NX, *k, NZ, *n))
    return;
  std::vector<double> S(NY + 2, 0.0), C(NY, 0.0);
  for (int j = 1; j <= NY; ++j) {
    S[j] = u_a[pad_at(NX, NY, *i, j, *k)];
    C[j - 1] = cellvalue[cell_at(NX, NY, NZ, *i, j, *k, *n)];
  }
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_uy_(S.data(), ny, dy, dy12, Re, dt, &ft, &fb, eta, C.data());
  if (g_status != NSE_OK) return;
  for (int j = 0; j <= NY + 1; ++j) u_a[pad_at(NX, NY, *i, j, *k)] = S[j];
}

// parallel_vy(i,k,v_a,...) :2950; gathers j = 1..ny-1, writes v_a(i,0:ny,k)
void parallel_vy_(const int* i, const int* k, double* v_a, const double* cellvalue,
                  const int* nx, const int* ny, const int* nz, const double* dy,
                  const double* dy12, const double* Re, const double* dt, const double* eta,
                  const int* n) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_vy") || !line_ok("parallel_vy", *i, NX, *k, NZ, *n))
    return;
  std::vector<double> S(NY + 2, 0.0), C(NY, 0.0);
  for (int j = 1; j <= NY - 1; ++j) {
    S[j] = v_a[pad_at(NX, NY, *i, j, *k)];
    C[j - 1] = cellvalue[cell_at(NX, NY, NZ, *i, j, *k, *n)];
  }
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_vy_(S.data(), ny, dy, dy12, Re, dt, &ft, &fb, eta, C.data());
  if (g_status != NSE_OK) return;
  for (int j = 0; j <= NY; ++j) v_a[pad_at(NX, NY, *i, j, *k)] = S[j];
}

// parallel_z(i,j,u_a,cellvalue,nx,ny,nz,dz,dz12,Re,dt,eta,n) :2912;
// writes u_a(i,j,0:nz+1)
void parallel_z_(const int* i, const int* j, double* u_a, const double* cellvalue,
                 const int* nx, const int* ny, const int* nz, const double* dz,
                 const double* dz12, const double* Re, const double* dt, const double* eta,
                 const int* n) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_z") || !line_ok("parallel_z", *i, NX, *j, NY, *n))
    return;
  std::vector<double> S(NZ + 2, 0.0), C(NZ, 0.0);
  for (int k = 1; k <= NZ; ++k) {
    S[k] = u_a[pad_at(NX, NY, *i, *j, k)];
    C[k - 1] = cellvalue[cell_at(NX, NY, NZ, *i, *j, k, *n)];
  }
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_solver_(S.data(), nz, dz, dz12, Re, dt, &ft, &fb, eta, C.data());
  if (g_status != NSE_OK) return;
  for (int k = 0; k <= NZ + 1; ++k) u_a[pad_at(NX, NY, *i, *j, k)] = S[k];
}

// parallel_x(j,k,u_a,cellvalue,nx,ny,nz,dx,dx12,Re,dt,eta,n) :2931;
// writes u_a(0:nx+1,j,k)
void parallel_x_(const int* j, const int* k, double* u_a, const double* cellvalue,
                 const int* nx, const int* ny, const int* nz, const double* dx,
                 const double* dx12, const double* Re, const double* dt, const double* eta,
                 const int* n) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_x") || !line_ok("parallel_x", *j, NY, *k, NZ, *n))
    return;
  std::vector<double> S(NX + 2, 0.0), C(NX, 0.0);
  for (int i = 1; i <= NX; ++i) {
    S[i] = u_a[pad_at(NX, NY, i, *j, *k)];
    C[i - 1] = cellvalue[cell_at(NX, NY, NZ, i, *j, *k, *n)];
  }
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_solver_(S.data(), nx, dx, dx12, Re, dt, &ft, &fb, eta, C.data());
  if (g_status != NSE_OK) return;
  for (int i = 0; i <= NX + 1; ++i) u_a[pad_at(NX, NY, i, *j, *k)] = S[i];
}

// gather of a temperature line along `dir` (0 x, 1 y, 2 z) through cell
// (a, b) of the other two directions: STX/rrx/llx/CUX of parallel_Tx/Ty/Tz.
// The reference leaves the end entries of its rr/ll locals unset while
// implicit_Tx/Ty read them (nse_dominik.f:2979-2984); they are taken here
// from the rhoCp and thc ghost cells of the line.
static int t_line(int dir, int a, int b, int NX, int NY, int NZ, const double* rhoCp,
                  const double* thc, const double* u_T, const double* cellvalue,
                  std::vector<double>& S, std::vector<double>& R, std::vector<double>& Lc,
                  std::vector<double>& C) {
  const int n = dir == 0 ? NX : (dir == 1 ? NY : NZ);
  S.assign(n + 2, 0.0); R.assign(n + 2, 0.0); Lc.assign(n + 2, 0.0); C.assign(n + 2, 0.0);
  for (int q = 0; q <= n + 1; ++q) {
    const int i = dir == 0 ? q : a, j = dir == 1 ? q : (dir == 0 ? a : b),
              k = dir == 2 ? q : b;
    const long c = pad_at(NX, NY, i, j, k);
    R[q] = rhoCp[c];
    Lc[q] = thc[c];
    if (q >= 1 && q <= n) {
      S[q] = u_T[c];
      C[q] = cellvalue[cell_at(NX, NY, NZ, i, j, k, 1)];
    }
  }
  return n;
}

// parallel_Tx(k,j,nx,ny,nz,rhoCp,thc,u_T,cellvalue,dx,dx12,Re,Sc,dt,eta) :2969;
// writes u_T(1:nx,j,k)
void parallel_tx_(const int* k, const int* j, const int* nx, const int* ny, const int* nz,
                  const double* rhoCp, const double* thc, double* u_T,
                  const double* cellvalue, const double* dx, const double* dx12,
                  const double* Re, const double* Sc, const double* dt, const double* eta) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_tx") || !line_ok("parallel_tx", *j, NY, *k, NZ, 1))
    return;
  std::vector<double> S, R, Lc, C;
  t_line(0, *j, *k, NX, NY, NZ, rhoCp, thc, u_T, cellvalue, S, R, Lc, C);
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_tx_(S.data(), nx, dx, dx12, Re, Sc, dt, Lc.data(), R.data(), &ft, &fb, eta,
               C.data());
  if (g_status != NSE_OK) return;
  for (int i = 1; i <= NX; ++i) u_T[pad_at(NX, NY, i, *j, *k)] = S[i];
}

// parallel_Ty(i,k,...,dy,dy12,Re,Sc,dt,eta) :2995; writes u_T(i,1:ny,k)
void parallel_ty_(const int* i, const int* k, const int* nx, const int* ny, const int* nz,
                  const double* rhoCp, const double* thc, double* u_T,
                  const double* cellvalue, const double* dy, const double* dy12,
                  const double* Re, const double* Sc, const double* dt, const double* eta) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_ty") || !line_ok("parallel_ty", *i, NX, *k, NZ, 1))
    return;
  std::vector<double> S, R, Lc, C;
  t_line(1, *i, *k, NX, NY, NZ, rhoCp, thc, u_T, cellvalue, S, R, Lc, C);
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_ty_(S.data(), ny, dy, dy12, Re, Sc, dt, Lc.data(), R.data(), &ft, &fb, C.data(),
               eta);
  if (g_status != NSE_OK) return;
  for (int j = 1; j <= NY; ++j) u_T[pad_at(NX, NY, *i, j, *k)] = S[j];
}

// parallel_Tz(i,j,...,dz,dz12,Re,Sc,dt,eta) :3021 (through implicit_Tx, as
// the reference does at :3039); writes u_T(i,j,1:nz)
void parallel_tz_(const int* i, const int* j, const int* nx, const int* ny, const int* nz,
                  const double* rhoCp, const double* thc, double* u_T,
                  const double* cellvalue, const double* dz, const double* dz12,
                  const double* Re, const double* Sc, const double* dt, const double* eta) {
  const int NX = *nx, NY = *ny, NZ = *nz;
  if (!dims_ok(NX, NY, NZ, "parallel_tz") || !line_ok("parallel_tz", *i, NX, *j, NY, 1))
    return;
  std::vector<double> S, R, Lc, C;
  t_line(2, *i, *j, NX, NY, NZ, rhoCp, thc, u_T, cellvalue, S, R, Lc, C);
  const double ft = 0.0, fb = 0.0;
  nse_clear_error();
  implicit_tx_(S.data(), nz, dz, dz12, Re, Sc, dt, Lc.data(), R.data(), &ft, &fb, eta,
               C.data());
  if (g_status != NSE_OK) return;
  for (int k = 1; k <= NZ; ++k) u_T[pad_at(NX, NY, *i, *j, k)] = S[k];
}

// ------------------------------------------------------------- SET_C ------
// grid setup (nse_dominik.f:553-607); O(n) host arithmetic, not a GPU path
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

void set_c_(const int* nx, const int* ny, const int* nz, double* x, double* x12, double* y,
            double* y12, double* z, double* z12, double* dx, double* dx12, double* dy,
            double* dy12, double* dz, double* dz12, const double* xl, const double* yl,
            const double* zl) {
  set_c_dir(*nx, *xl, x, x12, dx, dx12);
  set_c_dir(*ny, *yl, y, y12, dy, dy12);
  set_c_dir(*nz, *zl, z, z12, dz, dz12);
}

// y faces y12(j) = y0 + yl/2 (1 + tanh(g(2j/ny-1))/tanh g) for j = 0..ny,
// mirrored spacing in the ghost cells; x and z as SET_C
void nse_set_c_stretched(int nx, int ny, int nz, double* x, double* x12, double* y,
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
  double tg = tanh(gamma);
  for (int j = 0; j <= ny; ++j)
    y12[j] = y0 + 0.5 * yl * (1.0 + tanh(gamma * (2.0 * j / ny - 1.0)) / tg);
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

}  // extern "C"

// grid arrays staged for one legacy call
static bool stage_grid(Stage& st, int nx, int ny, int nz, const double* dx, const double* dy,
                       const double* dz, const double* dx12, const double* dy12,
                       const double* dz12, GridDev& g) {
  g.dx = st.up(dx, nx + 2);
  g.dy = st.up(dy, ny + 2);
  g.dz = st.up(dz, nz + 2);
  g.dx12 = dx12 ? st.up(dx12, nx + 2) : g.dx;
  g.dy12 = dy12 ? st.up(dy12, ny + 2) : g.dy;
  g.dz12 = dz12 ? st.up(dz12, nz + 2) : g.dz;
  return st.ok;
}

extern "C" {

// ----------------------------------------------------- tier-2 stencils ----
void set_bc_(double* u, double* v, double* w, double* p, const int* nx, const int* ny,
             const int* nz, double* T) {
  if (!dims_ok(*nx, *ny, *nz, "set_bc") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  double *du = st.up(u, d.ntot), *dv = st.up(v, d.ntot), *dw = st.up(w, d.ntot);
  double *dp = st.up(p, d.ntot), *dT = st.up(T, d.ntot);
  if (!st.ok) return;
  launch_set_bc(d, du, dv, dw, dp, dT, 0.0, 0.0, 31, st.s);
  st.down(u, du, d.ntot); st.down(v, dv, d.ntot); st.down(w, dw, d.ntot);
  st.down(p, dp, d.ntot); st.down(T, dT, d.ntot);
  st.finish();
}

static bool down_interior(Stage& st, double* h, const double* dv, const Dims& d) {
  if (!st.ok) return false;
  if (!copy_box_d2h(h, dv, d, 1, d.nx, 1, d.ny, 1, d.nz, st.s)) st.ok = false;
  return st.ok;
}

void set_convect_(double* u, double* u_v, double* v, double* v_v, double* w, double* w_v,
                  const double* dt, const int* nx, const int* ny, const int* nz,
                  const double* dx, const double* dy, const double* dz, const double* dx12,
                  const double* dy12, const double* dz12) {
  if (!dims_ok(*nx, *ny, *nz, "set_convect") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  double *du = st.up(u, d.ntot), *dv = st.up(v, d.ntot), *dw = st.up(w, d.ntot);
  double *duv = st.alloc(d.ntot), *dvv = st.alloc(d.ntot), *dwv = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_convect(d, g, du, dv, dw, duv, dvv, dwv, *dt, 1.0, st.s);
  down_interior(st, u_v, duv, d);
  down_interior(st, v_v, dvv, d);
  down_interior(st, w_v, dwv, d);
  st.finish();
}

void set_convection_for_scalar_(double* u, double* v, double* w, const double* dt,
                                const int* nx, const int* ny, const int* nz,
                                const double* dx, const double* dy, const double* dz,
                                const double* dx12, const double* dy12, const double* dz12,
                                double* T, double* u_vT, double* rhoCp) {
  if (!dims_ok(*nx, *ny, *nz, "set_convection_for_scalar") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  double *du = st.up(u, d.ntot), *dv = st.up(v, d.ntot), *dw = st.up(w, d.ntot);
  double *dT = st.up(T, d.ntot), *dr = st.up(rhoCp, d.ntot), *dout = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_convect_scalar(d, g, du, dv, dw, dT, dr, dout, *dt, 1.0, st.s);
  down_interior(st, u_vT, dout, d);
  st.finish();
}

void set_conduction_(double* u, double* u_d, double* v, double* v_d, double* w, double* w_d,
                     const double* Re, const double* dt, const int* nx, const int* ny,
                     const int* nz, const double* dx, const double* dy, const double* dz,
                     const double* dx12, const double* dy12, const double* dz12) {
  if (!dims_ok(*nx, *ny, *nz, "set_conduction") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  double *du = st.up(u, d.ntot), *dv = st.up(v, d.ntot), *dw = st.up(w, d.ntot);
  double *a = st.alloc(d.ntot), *b = st.alloc(d.ntot), *c = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_conduction(d, g, du, dv, dw, a, b, c, *Re, *dt, st.s);
  down_interior(st, u_d, a, d);
  down_interior(st, v_d, b, d);
  down_interior(st, w_d, c, d);
  st.finish();
}

void set_diffusion_for_scalar_(const double* Re, const double* dt, const int* nx,
                               const int* ny, const int* nz, const double* dx,
                               const double* dy, const double* dz, const double* dx12,
                               const double* dy12, const double* dz12, double* T,
                               double* u_dT, const double* Sc, double* thc, double* rhoCp) {
  if (!dims_ok(*nx, *ny, *nz, "set_diffusion_for_scalar") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  double *dT = st.up(T, d.ntot), *dl = st.up(thc, d.ntot), *dr = st.up(rhoCp, d.ntot);
  double* dout = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_diffusion_scalar(d, g, dT, dl, dr, dout, *Re, *Sc, *dt, st.s);
  down_interior(st, u_dT, dout, d);
  st.finish();
}

// ------------------------------------------------------- adjoint.f ----
void set_adj_convect_(double* u, double* u_v, double* v, double* v_v, double* w, double* w_v,
                      const double* Re, const double* dt, const int* nx, const int* ny,
                      const int* nz, const double* dx, const double* dy, const double* dz,
                      const double* dx12, const double* dy12, const double* dz12,
                      double* u_final, double* v_final, double* w_final) {
  (void)Re;
  if (!dims_ok(*nx, *ny, *nz, "set_adj_convect") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  double *du = st.up(u, d.ntot), *dv = st.up(v, d.ntot), *dw = st.up(w, d.ntot);
  double *duf = st.up(u_final, d.ntot), *dvf = st.up(v_final, d.ntot);
  double* dwf = st.up(w_final, d.ntot);
  double *duv = st.alloc(d.ntot), *dvv = st.alloc(d.ntot), *dwv = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_set_adj_convect(d, adj_grid(g), du, dv, dw, duf, dvf, dwf, duv, dvv, dwv, *dt, st.s);
  down_interior(st, u_v, duv, d);
  down_interior(st, v_v, dvv, d);
  down_interior(st, w_v, dwv, d);
  st.finish();
}

void set_adj_convection_for_scalar_(double* u, double* v, double* w, const double* Re,
                                    const double* dt, const int* nx, const int* ny,
                                    const int* nz, const double* dx, const double* dy,
                                    const double* dz, const double* dx12, const double* dy12,
                                    const double* dz12, double* T, double* u_vT,
                                    double* rhoCp, double* u_final, double* v_final,
                                    double* w_final) {
  (void)u; (void)v; (void)w; (void)Re;
  if (!dims_ok(*nx, *ny, *nz, "set_adj_convection_for_scalar") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  double *dT = st.up(T, d.ntot), *dr = st.up(rhoCp, d.ntot);
  double *duf = st.up(u_final, d.ntot), *dvf = st.up(v_final, d.ntot);
  double *dwf = st.up(w_final, d.ntot), *dout = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_set_adj_cscalar(d, adj_grid(g), dT, dr, duf, dvf, dwf, dout, *dt, st.s);
  down_interior(st, u_vT, dout, d);
  st.finish();
}

// adjoint temperature Tf (padded) or zero when Tf is null
static void adj_ns_scalar(const double* dt, int nx, int ny, int nz, const double* dx12,
                          const double* dy12, const double* dz12, const double* T,
                          const double* Tf, double* u_s, double* v_s, double* w_s) {
  if (!dims_ok(nx, ny, nz, "set_adj_ns_scalar") || !ensure_device()) return;
  Dims d = make_dims(nx, ny, nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx12, dy12, dz12, dx12, dy12, dz12, g)) return;
  double* dT = st.up(T, d.ntot);
  double* dTf = Tf ? st.up(Tf, d.ntot) : st.alloc(d.ntot);
  if (dTf && !Tf && !NSE_CUDA(cudaMemsetAsync(dTf, 0, d.ntot * sizeof(double), st.s)))
    st.ok = false;
  double *dus = st.alloc(d.ntot), *dvs = st.alloc(d.ntot), *dws = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_set_adj_ns_scalar(d, adj_grid(g), dT, dTf, dus, dvs, dws, *dt, st.s);
  down_interior(st, u_s, dus, d);
  down_interior(st, v_s, dvs, d);
  down_interior(st, w_s, dws, d);
  st.finish();
}

void set_adj_ns_scalar_(const double* dt, const int* nx, const int* ny, const int* nz,
                        const double* dx12, const double* dy12, const double* dz12, double* T,
                        double* u_s, double* v_s, double* w_s, double* u_final,
                        double* v_final, double* w_final) {
  (void)u_final; (void)v_final; (void)w_final;
  adj_ns_scalar(dt, *nx, *ny, *nz, dx12, dy12, dz12, T, nullptr, u_s, v_s, w_s);
}

int nse_adj_ns_scalar(const double* dt, int nx, int ny, int nz, const double* dx12,
                      const double* dy12, const double* dz12, const double* T,
                      const double* T_final, double* u_s, double* v_s, double* w_s) {
  nse_clear_error();
  if (!dt || !T || !T_final || !u_s || !v_s || !w_s) {
    set_error(NSE_ERR_ARG, "nse_adj_ns_scalar: null argument");
    return NSE_ERR_ARG;
  }
  adj_ns_scalar(dt, nx, ny, nz, dx12, dy12, dz12, T, T_final, u_s, v_s, w_s);
  return nse_last_status();
}

void set_immersed_boundary_(const double* eta, const int* nx, const int* ny, const int* nz,
                            const double* dt, double* u_l, double* v_l, double* w_l,
                            const double* dx, const double* dy, const double* dz,
                            double* T_l, double* cellvalue, double* u_ta, double* v_ta,
                            double* w_ta, const int* l, double* cons_cell) {
  (void)dx; (void)dy; (void)dz;
  if (!dims_ok(*nx, *ny, *nz, "set_immersed_boundary") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  double* dcv = st.up(cellvalue, 4 * (size_t)d.ncell);
  double *a = st.up(u_ta, d.ntot), *b = st.up(v_ta, d.ntot), *c = st.up(w_ta, d.ntot);
  double *ul = st.alloc(d.ntot), *vl = st.alloc(d.ntot), *wl = st.alloc(d.ntot);
  double* tl = st.alloc(d.ntot);
  if (!st.ok) return;
  if (*l == 1) {
    launch_build_face_masks(d, dcv, st.s);
    st.down(cellvalue + d.ncell, dcv + d.ncell, 3 * (size_t)d.ncell);
    *cons_cell = 0.0;
  }
  launch_ib_forcing(d, dcv, a, b, c, ul, vl, wl, tl, *eta, *dt, st.s);
  down_interior(st, u_l, ul, d);
  down_interior(st, v_l, vl, d);
  down_interior(st, w_l, wl, d);
  down_interior(st, T_l, tl, d);
  st.finish();
}

void set_explicit_(double* u_v, double* u_pre, double* u_d, double* u_a, double* v_v,
                   double* v_pre, double* v_d, double* v_a, double* w_v, double* w_pre,
                   double* w_d, double* w_a, double* u_l, double* v_l, double* w_l,
                   const int* nx, const int* ny, const int* nz, const int* l) {
  if (!dims_ok(*nx, *ny, *nz, "set_explicit") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  size_t n = d.ntot;
  double *uv = st.up(u_v, n), *up = st.up(u_pre, n), *ud = st.up(u_d, n), *ua = st.up(u_a, n);
  double *vv = st.up(v_v, n), *vp = st.up(v_pre, n), *vd = st.up(v_d, n), *va = st.up(v_a, n);
  double *wv = st.up(w_v, n), *wp = st.up(w_pre, n), *wd = st.up(w_d, n), *wa = st.up(w_a, n);
  double *ul = st.up(u_l, n), *vl = st.up(v_l, n), *wl = st.up(w_l, n);
  if (!st.ok) return;
  launch_explicit(d, uv, up, ud, ua, vv, vp, vd, va, wv, wp, wd, wa, ul, vl, wl, *l, st.s);
  st.down(u_a, ua, n); st.down(v_a, va, n); st.down(w_a, wa, n);
  down_interior(st, u_pre, up, d);
  down_interior(st, v_pre, vp, d);
  down_interior(st, w_pre, wp, d);
  st.finish();
}

void set_explicit_for_tempreture_(double* u_vT, double* u_dT, double* u_T, double* T_pre,
                                  double* T_l, const int* nx, const int* ny, const int* nz,
                                  const int* l) {
  if (!dims_ok(*nx, *ny, *nz, "set_explicit_for_tempreture") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  size_t n = d.ntot;
  double *vt = st.up(u_vT, n), *dtt = st.up(u_dT, n), *ut = st.up(u_T, n);
  double *tp = st.up(T_pre, n), *tl = st.up(T_l, n);
  if (!st.ok) return;
  launch_explicit_T(d, vt, dtt, ut, tp, tl, *l, st.s);
  st.down(u_T, ut, n);
  down_interior(st, T_pre, tp, d);
  st.finish();
}

void solve_u_temp_(double* u_a, double* v_a, double* w_a, const int* nx, const int* ny,
                   const int* nz, const double* dx, const double* dy, const double* dz,
                   const double* dx12, const double* dy12, const double* dz12,
                   const double* Re, const double* dt, const double* eta,
                   double* cellvalue, double* u, double* v, double* w) {
  if (!dims_ok(*nx, *ny, *nz, "solve_u_temp") || !ensure_device()) return;
  if (*ny < 2) { set_error(NSE_ERR_ARG, "solve_u_temp: ny=%d < 2", *ny); return; }
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  size_t n = d.ntot;
  double *ua = st.up(u_a, n), *va = st.up(v_a, n), *wa = st.up(w_a, n);
  double *du = st.up(u, n), *dv = st.up(v, n), *dw = st.up(w, n);
  double* dcv = st.up(cellvalue, 4 * (size_t)d.ncell);
  LineScratch sc{st.alloc(n), st.alloc(n)};
  if (!st.ok) return;
  double* fa[3] = {ua, va, wa};
  double* fo[3] = {du, dv, dw};
  for (int comp = 0; comp < 3; ++comp) {
    const double* col = dcv + (size_t)(comp + 1) * d.ncell;
    launch_penalize(d, fo[comp], fa[comp], col, *eta, *dt, 0.0, st.s);
    launch_vel_line_col(d, g, fa[comp], col, 1, comp, *Re, *dt, *eta, sc, st.s);
    launch_vel_line_col(d, g, fa[comp], col, 2, comp, *Re, *dt, *eta, sc, st.s);
    launch_vel_line_col(d, g, fa[comp], col, 0, comp, *Re, *dt, *eta, sc, st.s);
  }
  st.down(u_a, ua, n); st.down(v_a, va, n); st.down(w_a, wa, n);
  st.finish();
}

void solve_t_(double* u_T, const int* nx, const int* ny, const int* nz, const double* dx,
              const double* dy, const double* dz, const double* dx12, const double* dy12,
              const double* dz12, const double* Re, const double* Sc, const double* dt,
              double* rhoCp, double* thc, double* cellvalue, const double* eta) {
  if (!dims_ok(*nx, *ny, *nz, "solve_t") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  size_t n = d.ntot;
  double *ut = st.up(u_T, n), *dr = st.up(rhoCp, n), *dl = st.up(thc, n);
  double* dcv = st.up(cellvalue, d.ncell);
  LineScratch sc{st.alloc(n), st.alloc(n)};
  if (!st.ok) return;
  launch_ysolve_T(d, g, ut, dcv, dr, dl, 1.0, 1.0, *Re, *Sc, *dt, *eta, 0.0, 0.0, sc, st.s);
  launch_xsolve_T(d, g, ut, dcv, dr, dl, 1.0, 1.0, *Re, *Sc, *dt, *eta, sc, st.s);
  launch_zsolve_T(d, g, ut, dcv, dr, dl, 1.0, 1.0, *Re, *Sc, *dt, *eta, sc, st.s);
  down_interior(st, u_T, ut, d);
  st.finish();
}

}  // extern "C"

// ------------------------------------------------------ Poisson staging ----
namespace nse {
struct PoissonBufs {
  DBuf spec, scr, AC, KXZ, twx, twz, twxf, twzf, spn_im;
  PoissonPlan pp;
  // SPN pivot table of the fast form (k_spn_babe); none when the plan's rows
  // do not fit the kernel's shared memory
  bool build_tables(cudaStream_t s) {
    if (spn_split(pp) == 0) return true;
    size_t n = (size_t)pp.Hp * pp.ny * pp.nz * sizeof(double);
    if (!spn_im.ensure(n)) return false;
    launch_spn_tables(pp, spn_im.as<double>(), s);
    pp.spn_im = spn_im.as<double>();
    return NSE_CUDA(cudaGetLastError());
  }
  bool build(int nx, int ny, int nz, const double* dx, const double* dy, const double* dz,
             const double* dy12, double xl, double zl, cudaStream_t s) {
    if (!fft_size_ok(nx) || !fft_size_ok(nz)) {
      set_error(NSE_ERR_ARG, "FFT sizes nx=%d nz=%d must be products of 2, 3 and 5", nx, nz);
      return false;
    }
    int H = nx / 2 + 1;
    int Hp = (H + 7) / 8 * 8;
    // AC (3 ny) followed by the reciprocals of AC3 for SP0B's marching
    std::vector<double> AC(4 * (size_t)ny), KXZ((size_t)H * (nz + 1)), twx(2 * (size_t)nx),
        twz(2 * (size_t)nz);
    poisson_plan_tables(nx, ny, nz, dx, dy, dz, dy12, xl, zl, AC.data(), KXZ.data(),
                        twx.data(), twz.data());
    for (int r = 0; r < ny; ++r) AC[3 * (size_t)ny + r] = 1.0 / AC[2 * (size_t)ny + r];
    size_t nspec = (size_t)Hp * ny * nz;
    if (!spec.ensure(2 * nspec * sizeof(double)) || !scr.ensure(nspec * sizeof(double)) ||
        !this->AC.ensure(AC.size() * 8) || !this->KXZ.ensure(KXZ.size() * 8) ||
        !this->twx.ensure(twx.size() * 8) || !this->twz.ensure(twz.size() * 8))
      return false;
    std::vector<float> twxf_h(twx.begin(), twx.end()), twzf_h(twz.begin(), twz.end());
    if (!twxf.ensure(twxf_h.size() * 4) || !twzf.ensure(twzf_h.size() * 4)) return false;
    if (!NSE_CUDA(cudaMemcpyAsync(twxf.p, twxf_h.data(), twxf_h.size() * 4, cudaMemcpyHostToDevice, s)) ||
        !NSE_CUDA(cudaMemcpyAsync(twzf.p, twzf_h.data(), twzf_h.size() * 4, cudaMemcpyHostToDevice, s)) ||
        !NSE_CUDA(cudaMemcpyAsync(this->AC.p, AC.data(), AC.size() * 8, cudaMemcpyHostToDevice, s)) ||
        !NSE_CUDA(cudaMemcpyAsync(this->KXZ.p, KXZ.data(), KXZ.size() * 8, cudaMemcpyHostToDevice, s)) ||
        !NSE_CUDA(cudaMemcpyAsync(this->twx.p, twx.data(), twx.size() * 8, cudaMemcpyHostToDevice, s)) ||
        !NSE_CUDA(cudaMemcpyAsync(this->twz.p, twz.data(), twz.size() * 8, cudaMemcpyHostToDevice, s)))
      return false;
    // the host vectors die here: wait for the copies
    if (!NSE_CUDA(cudaStreamSynchronize(s))) return false;
    pp.nx = nx; pp.ny = ny; pp.nz = nz; pp.H = H; pp.Hp = Hp;
    pp.spec = spec.as<double>(); pp.scr = scr.as<double>();
    pp.AC = this->AC.as<double>(); pp.KXZ = this->KXZ.as<double>();
    pp.rAC3 = pp.AC + 3 * (size_t)ny;
    pp.twx = this->twx.as<double>(); pp.twz = this->twz.as<double>();
    pp.twx_f = twxf.as<float>(); pp.twz_f = twzf.as<float>();
    pp.spn_im = nullptr;
    return true;
  }
  void release() {
    spec.release(); scr.release(); AC.release(); KXZ.release(); twx.release(); twz.release();
    twxf.release(); twzf.release(); spn_im.release();
  }
};
static PoissonBufs& legacy_poisson() {
  static PoissonBufs pb;
  return pb;
}
// reference-layout PHIT for legacy spn_/sp0b_ calls: plane-major with ghosts
// is converted to the internal spectrum and back
}  // namespace nse

// single-thread SP0B on the reference PHIT layout (mkp.f:263-290), including
// the ghost entries PHIT(0,0,0) = 0 and PHIT(0,NY+1,0) = PHIT(0,NY,0)
__global__ void k_sp0b_phit(double2* col, long sj, int ny, const double* AC) {
  if (blockIdx.x || threadIdx.x) return;
  double2 Dn = col[sj * 1];
  col[0] = make_double2(0.0, 0.0);
  col[sj] = make_double2(0.0, 0.0);
  double2 pm = make_double2(0.0, 0.0), pc = pm;
  for (int J = 1; J <= ny - 1; ++J) {
    double2 Dj = Dn;
    Dn = col[sj * (J + 1)];
    double a1 = AC[J - 1], a2 = AC[J - 1 + ny], a3 = AC[J - 1 + 2 * ny];
    double2 pn = make_double2((Dj.x - a1 * pm.x - a2 * pc.x) / a3,
                              (Dj.y - a1 * pm.y - a2 * pc.y) / a3);
    col[sj * (J + 1)] = pn;
    pm = pc;
    pc = pn;
  }
  col[sj * (ny + 1)] = col[sj * ny];
}

extern "C" {

// ------------------------------------------------------------ p2s / s2p ----
void p2s_(double* FP, double* FPT, const int* NX, const int* NY, const int* NZ) {
  if (!dims_ok(*NX, *NY, *NZ, "p2s") || !ensure_device()) return;
  int nx = *NX, ny = *NY, nz = *NZ;
  Dims d = make_dims(nx, ny, nz);
  Stage st;
  std::vector<double> unit(std::max(nx, std::max(ny, nz)) + 2, 1.0);
  PoissonBufs& pb = legacy_poisson();
  if (!pb.build(nx, ny, nz, unit.data(), unit.data(), unit.data(), unit.data(), 1.0, 1.0, st.s))
    return;
  double* dfp = st.up(FP, d.ntot);
  int H = nx / 2 + 1;
  size_t nphit = 2 * (size_t)H * (ny + 2) * (nz + 2);
  double* dphit = st.alloc(nphit);
  if (!st.ok) return;
  GridDev g{};
  launch_fft_fwd_x(pb.pp, d, dfp, nullptr, nullptr, nullptr, g, 1.0, 0, st.s);
  launch_fft_z(pb.pp, false, st.s);
  launch_spec_to_phit(pb.pp, dphit, st.s);
  // written entries: J = 1..NY, K = 0..NZ-1, all kx
  size_t row = (size_t)H * 2 * sizeof(double);
  NSE_CUDA(cudaMemcpy2DAsync(FPT + 2 * (size_t)H, row * (ny + 2), dphit + 2 * (size_t)H,
                             row * (ny + 2), row * ny, nz, cudaMemcpyDeviceToHost, st.s));
  st.finish();
}

void s2p_(double* FPT, double* FP, const int* NX, const int* NY, const int* NZ) {
  if (!dims_ok(*NX, *NY, *NZ, "s2p") || !ensure_device()) return;
  int nx = *NX, ny = *NY, nz = *NZ;
  Dims d = make_dims(nx, ny, nz);
  Stage st;
  std::vector<double> unit(std::max(nx, std::max(ny, nz)) + 2, 1.0);
  PoissonBufs& pb = legacy_poisson();
  if (!pb.build(nx, ny, nz, unit.data(), unit.data(), unit.data(), unit.data(), 1.0, 1.0, st.s))
    return;
  int H = nx / 2 + 1;
  size_t nphit = 2 * (size_t)H * (ny + 2) * (nz + 2);
  double* dphit = st.up(FPT, nphit);
  double* dfp = st.alloc(d.ntot);
  if (!st.ok) return;
  launch_phit_to_spec(pb.pp, dphit, st.s);
  launch_fft_z(pb.pp, true, st.s);
  launch_fft_inv_x(pb.pp, d, dfp, st.s);
  // written entries: FP(0:NX, J, 0:NZ) for J = 1..NY
  copy_box_d2h(FP, dfp, d, 0, nx, 1, ny, 0, nz, st.s);
  st.finish();
}

// --------------------------------------------------- SPN / SP0B / PHIBC ----
void spn_(const int* NX, const int* NY, const int* NZ, const double* AC, const double* KXZ,
          double* PHIT) {
  if (!dims_ok(*NX, *NY, *NZ, "spn") || !ensure_device()) return;
  int nx = *NX, ny = *NY, nz = *NZ;
  Stage st;
  int H = nx / 2 + 1;
  int Hp = (H + 7) / 8 * 8;
  size_t nphit = 2 * (size_t)H * (ny + 2) * (nz + 2);
  double* dphit = st.up(PHIT, nphit);
  double* dAC = st.up(AC, 3 * (size_t)ny);
  double* dK = st.up(KXZ, (size_t)H * (nz + 1));
  double* spec = st.alloc(2 * (size_t)Hp * ny * nz);
  double* scr = st.alloc((size_t)Hp * ny * nz);
  if (!st.ok) return;
  PoissonPlan pp{};
  pp.nx = nx; pp.ny = ny; pp.nz = nz; pp.H = H; pp.Hp = Hp;
  pp.spec = spec; pp.scr = scr; pp.AC = dAC; pp.KXZ = dK;
  launch_phit_to_spec(pp, dphit, st.s);
  launch_spn(pp, true, false, st.s);
  launch_spec_to_phit(pp, dphit, st.s);
  size_t row = (size_t)H * 2 * sizeof(double);
  NSE_CUDA(cudaMemcpy2DAsync(PHIT + 2 * (size_t)H, row * (ny + 2), dphit + 2 * (size_t)H,
                             row * (ny + 2), row * ny, nz, cudaMemcpyDeviceToHost, st.s));
  st.finish();
}

void sp0b_(const int* NX, const int* NY, const int* NZ, const double* AC, double* PHIT) {
  if (!dims_ok(*NX, *NY, *NZ, "sp0b") || !ensure_device()) return;
  int nx = *NX, ny = *NY;
  Stage st;
  int H = nx / 2 + 1;
  // the column PHIT(0, 0:NY+1, 0) (stride H complex)
  double* col = st.alloc(2 * (size_t)H * (ny + 2));
  double* dAC = st.up(AC, 3 * (size_t)ny);
  if (!st.ok) return;
  size_t row = (size_t)H * 2 * sizeof(double);
  NSE_CUDA(cudaMemcpy2DAsync(col, row, PHIT, row, 2 * sizeof(double), ny + 2,
                             cudaMemcpyHostToDevice, st.s));
  count_launch();
  k_sp0b_phit<<<1, 32, 0, st.s>>>(reinterpret_cast<double2*>(col), H, ny, dAC);
  NSE_CUDA(cudaMemcpy2DAsync(PHIT, row, col, row, 2 * sizeof(double), ny + 2,
                             cudaMemcpyDeviceToHost, st.s));
  st.finish();
}

void phibc_(const int* NX, const int* NY, const int* NZ, double* PHI) {
  if (!dims_ok(*NX, *NY, *NZ, "phibc") || !ensure_device()) return;
  Dims d = make_dims(*NX, *NY, *NZ);
  Stage st;
  double* dphi = st.up(PHI, d.ntot);
  if (!st.ok) return;
  launch_phibc(d, dphi, st.s);
  st.down(PHI, dphi, d.ntot);
  st.finish();
}

// ------------------------------------------------------------------ MKP ----
void mkp_(double* p, double* u_temp, double* v_temp, double* w_temp, const double* dt,
          const double* dx, const double* dy, const double* dz, const double* dx12,
          const double* dy12, const double* dz12, const double* Re, const int* nx,
          const int* ny, const int* nz, const void* ompnthreads, double* u_ta, double* v_ta,
          double* w_ta, double* u_ep2, double* v_ep2, double* w_ep2, double* divu,
          double* u, double* v, double* w, const double* xl, const double* zl) {
  (void)Re; (void)ompnthreads;
  if (!dims_ok(*nx, *ny, *nz, "mkp") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  PoissonBufs& pb = legacy_poisson();
  if (!pb.build(d.nx, d.ny, d.nz, dx, dy, dz, dy12, *xl, *zl, st.s)) return;
  GridDev g;
  if (!stage_grid(st, d.nx, d.ny, d.nz, dx, dy, dz, dx12, dy12, dz12, g)) return;
  size_t n = d.ntot;
  double *ut = st.up(u_temp, n), *vt = st.up(v_temp, n), *wt = st.up(w_temp, n);
  double *dp = st.up(p, n), *a = st.up(u_ta, n), *b = st.up(v_ta, n), *c = st.up(w_ta, n);
  double *du = st.alloc(n), *dv = st.alloc(n), *dw = st.alloc(n);
  double *e1 = st.alloc(n), *e2 = st.alloc(n), *e3 = st.alloc(n), *dd = st.alloc(n);
  double* phi = st.alloc(n);
  if (!st.ok) return;
  NSE_CUDA(cudaMemsetAsync(phi, 0, n * sizeof(double), st.s));
  launch_fft_fwd_x(pb.pp, d, nullptr, ut, vt, wt, g, *dt, 1, st.s);
  launch_fft_z(pb.pp, false, st.s);
  launch_spn(pb.pp, true, true, st.s);
  launch_fft_z(pb.pp, true, st.s);
  launch_fft_inv_x(pb.pp, d, phi, st.s);
  launch_phibc(d, phi, st.s);
  launch_correct(d, g, phi, ut, vt, wt, dp, du, dv, dw, a, b, c, e1, e2, e3, dd, *dt, st.s);
  int X = d.nx, Y = d.ny, Z = d.nz;
  copy_box_d2h(u, du, d, 0, X, 0, Y, 0, Z, st.s);
  copy_box_d2h(v, dv, d, 0, X, 0, Y, 0, Z, st.s);
  copy_box_d2h(w, dw, d, 0, X, 0, Y, 0, Z, st.s);
  copy_box_d2h(u_ta, a, d, 0, X, 0, Y, 0, Z, st.s);
  copy_box_d2h(v_ta, b, d, 0, X, 0, Y, 0, Z, st.s);
  copy_box_d2h(w_ta, c, d, 0, X, 0, Y, 0, Z, st.s);
  down_interior(st, p, dp, d);
  down_interior(st, u_ep2, e1, d);
  down_interior(st, v_ep2, e2, d);
  down_interior(st, w_ep2, e3, d);
  down_interior(st, divu, dd, d);
  st.finish();
}

// ---------------------------------------------------------- set_levelset ----
// Fortran Ew.d edit descriptor (w = 15, d = 7): [-]0.ddddddd E+ee, right-justified
static void fortran_e15_7(char* out, double v) {
  char m[32];
  if (v == 0.0 || !isfinite(v)) {
    if (v == 0.0) snprintf(m, sizeof(m), "0.0000000E+00");
    else snprintf(m, sizeof(m), "%s", isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
    snprintf(out, 32, "%15s", m);
    return;
  }
  char t[32];
  snprintf(t, sizeof(t), "%.6E", fabs(v));  // d.ddddddE+xx, 7 significant digits
  int e = atoi(t + 9) + 1;
  char digits[8] = {t[0], t[2], t[3], t[4], t[5], t[6], t[7], 0};
  snprintf(m, sizeof(m), "%s0.%sE%c%02d", v < 0 ? "-" : "", digits, e < 0 ? '-' : '+',
           e < 0 ? -e : e);
  snprintf(out, 32, "%15s", m);
}

// legacy ASCII VTK STRUCTURED_GRID file of set_levelset.f:131-156 / :171-198
static void write_vtk(const char* path, const char* scalars, int nx, int ny, int nz,
                      const double* x, const double* y, const double* z, const double* val,
                      long si, long sj, long sk, long off) {
  FILE* f = fopen(path, "w");
  if (!f) { set_error(NSE_ERR_ARG, "cannot write %s", path); return; }
  fprintf(f, "# vtk DataFile Version 3.8.1\n3D structure of vessel\nASCII \n"
             "DATASET STRUCTURED_GRID\nDIMENSIONS %4d%4d%4d\nPOINTS %9d float\n",
          nx, ny, nz, nx * ny * nz);
  char a[32], b[32], c[32];
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        fortran_e15_7(a, x[i]); fortran_e15_7(b, y[j]); fortran_e15_7(c, z[k]);
        fprintf(f, "%s%s%s\n", a, b, c);
      }
  fprintf(f, "POINT_DATA %9d\n%s\nLOOKUP_TABLE default\n", nx * ny * nz, scalars);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        fortran_e15_7(a, val[off + i * si + j * sj + k * sk]);
        fprintf(f, "%s\n", a);
      }
  fclose(f);
}

static bool run_levelset(const Dims& d, const GridDev& g, const double* dphi0, double* dphi,
                         double* dtmp, double* dcv1, int nnn, double dtau, double width,
                         cudaStream_t s) {
  if (!NSE_CUDA(cudaMemcpyAsync(dphi, dphi0, d.ntot * sizeof(double), cudaMemcpyDeviceToDevice, s)))
    return false;
  double* cur = dphi;
  double* nxt = dtmp;
  for (int it = 0; it <= nnn; ++it) {
    launch_levelset_iter(d, g, dphi0, cur, nxt, dtau, s);
    launch_levelset_bc(d, nxt, s);
    double* t = cur; cur = nxt; nxt = t;
  }
  if (cur != dphi &&
      !NSE_CUDA(cudaMemcpyAsync(dphi, cur, d.ntot * sizeof(double), cudaMemcpyDeviceToDevice, s)))
    return false;
  launch_levelset_mask(d, g, dphi, dcv1, width, s);
  return NSE_CUDA(cudaGetLastError());
}

void set_levelset_(const int* nx, const int* ny, const int* nz, const double* dx,
                   const double* dx12, const double* dy12, const double* dz12,
                   const double* phi0, double* phi, const double* x, const double* y,
                   const double* z, double* cellvalue) {
  if (!dims_ok(*nx, *ny, *nz, "set_levelset") || !ensure_device()) return;
  Dims d = make_dims(*nx, *ny, *nz);
  Stage st;
  GridDev g;
  g.dx = st.up(dx, d.nx + 2);
  g.dx12 = st.up(dx12, d.nx + 2);
  g.dy12 = st.up(dy12, d.ny + 2);
  g.dz12 = st.up(dz12, d.nz + 2);
  g.dy = g.dy12;
  g.dz = g.dz12;
  double* d0 = st.up(phi0, d.ntot);
  double *dphi = st.alloc(d.ntot), *dtmp = st.alloc(d.ntot), *dcv = st.alloc(d.ncell);
  if (!st.ok) return;
  if (!run_levelset(d, g, d0, dphi, dtmp, dcv, 2000, 1.0e-3, 1.0, st.s)) return;
  st.down(phi, dphi, d.ntot);
  st.down(cellvalue, dcv, d.ncell);
  if (!st.finish()) return;
  const char* novtk = getenv("NSEGPU_NO_VTK");
  if (!(novtk && novtk[0] == '1')) {
    write_vtk("levelset.vtk", "SCALARS phi float64", d.nx, d.ny, d.nz, x, y, z, phi, 1, d.sx,
              d.sy, 0);
    write_vtk("cellvalue1.vtk", "SCALARS PHI float", d.nx, d.ny, d.nz, x, y, z, cellvalue, 1,
              d.nx, (long)d.nx * d.ny, -(1 + d.nx + (long)d.nx * d.ny));
  }
}

// list-directed read of structure.dat (set_levelset.f:202-214): four numbers
// per record (x y z phi0), i fastest; Fortran D exponents are accepted
void readgrid3d_(const int* nx, const int* ny, const int* nz, double* phi0) {
  Dims d = make_dims(*nx, *ny, *nz);
  FILE* f = fopen("structure.dat", "r");
  if (!f) { set_error(NSE_ERR_ARG, "readgrid3d: cannot open structure.dat"); return; }
  char tok[128];
  auto next = [&](double& v) -> bool {
    if (fscanf(f, " %127[^ \t\r\n,]", tok) != 1) return false;
    for (char* c = tok; *c; ++c)
      if (*c == 'd' || *c == 'D') *c = 'e';
    v = strtod(tok, nullptr);
    int ch = fgetc(f);
    if (ch != ',' && ch != EOF) ungetc(ch, f);
    return true;
  };
  for (int k = 1; k <= d.nz; ++k)
    for (int j = 1; j <= d.ny; ++j)
      for (int i = 1; i <= d.nx; ++i) {
        double a, b, c, v;
        if (!next(a) || !next(b) || !next(c) || !next(v)) {
          fclose(f);
          set_error(NSE_ERR_ARG, "readgrid3d: structure.dat ended at cell %d %d %d", i, j, k);
          return;
        }
        phi0[d.P(i, j, k)] = v;
      }
  fclose(f);
}

}  // extern "C"

// ============================================================ tier 3 =======
// launch-shape choices of the autotuner, per grid and form, for the process
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tune;
// NSEGPU_TUNE_LOG set: every autotuner candidate's time goes to stderr
static void tune_log(const char* key, int cand, float ms) {
  static const bool on = getenv("NSEGPU_TUNE_LOG") != nullptr;
  if (on) fprintf(stderr, "nsegpu tune [%s] candidate %d: %.4f ms\n", key, cand, ms);
}

struct nse_ctx {
  nse_config cfg;
  Dims d;
  int l;
  cudaStream_t own, stream;
  std::vector<double> hx, hx12, hy, hy12, hz, hz12, hdx, hdx12, hdy, hdy12, hdz, hdz12;
  DBuf grid;
  GridDev g;
  GridRcp rg;
  DBuf f[NSE_NUM_FIELDS];
  DBuf ua, va, wa, uT, sa, sb, tmp, mon;
  PoissonBufs pb;
  // per-phase CUDA events of profiled steps: ev[step][phase boundary]
  std::vector<cudaEvent_t> ev;
  int prof_cap = 0, prof_n = 0;
  // tiled line solver: per-row tables of mask-free lines (7 tables: y UL_U,
  // UL_V, UL_T; z CYC_VEL, CYC_T; x CYC_VEL, CYC_T) and per-line mask flags
  DBuf ltab, lflags;
  LineTab tab[7];
  bool mask_dirty = true;
  // per (direction, component): slot of every line (-1 = mask-free), the
  // line ids of the masked lines and their coefficient tables
  DBuf slots[3][4], ids[3][4], mtab[3][4];
  int nmasked[3][4] = {};
  // partitioned line solver of the fast form (k_lines_part.cu): one table
  // per (direction, component) for the mask-free lines and one per masked line
  bool part = false;
  DBuf ptab[3][4], pmtab[3][4];
  // mixed-precision form: FP32 intermediates (u*, v*, w*, the temperature
  // work field, the AB2 histories, u_ta, u_ep2, divu) and FP32 line tables
  DBuf lsphi;  // level set of the last nse_levelset (the reference's phi)
  bool mixed = false;
  bool math64 = false;   // FP64 arithmetic in the right-hand side (FP32 storage)
  bool lines64 = false;  // FP64 arithmetic in the line sweeps (FP32 storage)
  int refine = 1;
  DBuf ptab_f[3][4], pmtab_f[3][4];
  // when set (adjoint replays), each line-solve pass copies its input to
  // rec[4*comp + pass] and the final line output to rec[4*comp + 3]
  // (comp 0 u, 1 v, 2 w, 3 T; velocity passes y, z, x; temperature y, x, z)
  double* const* rec = nullptr;
  // side streams of the line passes (FP64 fast form): v, w and T run their
  // y/z/x chains beside u's, forked from and joined back into `stream`
  cudaStream_t side[3] = {};
  cudaEvent_t lfork = nullptr, ljoin[3] = {};
  // launch shapes of the partitioned line passes (LineArgs::yzshape per
  // direction and component, x lines per warp iteration per component),
  // chosen by autotune_lines before the first step
  int yzshape[3][4] = {};
  int xnl[4] = {};
  bool tuned = false;
  // launch shape of the fast right-hand-side kernel (autotune_rhs)
  int rhs_shape = 0;
  bool rhs_tuned = false;
  // launch shape of the pipelined correction (autotune_correct)
  int corr_shape = 0;
  bool corr_tuned = false;
  // kx slices of the z transforms and SPN of the FP64 solve (autotune_mid)
  int mid_chunks = 1;
  bool mid_tuned = false;
  // form of the fast two-ended SPN, TMA tiles or cp.async staging
  // (autotune_spn_form; the plan's spn_cp)
  bool spn_tuned = false;
  // one-step CUDA graphs of nse_step (step_replay), one per temperature
  // buffer a step starts from, with the buffer pair the step leaves behind
  cudaGraphExec_t sg[2] = {nullptr, nullptr};
  void* sg_t[2] = {nullptr, nullptr};
  DBuf sg_T[2], sg_uT[2];
  long long sg_nk[2] = {0, 0};    // kernels in each graph
  unsigned long long sg_sig = 0;  // launch shapes the graphs were captured with
  void* hpin = nullptr;           // pinned staging of the masked line lists
  size_t hpin_n = 0;              // its capacity (ints)
  bool sg_off = false;            // a capture failed: step eagerly from now on
};

namespace {
// the launch-shape state a step's launches depend on (autotuners, setters)
unsigned long long shape_sig(const nse_ctx* x) {
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](long long v) { h = (h ^ (unsigned long long)v) * 1099511628211ull; };
  for (int dir = 0; dir < 3; ++dir)
    for (int comp = 0; comp < 4; ++comp) mix(x->yzshape[dir][comp]);
  for (int comp = 0; comp < 4; ++comp) mix(x->xnl[comp]);
  mix(x->rhs_shape);
  mix(x->corr_shape);
  mix(x->mid_chunks);
  mix(x->pb.pp.spn_cp);
  mix((x->tuned ? 1 : 0) | (x->rhs_tuned ? 2 : 0) | (x->corr_tuned ? 4 : 0) |
      (x->mid_tuned ? 8 : 0) | (x->spn_tuned ? 16 : 0));
  // the masked line lists: their lengths set launch grids, and a longer list
  // can move its tables
  for (int dir = 0; dir < 3; ++dir)
    for (int comp = 0; comp < 4; ++comp) {
      mix(x->nmasked[dir][comp]);
      for (const DBuf* b : {&x->slots[dir][comp], &x->ids[dir][comp], &x->mtab[dir][comp],
                            &x->pmtab[dir][comp], &x->pmtab_f[dir][comp]})
        mix((long long)(uintptr_t)b->p);
    }
  return h;
}
void drop_step_graphs(nse_ctx* x) {
  for (int k = 0; k < 2; ++k) {
    if (x->sg[k]) cudaGraphExecDestroy(x->sg[k]);
    x->sg[k] = nullptr;
    x->sg_t[k] = nullptr;
  }
}
}  // namespace

enum { TB_Y_U = 0, TB_Y_V, TB_Y_T, TB_Z_V, TB_Z_T, TB_X_V, TB_X_T };
static int line_kind(int dir, int comp);
static LineArgs line_args(nse_ctx* x, int comp);

static bool build_line_tables(nse_ctx* x) {
  const Dims& d = x->d;
  const nse_config& c = x->cfg;
  int L = std::max(d.nx, std::max(d.ny, d.nz)) + 2;
  size_t per = 10 * (size_t)L;
  if (!x->ltab.ensure(7 * per * sizeof(double))) return false;
  size_t nfl = 4 * ((size_t)d.nx * d.nz + (size_t)d.nx * d.ny + (size_t)d.ny * d.nz);
  if (!x->lflags.ensure(nfl)) return false;
  double* base = x->ltab.as<double>();
  struct T { int n, kind; const double *D, *D12; bool temp; } spec[7] = {
      {d.ny, LK_UL_U, x->g.dy, x->g.dy12, false}, {d.ny, LK_UL_V, x->g.dy, x->g.dy12, false},
      {d.ny, LK_UL_T, x->g.dy, x->g.dy12, true},  {d.nz, LK_CYC_VEL, x->g.dz, x->g.dz12, false},
      {d.nz, LK_CYC_T, x->g.dz, x->g.dz12, true}, {d.nx, LK_CYC_VEL, x->g.dx, x->g.dx12, false},
      {d.nx, LK_CYC_T, x->g.dx, x->g.dx12, true}};
  std::vector<double> dens(7);
  for (int t = 0; t < 7; ++t) {
    LineArgs a{};
    a.beta = spec[t].temp ? c.dt / c.Re / c.Sc / 2.0 : c.dt / c.Re / 2.0;
    a.dt = c.dt; a.eta = c.eta; a.r0 = c.rho_cp; a.l0 = c.thc;
    double* b = base + t * per;
    int Ln = spec[t].n + 2;
    launch_line_table(spec[t].n, spec[t].D, spec[t].D12, a, spec[t].kind, b, x->own);
    LineTab& tb = x->tab[t];
    tb.l = b; tb.dm = b + Ln; tb.rdm = b + 2 * Ln; tb.up = b + 3 * Ln; tb.a = b + 4 * Ln;
    tb.gam = b + 5 * Ln; tb.bet = b + 6 * Ln; tb.rbet = b + 7 * Ln; tb.z = b + 8 * Ln;
    if (!NSE_CUDA(cudaMemcpyAsync(&dens[t], b + 9 * Ln, sizeof(double), cudaMemcpyDeviceToHost,
                                  x->own)))
      return false;
  }
  if (!NSE_CUDA(cudaStreamSynchronize(x->own))) return false;
  for (int t = 0; t < 7; ++t) x->tab[t].den = dens[t];
  x->part = !(c.flags & NSE_FLAG_EXACT) && part_lines_supported(d);
  if (x->mixed && !x->part) {
    set_error(NSE_ERR_ARG,
              "nse_ctx_create: the mixed-precision form needs nx = 32*M (M in 3,4,5,6,8,16), "
              "12 to 512 cells in y and z, and no NSE_FLAG_EXACT");
    return false;
  }
  if (x->part) {
    for (int dir = 0; dir < 3; ++dir)
      for (int comp = 0; comp < 4; ++comp) {
        LineArgs a = line_args(x, comp);
        int kind = line_kind(dir, comp);
        if (!x->ptab[dir][comp].ensure(part_table_stride(dir, kind, d) * sizeof(double)))
          return false;
        launch_part_tables(dir, kind, d, x->g, nullptr, a, nullptr, 1,
                           x->ptab[dir][comp].as<double>(), x->own);
        if (x->mixed) {
          size_t n = part_table_stride32(dir, kind, d);
          if (!x->ptab_f[dir][comp].ensure(n * sizeof(float))) return false;
          launch_round_line_table(dir, kind, d, x->g, nullptr, a, nullptr,
                                  x->ptab[dir][comp].as<double>(),
                                  x->ptab_f[dir][comp].as<float>(), 1, x->own);
        }
      }
    if (!NSE_CUDA(cudaStreamSynchronize(x->own))) return false;
  }
  return true;
}

// flags of lines touching the mask, per direction and component
static unsigned char* flags_of(nse_ctx* x, int dir, int comp) {
  const Dims& d = x->d;
  unsigned char* f = x->lflags.as<unsigned char>();
  size_t yz = (size_t)d.nx * d.nz, zz = (size_t)d.nx * d.ny, xz = (size_t)d.ny * d.nz;
  if (dir == 1) return f + comp * yz;
  if (dir == 2) return f + 4 * yz + comp * zz;
  return f + 4 * yz + 4 * zz + comp * xz;
}

static int line_kind(int dir, int comp) {
  if (dir == 1) return comp == 1 ? LK_UL_V : (comp == 3 ? LK_UL_T : LK_UL_U);
  return comp == 3 ? LK_CYC_T : LK_CYC_VEL;
}

static LineArgs line_args(nse_ctx* x, int comp) {
  const nse_config& c = x->cfg;
  LineArgs a{};
  a.beta = comp == 3 ? c.dt / c.Re / c.Sc / 2.0 : c.dt / c.Re / 2.0;
  a.dt = c.dt; a.eta = c.eta; a.r0 = c.rho_cp; a.l0 = c.thc;
  a.comp = comp;
  a.jtop = comp == 1 ? x->d.ny - 1 : x->d.ny;
  return a;
}

static void line_shape(const nse_ctx* x, int dir, int comp, LineArgs& la) {
  la.yzshape = x->yzshape[dir][comp];
  la.xnl = x->xnl[comp];
}

// after a mask change: flag the lines that touch the mask, give each of them
// a slot and build its coefficient table (the mask is fixed between changes,
// so the sweep is reused by every step)
static bool ensure_side(nse_ctx* x);
static bool refresh_line_flags(nse_ctx* x, cudaStream_t s) {
  if (!x->mask_dirty) return true;
  const Dims& d = x->d;
  const double* c1 = x->f[NSE_CELLVALUE].as<double>();
  // the twelve line passes' flag and table kernels are independent and each
  // is latency-bound (one thread per line), so they run on the context's
  // stream and its three side streams, forked from and joined back into s
  // (one stream with NSE_FLAG_ONE_STREAM)
  cudaStream_t st[4] = {s, s, s, s};
  const bool fan = !(x->cfg.flags & NSE_FLAG_ONE_STREAM) && ensure_side(x);
  if (fan)
    for (int q = 0; q < 3; ++q) st[1 + q] = x->side[q];
  auto fork = [&]() {
    if (!fan) return;
    NSE_CUDA(cudaEventRecord(x->lfork, s));
    for (int q = 0; q < 3; ++q) NSE_CUDA(cudaStreamWaitEvent(x->side[q], x->lfork, 0));
  };
  auto join = [&]() {
    if (!fan) return;
    for (int q = 0; q < 3; ++q) {
      NSE_CUDA(cudaEventRecord(x->ljoin[q], x->side[q]));
      NSE_CUDA(cudaStreamWaitEvent(s, x->ljoin[q], 0));
    }
  };
  fork();
  for (int comp = 0; comp < 4; ++comp) {
    int jtop = (comp == 1) ? d.ny - 1 : d.ny;
    for (int dir = 0; dir < 3; ++dir)
      launch_line_flags(d, c1, dir, comp, jtop, flags_of(x, dir, comp), st[(dir * 4 + comp) & 3]);
  }
  join();
  size_t nfl = 4 * ((size_t)d.nx * d.nz + (size_t)d.nx * d.ny + (size_t)d.ny * d.nz);
  std::vector<unsigned char> hf(nfl);
  if (!NSE_CUDA(cudaMemcpyAsync(hf.data(), x->lflags.p, nfl, cudaMemcpyDeviceToHost, s)) ||
      !NSE_CUDA(cudaStreamSynchronize(s)))
    return false;
  auto lines_of = [&](int dir, int comp) {
    const LineArgs a = line_args(x, comp);
    return dir == 1 ? (long)d.nx * d.nz : (dir == 2 ? (long)d.nx * a.jtop : (long)a.jtop * d.nz);
  };
  // the slot and id lists of every line pass go through one pinned host
  // buffer (kept by the context), so their copies are asynchronous and the
  // refresh waits once, at its end
  size_t cap = 0;
  for (int dir = 0; dir < 3; ++dir)
    for (int comp = 0; comp < 4; ++comp) cap += 2 * (size_t)lines_of(dir, comp);
  if (x->hpin_n < cap) {
    if (x->hpin) cudaFreeHost(x->hpin);
    x->hpin = nullptr;
    x->hpin_n = 0;
    if (!NSE_CUDA(cudaMallocHost(&x->hpin, cap * sizeof(int)))) return false;
    x->hpin_n = cap;
  }
  int* hp = static_cast<int*>(x->hpin);
  fork();
  for (int dir = 0; dir < 3; ++dir)
    for (int comp = 0; comp < 4; ++comp) {
      cudaStream_t s = st[(dir * 4 + comp) & 3];
      LineArgs a = line_args(x, comp);
      const long nlines = lines_of(dir, comp);
      const unsigned char* fl = hf.data() + (flags_of(x, dir, comp) - x->lflags.as<unsigned char>());
      int* slot = hp;
      int* idl = hp + nlines;
      long nid = 0;
      for (long t = 0; t < nlines; ++t) {
        slot[t] = fl[t] ? (int)nid : -1;
        if (fl[t]) idl[nid++] = (int)t;
      }
      hp += nlines + nid;
      const size_t nids = (size_t)nid;
      int kind = line_kind(dir, comp);
      int n = dir == 0 ? d.nx : (dir == 1 ? d.ny : d.nz);
      size_t stride = line_table_stride(kind, n);
      x->nmasked[dir][comp] = (int)nids;
      if (!x->slots[dir][comp].ensure(nlines * sizeof(int)) ||
          !x->ids[dir][comp].ensure(std::max<size_t>(1, nids) * sizeof(int)) ||
          !x->mtab[dir][comp].ensure(std::max<size_t>(1, nids) * stride * sizeof(double)))
        return false;
      if (!NSE_CUDA(cudaMemcpyAsync(x->slots[dir][comp].p, slot, nlines * sizeof(int),
                                    cudaMemcpyHostToDevice, s)))
        return false;
      if (nids > 0 &&
          !NSE_CUDA(cudaMemcpyAsync(x->ids[dir][comp].p, idl, nids * sizeof(int),
                                    cudaMemcpyHostToDevice, s)))
        return false;
      launch_line_tables_masked(dir, kind, d, x->g, c1, a, x->ids[dir][comp].as<int>(),
                                (int)nids, x->mtab[dir][comp].as<double>(), s);
      if (x->part) {
        size_t ps = part_table_stride(dir, kind, d);
        if (!x->pmtab[dir][comp].ensure(std::max<size_t>(1, nids) * ps * sizeof(double)))
          return false;
        launch_part_tables(dir, kind, d, x->g, c1, a, x->ids[dir][comp].as<int>(),
                           (int)nids, x->pmtab[dir][comp].as<double>(), s);
        if (x->mixed) {
          size_t n = std::max<size_t>(1, nids) * part_table_stride32(dir, kind, d);
          if (!x->pmtab_f[dir][comp].ensure(n * sizeof(float))) return false;
          launch_round_line_table(dir, kind, d, x->g, c1, a, x->ids[dir][comp].as<int>(),
                                  x->pmtab[dir][comp].as<double>(),
                                  x->pmtab_f[dir][comp].as<float>(), (long)nids, s);
        }
      }
    }
  join();
  if (!NSE_CUDA(cudaStreamSynchronize(s))) return false;
  x->mask_dirty = false;
  return true;
}

// phases of one step, in launch order
enum {
  PH_BC = 0, PH_RHS, PH_YVEL, PH_ZVEL, PH_XVEL, PH_YT, PH_XT, PH_ZT, PH_BC2, PH_FFTX_F,
  PH_FFTZ_F, PH_SPN, PH_FFTZ_I, PH_FFTX_I, PH_PHIBC, PH_REFINE, PH_CORRECT, PH_COUNT
};

static void mark(nse_ctx* x, int phase) {
  if (x->prof_n >= x->prof_cap) return;
  cudaEventRecord(x->ev[(size_t)x->prof_n * (PH_COUNT + 1) + phase], x->stream);
}

// the side streams and events of the concurrent line passes (made on first use)
static bool ensure_side(nse_ctx* x) {
  if (x->lfork) return true;
  for (int q = 0; q < 3; ++q)
    if (!NSE_CUDA(cudaStreamCreateWithFlags(&x->side[q], cudaStreamNonBlocking)) ||
        !NSE_CUDA(cudaEventCreateWithFlags(&x->ljoin[q], cudaEventDisableTiming)))
      return false;
  return NSE_CUDA(cudaEventCreateWithFlags(&x->lfork, cudaEventDisableTiming));
}

// the concurrent form (line chains on side streams): not with
// NSE_FLAG_ONE_STREAM, and not in profiled steps, whose phases are
// timed one after another on the context's stream
static bool concurrent(nse_ctx* x) {
  return !(x->cfg.flags & NSE_FLAG_ONE_STREAM) && x->prof_n >= x->prof_cap && ensure_side(x);
}


static double* F(nse_ctx* c, int id) { return c->f[id].as<double>(); }
static float* F32(nse_ctx* c, int id) { return c->f[id].as<float>(); }
// fields held in FP32 by the mixed-precision form
static bool f32_field(const nse_ctx* x, int id) {
  if (!x->mixed) return false;
  switch (id) {
    case NSE_U_TA: case NSE_V_TA: case NSE_W_TA: case NSE_U_PRE: case NSE_V_PRE:
    case NSE_W_PRE: case NSE_T_PRE: case NSE_DIVU: case NSE_U_EP2: case NSE_V_EP2:
    case NSE_W_EP2:
      return true;
    default:
      return false;
  }
}

static int status_or(int fallback) { return g_status != NSE_OK ? g_status : fallback; }

extern "C" {

int nse_ctx_create(const nse_config* cfg, nse_ctx** out) {
  nse_clear_error();
  if (!cfg || !out) { set_error(NSE_ERR_ARG, "nse_ctx_create: null argument"); return NSE_ERR_ARG; }
  *out = nullptr;
  const nse_config& c = *cfg;
  if (c.nx < 2 || c.ny < 3 || c.nz < 2) {
    set_error(NSE_ERR_ARG, "nse_ctx_create: need nx>=2, ny>=3, nz>=2 (got %d %d %d)", c.nx, c.ny, c.nz);
    return NSE_ERR_ARG;
  }
  if (!fft_size_ok(c.nx) || !fft_size_ok(c.nz)) {
    set_error(NSE_ERR_ARG, "nse_ctx_create: nx=%d, nz=%d must be products of 2, 3 and 5", c.nx, c.nz);
    return NSE_ERR_ARG;
  }
  if (!(c.dt > 0) || !(c.Re > 0) || !(c.Sc > 0) || !(c.rho_cp > 0) || !(c.thc > 0)) {
    set_error(NSE_ERR_ARG, "nse_ctx_create: dt, Re, Sc, rho_cp, thc must be positive");
    return NSE_ERR_ARG;
  }
  if (c.precision != NSE_FP64 && c.precision != NSE_MIXED) {
    set_error(NSE_ERR_ARG, "nse_ctx_create: precision %d not available", c.precision);
    return NSE_ERR_ARG;
  }
  // arguments are checked first, so a bad call reports NSE_ERR_ARG with or
  // without a usable GPU
  if (!ensure_device()) return NSE_ERR_CUDA;
  nse_ctx* x = new nse_ctx();
  x->cfg = c;
  x->mixed = c.precision == NSE_MIXED;
  x->refine = (c.flags & NSE_FLAG_REFINE2) ? 2 : 1;
  x->math64 = (c.flags & NSE_FLAG_MATH64) != 0;
  x->lines64 = (c.flags & NSE_FLAG_LINES64) != 0;
  x->d = make_dims(c.nx, c.ny, c.nz);
  x->l = 1;
  cudaStreamCreateWithFlags(&x->own, cudaStreamNonBlocking);
  x->stream = x->own;
  int nx = c.nx, ny = c.ny, nz = c.nz;
  auto V = [](int n) { return std::vector<double>(n + 2, 0.0); };
  x->hx = V(nx); x->hx12 = V(nx); x->hdx = V(nx); x->hdx12 = V(nx);
  x->hy = V(ny); x->hy12 = V(ny); x->hdy = V(ny); x->hdy12 = V(ny);
  x->hz = V(nz); x->hz12 = V(nz); x->hdz = V(nz); x->hdz12 = V(nz);
  nse_set_c_stretched(nx, ny, nz, x->hx.data(), x->hx12.data(), x->hy.data(), x->hy12.data(),
                      x->hz.data(), x->hz12.data(), x->hdx.data(), x->hdx12.data(),
                      x->hdy.data(), x->hdy12.data(), x->hdz.data(), x->hdz12.data(), c.xl,
                      c.yl, c.zl, c.y0, c.ystretch);
  size_t gtot = 4 * (size_t)(nx + 2) + 4 * (size_t)(ny + 2) + 4 * (size_t)(nz + 2);
  bool ok = x->grid.ensure(gtot * sizeof(double));
  if (ok) {
    double* gp = x->grid.as<double>();
    std::vector<double> all;
    for (auto* v : {&x->hdx, &x->hdy, &x->hdz, &x->hdx12, &x->hdy12, &x->hdz12})
      all.insert(all.end(), v->begin(), v->end());
    for (auto* v : {&x->hdx, &x->hdy, &x->hdz, &x->hdx12, &x->hdy12, &x->hdz12})
      for (double e : *v) all.push_back(1.0 / e);
    ok = NSE_CUDA(cudaMemcpy(gp, all.data(), gtot * sizeof(double), cudaMemcpyHostToDevice));
    x->g.dx = gp; gp += nx + 2;
    x->g.dy = gp; gp += ny + 2;
    x->g.dz = gp; gp += nz + 2;
    x->g.dx12 = gp; gp += nx + 2;
    x->g.dy12 = gp; gp += ny + 2;
    x->g.dz12 = gp; gp += nz + 2;
    x->rg.rdx = gp; gp += nx + 2;
    x->rg.rdy = gp; gp += ny + 2;
    x->rg.rdz = gp; gp += nz + 2;
    x->rg.rdx12 = gp; gp += nx + 2;
    x->rg.rdy12 = gp; gp += ny + 2;
    x->rg.rdz12 = gp;
  }
  size_t fb = x->d.ntot * sizeof(double);
  for (int id = 0; ok && id < NSE_NUM_FIELDS; ++id) {
    size_t nb = (id == NSE_CELLVALUE) ? x->d.ncell * sizeof(double) : fb;
    ok = x->f[id].ensure(nb) && NSE_CUDA(cudaMemset(x->f[id].p, 0, nb));
  }
  for (DBuf* b : {&x->ua, &x->va, &x->wa, &x->uT, &x->sa, &x->sb, &x->tmp})
    ok = ok && b->ensure(fb) && NSE_CUDA(cudaMemset(b->p, 0, fb));
  ok = ok && x->mon.ensure((6 + 6 * 592) * sizeof(double));
  ok = ok && x->pb.build(nx, ny, nz, x->hdx.data(), x->hdy.data(), x->hdz.data(),
                         x->hdy12.data(), c.xl, c.zl, x->own);
  ok = ok && ((c.flags & NSE_FLAG_EXACT) || x->pb.build_tables(x->own));
  x->pb.pp.spn_cp = (c.flags & NSE_FLAG_SPN_CPASYNC) ? 1 : 0;
  ok = ok && build_line_tables(x);
  if (!ok) {
    nse_ctx_destroy(x);
    return status_or(NSE_ERR_NOMEM);
  }
  *out = x;
  return NSE_OK;
}

int nse_ctx_destroy(nse_ctx* x) {
  if (!x) return NSE_OK;
  if (x->own) cudaStreamSynchronize(x->own);
  if (x->stream) cudaStreamSynchronize(x->stream);
  drop_step_graphs(x);
  if (x->hpin) cudaFreeHost(x->hpin);
  x->hpin = nullptr;
  for (auto& b : x->f) b.release();
  for (DBuf* b : {&x->grid, &x->ua, &x->va, &x->wa, &x->uT, &x->sa, &x->sb, &x->tmp, &x->mon,
                 &x->ltab, &x->lflags, &x->lsphi})
    b->release();
  x->pb.release();
  for (int dir = 0; dir < 3; ++dir)
    for (int comp = 0; comp < 4; ++comp) {
      x->slots[dir][comp].release();
      x->ids[dir][comp].release();
      x->mtab[dir][comp].release();
      x->ptab[dir][comp].release();
      x->pmtab[dir][comp].release();
      x->ptab_f[dir][comp].release();
      x->pmtab_f[dir][comp].release();
    }
  for (cudaEvent_t e : x->ev) cudaEventDestroy(e);
  for (int q = 0; q < 3; ++q) {
    if (x->side[q]) {
      cudaStreamSynchronize(x->side[q]);
      cudaStreamDestroy(x->side[q]);
    }
    if (x->ljoin[q]) cudaEventDestroy(x->ljoin[q]);
  }
  if (x->lfork) cudaEventDestroy(x->lfork);
  if (x->own) cudaStreamDestroy(x->own);
  delete x;
  return NSE_OK;
}

int nse_ctx_set_stream(nse_ctx* x, void* stream) {
  if (!x) return NSE_ERR_ARG;
  x->stream = stream ? (cudaStream_t)stream : x->own;
  return NSE_OK;
}

int nse_ctx_upload(nse_ctx* x, int id, const double* host) {
  if (!x || !host || id < 0 || id >= NSE_NUM_FIELDS) {
    set_error(NSE_ERR_ARG, "nse_ctx_upload: bad argument (field %d)", id);
    return NSE_ERR_ARG;
  }
  size_t n = (id == NSE_CELLVALUE) ? x->d.ncell : x->d.ntot;
  if (id == NSE_CELLVALUE) x->mask_dirty = true;
  if (f32_field(x, id)) {
    std::vector<float> h(host, host + n);
    if (!NSE_CUDA(cudaMemcpyAsync(x->f[id].p, h.data(), n * sizeof(float),
                                  cudaMemcpyHostToDevice, x->stream)))
      return status_or(NSE_ERR_CUDA);
    return NSE_CUDA(cudaStreamSynchronize(x->stream)) ? NSE_OK : status_or(NSE_ERR_CUDA);
  }
  if (!NSE_CUDA(cudaMemcpyAsync(x->f[id].p, host, n * sizeof(double), cudaMemcpyHostToDevice,
                                x->stream)))
    return status_or(NSE_ERR_CUDA);
  return NSE_CUDA(cudaStreamSynchronize(x->stream)) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

int nse_ctx_download(nse_ctx* x, int id, double* host) {
  if (!x || !host || id < 0 || id >= NSE_NUM_FIELDS) {
    set_error(NSE_ERR_ARG, "nse_ctx_download: bad argument (field %d)", id);
    return NSE_ERR_ARG;
  }
  size_t n = (id == NSE_CELLVALUE) ? x->d.ncell : x->d.ntot;
  if (f32_field(x, id)) {
    std::vector<float> h(n);
    if (!NSE_CUDA(cudaMemcpyAsync(h.data(), x->f[id].p, n * sizeof(float),
                                  cudaMemcpyDeviceToHost, x->stream)) ||
        !NSE_CUDA(cudaStreamSynchronize(x->stream)))
      return status_or(NSE_ERR_CUDA);
    for (size_t t = 0; t < n; ++t) host[t] = (double)h[t];
    return NSE_OK;
  }
  if (!NSE_CUDA(cudaMemcpyAsync(host, x->f[id].p, n * sizeof(double), cudaMemcpyDeviceToHost,
                                x->stream)))
    return status_or(NSE_ERR_CUDA);
  return NSE_CUDA(cudaStreamSynchronize(x->stream)) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

int nse_ctx_grid(nse_ctx* x, double* xx, double* x12, double* y, double* y12, double* z,
                 double* z12, double* dx, double* dx12, double* dy, double* dy12, double* dz,
                 double* dz12) {
  if (!x) return NSE_ERR_ARG;
  auto cp = [](double* dst, const std::vector<double>& v) {
    if (dst) memcpy(dst, v.data(), v.size() * sizeof(double));
  };
  cp(xx, x->hx); cp(x12, x->hx12); cp(y, x->hy); cp(y12, x->hy12); cp(z, x->hz); cp(z12, x->hz12);
  cp(dx, x->hdx); cp(dx12, x->hdx12); cp(dy, x->hdy); cp(dy12, x->hdy12); cp(dz, x->hdz);
  cp(dz12, x->hdz12);
  return NSE_OK;
}

int nse_ctx_set_step(nse_ctx* x, int l) {
  if (!x || l < 1) return NSE_ERR_ARG;
  x->l = l;
  return NSE_OK;
}
int nse_ctx_get_step(nse_ctx* x) { return x ? x->l : -1; }

int nse_start(nse_ctx* x) {
  if (!x) return NSE_ERR_ARG;
  size_t fb = x->d.ntot * sizeof(double);
  const int src[4] = {NSE_U, NSE_V, NSE_W, NSE_T};
  const int dst[4] = {NSE_U_PRE, NSE_V_PRE, NSE_W_PRE, NSE_T_PRE};
  for (int q = 0; q < 4; ++q) {
    if (x->mixed) {
      launch_round_table(F(x, src[q]), F32(x, dst[q]), (long)x->d.ntot, x->stream);
      continue;
    }
    if (!NSE_CUDA(cudaMemcpyAsync(x->f[dst[q]].p, x->f[src[q]].p, fb, cudaMemcpyDeviceToDevice,
                                  x->stream)))
      return status_or(NSE_ERR_CUDA);
  }
  return NSE_CUDA(cudaGetLastError()) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

// the three-pass Poisson solve (k_poisson2d.cu) of the fast forms, when asked
// for with NSE_FLAG_POISSON3 (NX = NZ = 256 and ny = 16 m)
static bool poisson3(const nse_ctx* x) {
  return (x->cfg.flags & NSE_FLAG_POISSON3) && !(x->cfg.flags & NSE_FLAG_EXACT) &&
         poisson3_ok(x->pb.pp);
}

// SPN + SP0B of the fast forms (FP64 spectrum): the TMA-tile solver with
// NSE_FLAG_SPN_TMA, else the two-ended solver
static void ctx_spn(nse_ctx* x, bool part) {
  const PoissonPlan& pp = x->pb.pp;
  if ((x->cfg.flags & NSE_FLAG_SPN_TMA) && launch_spn_tma(pp, x->stream)) return;
  if (part) launch_spn_part(pp, x->stream);
  else launch_spn_fast(pp, x->stream);
}

// z forward -> SPN/SP0B -> z inverse of the FP64 five-pass solve, phase-
// marked; in kx slices (launch_poisson_mid) when the autotuner chose them,
// all three passes then counted as the SPN phase
static void ctx_poisson_mid(nse_ctx* x, bool part) {
  const PoissonPlan& pp = x->pb.pp;
  cudaStream_t s = x->stream;
  if (x->mid_chunks > 1 && !part && !(x->cfg.flags & NSE_FLAG_SPN_TMA)) {
    mark(x, PH_FFTZ_F);
    mark(x, PH_SPN);
    launch_poisson_mid(pp, x->mid_chunks, s);
    mark(x, PH_FFTZ_I);
    return;
  }
  mark(x, PH_FFTZ_F);
  launch_fft_z(pp, false, s);
  mark(x, PH_SPN);
  ctx_spn(x, part);
  mark(x, PH_FFTZ_I);
  launch_fft_z(pp, true, s);
}

// The number of kx slices of the middle passes, timed before the first FP64
// solve of a context while the spectrum holds nothing the solve needs (the
// forward x pass overwrites all of it next): the candidates run the three
// passes on whatever the spectrum holds, which costs the same time as on a
// real spectrum and changes no state.
// The form of the two-ended SPN (TMA tiles or per-thread cp.async staging;
// the same bits), timed once per grid before the first FP64 solve of a
// context: the spectrum is zeroed first (the forward x pass overwrites all of
// it next), so the candidates time the solve on defined values.
static void autotune_spn_form(nse_ctx* x) {
  if (x->spn_tuned) return;
  PoissonPlan& pp = x->pb.pp;
  if (!pp.spn_im || (x->cfg.flags & (NSE_FLAG_EXACT | NSE_FLAG_SPN_TMA | NSE_FLAG_SPN_CPASYNC |
                                     NSE_FLAG_NO_AUTOTUNE))) {
    x->spn_tuned = true;
    return;
  }
  cudaStream_t s = x->stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  char key[96];
  snprintf(key, sizeof(key), "spn %d %d %d", x->d.nx, x->d.ny, x->d.nz);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      pp.spn_cp = it->second;
      x->spn_tuned = true;
      return;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  cudaMemsetAsync(pp.spec, 0, 2 * sizeof(double) * (size_t)pp.Hp * pp.ny * pp.nz, s);
  int best = 0;
  float best_ms = 1e30f;
  for (int form = 0; form < 2; ++form) {
    pp.spn_cp = form;
    launch_spn_fast(pp, s);
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; ++r) launch_spn_fast(pp, s);
    cudaEventRecord(e1, s);
    float ms = 1e30f;
    if (cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best_ms) {
      best_ms = ms;
      best = form;
    }
    tune_log(key, form, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pp.spn_cp = best;
  x->spn_tuned = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
}

static void autotune_mid(nse_ctx* x) {
  autotune_spn_form(x);
  if (x->mid_tuned) return;
  const PoissonPlan& pp = x->pb.pp;
  const int G = poisson_mid_groups(pp);
  if (G < 2 || (x->cfg.flags & (NSE_FLAG_EXACT | NSE_FLAG_SPN_TMA))) {
    x->mid_tuned = true;
    return;
  }
  if (x->cfg.flags & (NSE_FLAG_MID_SLICES | NSE_FLAG_NO_AUTOTUNE)) {
    x->mid_chunks = (x->cfg.flags & NSE_FLAG_MID_SLICES) ? (G < 3 ? G : 3) : 1;
    x->mid_tuned = true;
    return;
  }
  cudaStream_t s = x->stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  char key[96];
  snprintf(key, sizeof(key), "mid %d %d %d", x->d.nx, x->d.ny, x->d.nz);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      x->mid_chunks = it->second;
      x->mid_tuned = true;
      return;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  int best = 1;
  float best_ms = 1e30f;
  const int cand[5] = {1, 2, 3, 5, 9};
  for (int ci = 0; ci < 5; ++ci) {
    const int nc = cand[ci];
    if (nc > G) break;
    launch_poisson_mid(pp, nc, s);
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; ++r) launch_poisson_mid(pp, nc, s);
    cudaEventRecord(e1, s);
    float ms = 1e30f;
    if (cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best_ms) {
      best_ms = ms;
      best = nc;
    }
    tune_log(key, nc, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  x->mid_chunks = best;
  x->mid_tuned = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
}

// P2S -> SPN/SP0B -> S2P -> PHIBC on phi (FP64), phase-marked
static void ctx_poisson64(nse_ctx* x, double* phi, bool div_marked) {
  const Dims& d = x->d;
  cudaStream_t s = x->stream;
  const PoissonPlan& pp = x->pb.pp;
  if (!div_marked) mark(x, PH_FFTX_F);
  if (poisson3(x)) {
    launch_p2s256(pp, d, phi, s);
    mark(x, PH_FFTZ_F);
    mark(x, PH_SPN);
    ctx_spn(x, true);
    mark(x, PH_FFTZ_I);
    mark(x, PH_FFTX_I);
    launch_s2p256_phibc(pp, d, phi, s);
    mark(x, PH_PHIBC);
    return;
  }
  if (!div_marked) autotune_mid(x);
  launch_fft_fwd_x(pp, d, phi, nullptr, nullptr, nullptr, x->g, 1.0, 0, s);
  ctx_poisson_mid(x, false);
  mark(x, PH_FFTX_I);
  launch_fft_inv_x(pp, d, phi, s);
  mark(x, PH_PHIBC);
  launch_phibc(d, phi, s);
}

// The pipelined correction's launch shapes, timed inside the first step's
// MKP with the solved phi: the kernel reads the old u_ta and writes the new
// one in place, so the timing runs read and write scratch copies of u_ta (its
// other outputs are rewritten by the step's own correction right after).
extern "C++" {
template <class H>
static void autotune_correct(nse_ctx* x, const H* ut, const H* vt, const H* wt) {
  if (x->corr_tuned) return;
  if (x->cfg.flags & (NSE_FLAG_NO_AUTOTUNE | NSE_FLAG_EXACT)) {
    x->corr_tuned = true;
    return;
  }
  cudaStream_t s = x->stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  const Dims& d = x->d;
  char key[96];
  snprintf(key, sizeof(key), "corr %d %d %d %d", d.nx, d.ny, d.nz, x->mixed ? 1 : 0);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      x->corr_shape = it->second;
      x->corr_tuned = true;
      return;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  const size_t hb = d.ntot * sizeof(H);
  H* ta[3] = {x->sa.as<H>(), x->sb.as<H>(), x->tmp.as<H>()};
  const int tid[3] = {NSE_U_TA, NSE_V_TA, NSE_W_TA};
  for (int q = 0; q < 3; ++q)
    cudaMemcpyAsync(ta[q], x->f[tid[q]].p, hb, cudaMemcpyDeviceToDevice, s);
  int best = 0;
  float best_ms = 1e30f;
  const int nshape = sizeof(H) == 4 ? 4 : 16;  // shapes 4-15: the FP64 TMA rings
  for (int shape = 0; shape < nshape; ++shape) {
    auto run = [&]() {
      if constexpr (sizeof(H) == 4)
        launch_correct_f32(d, x->rg, F(x, NSE_PHI), ut, vt, wt, F(x, NSE_P), F(x, NSE_U),
                           F(x, NSE_V), F(x, NSE_W), ta[0], ta[1], ta[2], F32(x, NSE_U_EP2),
                           F32(x, NSE_V_EP2), F32(x, NSE_W_EP2), F32(x, NSE_DIVU), x->cfg.dt, s,
                           shape);
      else
        launch_correct_pipe(d, x->rg, F(x, NSE_PHI), ut, vt, wt, F(x, NSE_P), F(x, NSE_U),
                            F(x, NSE_V), F(x, NSE_W), ta[0], ta[1], ta[2], F(x, NSE_U_EP2),
                            F(x, NSE_V_EP2), F(x, NSE_W_EP2), F(x, NSE_DIVU), x->cfg.dt, s,
                            shape);
    };
    run();
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; ++r) run();
    cudaEventRecord(e1, s);
    float ms = 1e30f;
    if (cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best_ms) {
      best_ms = ms;
      best = shape;
    }
    tune_log(key, shape, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  x->corr_shape = best;
  x->corr_tuned = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
}
}  // extern "C++"

// MKP in the mixed-precision form: FP32 u*, v*, w*; the FP64 solve of their
// FP64 divergence (or, with NSE_FLAG_POISSON32, the FP32 spectral solve with
// FP64 residual refinement); FP64 correction of the FP64 state
static void ctx_mkp_f32(nse_ctx* x, const float* ut, const float* vt, const float* wt) {
  const Dims& d = x->d;
  cudaStream_t s = x->stream;
  const PoissonPlan& pp = x->pb.pp;
  double* phi = F(x, NSE_PHI);
  const double dt = x->cfg.dt, dx = x->hdx[1], dz = x->hdz[1];
  const bool p64 = (x->cfg.flags & NSE_FLAG_POISSON32) == 0;
  mark(x, PH_FFTX_F);
  if (p64 && poisson3(x)) {
    launch_div_src32(d, x->rg, ut, vt, wt, dt, phi, s);
    ctx_poisson64(x, phi, true);
  } else if (p64) {
    autotune_mid(x);
    launch_div_src32(d, x->rg, ut, vt, wt, dt, phi, s);
    launch_fft_fwd_x(pp, d, phi, nullptr, nullptr, nullptr, x->g, 1.0, 0, s);
  } else {
    launch_fft_fwd_x_f32(pp, d, x->g, x->rg, ut, vt, wt, dt, nullptr, dx, dz, 1, s);
  }
  if (!(p64 && poisson3(x))) {
    if (p64) {
      ctx_poisson_mid(x, false);
    } else {
      mark(x, PH_FFTZ_F);
      launch_fft_z_f32(pp, false, s);
      mark(x, PH_SPN);
      launch_spn_fast_f32(pp, s);
      mark(x, PH_FFTZ_I);
      launch_fft_z_f32(pp, true, s);
    }
    mark(x, PH_FFTX_I);
    if (p64) launch_fft_inv_x(pp, d, phi, s);
    else launch_fft_inv_x_f32(pp, d, phi, false, s);
    mark(x, PH_PHIBC);
    launch_phibc(d, phi, s);
  }
  mark(x, PH_REFINE);
  for (int r = 0; !p64 && r < x->refine; ++r) {
    launch_fft_fwd_x_f32(pp, d, x->g, x->rg, ut, vt, wt, dt, phi, dx, dz, 2, s);
    launch_fft_z_f32(pp, false, s);
    launch_spn_fast_f32(pp, s);
    launch_fft_z_f32(pp, true, s);
    launch_fft_inv_x_f32(pp, d, phi, true, s);
    launch_phibc(d, phi, s);
  }
  if (!x->rec) autotune_correct<float>(x, ut, vt, wt);
  mark(x, PH_CORRECT);
  launch_correct_f32(d, x->rg, phi, ut, vt, wt, F(x, NSE_P), F(x, NSE_U), F(x, NSE_V),
                     F(x, NSE_W), F32(x, NSE_U_TA), F32(x, NSE_V_TA), F32(x, NSE_W_TA),
                     F32(x, NSE_U_EP2), F32(x, NSE_V_EP2), F32(x, NSE_W_EP2), F32(x, NSE_DIVU),
                     dt, s, x->corr_shape);
  mark(x, PH_COUNT);
}

// MKP (mkp.f:9-220) with u_temp = (ut, vt, wt); writes u, v, w, p, u_ta,
// u_ep2, divu of the context and leaves phi in the NSE_PHI field
static void ctx_mkp(nse_ctx* x, const double* ut, const double* vt, const double* wt) {
  const Dims& d = x->d;
  cudaStream_t s = x->stream;
  double* phi = F(x, NSE_PHI);
  const PoissonPlan& pp = x->pb.pp;
  const GridRcp* rg = (x->cfg.flags & NSE_FLAG_EXACT) ? nullptr : &x->rg;
  mark(x, PH_FFTX_F);
  if (rg && poisson3(x)) {
    launch_div_src(d, *rg, ut, vt, wt, x->cfg.dt, phi, s);
    ctx_poisson64(x, phi, true);
  } else if (rg) {
    autotune_mid(x);
    // phi is free until the inverse x pass: it holds the divergence samples
    launch_div_src(d, *rg, ut, vt, wt, x->cfg.dt, phi, s);
    launch_fft_fwd_x(pp, d, phi, nullptr, nullptr, nullptr, x->g, 1.0, 0, s);
  } else {
    launch_fft_fwd_x(pp, d, nullptr, ut, vt, wt, x->g, x->cfg.dt, 1, s, rg);
  }
  if (!(rg && poisson3(x))) {
    if (rg) {
      ctx_poisson_mid(x, false);
    } else {
      mark(x, PH_FFTZ_F);
      launch_fft_z(pp, false, s);
      mark(x, PH_SPN);
      launch_spn_fast(pp, s);
      mark(x, PH_FFTZ_I);
      launch_fft_z(pp, true, s);
    }
    mark(x, PH_FFTX_I);
    launch_fft_inv_x(pp, d, phi, s);
    mark(x, PH_PHIBC);
    launch_phibc(d, phi, s);
  }
  mark(x, PH_REFINE);
  mark(x, PH_CORRECT);
  if (x->cfg.flags & NSE_FLAG_EXACT)
    launch_correct(d, x->g, phi, ut, vt, wt, F(x, NSE_P), F(x, NSE_U), F(x, NSE_V), F(x, NSE_W),
                   F(x, NSE_U_TA), F(x, NSE_V_TA), F(x, NSE_W_TA), F(x, NSE_U_EP2),
                   F(x, NSE_V_EP2), F(x, NSE_W_EP2), F(x, NSE_DIVU), x->cfg.dt, s);
  else {
    if (!x->rec) autotune_correct<double>(x, ut, vt, wt);
    launch_correct_pipe(d, x->rg, phi, ut, vt, wt, F(x, NSE_P), F(x, NSE_U), F(x, NSE_V),
                        F(x, NSE_W), F(x, NSE_U_TA), F(x, NSE_V_TA), F(x, NSE_W_TA),
                        F(x, NSE_U_EP2), F(x, NSE_V_EP2), F(x, NSE_W_EP2), F(x, NSE_DIVU),
                        x->cfg.dt, s, x->corr_shape);
  }
  mark(x, PH_COUNT);
}

int nse_project(nse_ctx* x) {
  if (!x) return NSE_ERR_ARG;
  size_t fb = x->d.ntot * sizeof(double);
  cudaStream_t s = x->stream;
  // the boundary conditions of u, v, w are applied first, as the time loop
  // does before MKP (nse_dominik.f:441): walls v = 0 and periodic ghosts make
  // the divergence compatible with the Neumann problem
  const nse_config& c = x->cfg;
  if (x->mixed) {
    const long n = (long)x->d.ntot;
    float *ua = x->ua.as<float>(), *va = x->va.as<float>(), *wa = x->wa.as<float>();
    launch_round_table(F(x, NSE_U), ua, n, s);
    launch_round_table(F(x, NSE_V), va, n, s);
    launch_round_table(F(x, NSE_W), wa, n, s);
    launch_set_bc_f32(x->d, ua, va, wa, nullptr, nullptr, c.t_bot, c.t_top, 7, s);
    ctx_mkp_f32(x, ua, va, wa);
    return NSE_CUDA(cudaGetLastError()) ? NSE_OK : status_or(NSE_ERR_CUDA);
  }
  if (!NSE_CUDA(cudaMemcpyAsync(x->ua.p, x->f[NSE_U].p, fb, cudaMemcpyDeviceToDevice, s)) ||
      !NSE_CUDA(cudaMemcpyAsync(x->va.p, x->f[NSE_V].p, fb, cudaMemcpyDeviceToDevice, s)) ||
      !NSE_CUDA(cudaMemcpyAsync(x->wa.p, x->f[NSE_W].p, fb, cudaMemcpyDeviceToDevice, s)))
    return status_or(NSE_ERR_CUDA);
  launch_set_bc(x->d, x->ua.as<double>(), x->va.as<double>(), x->wa.as<double>(), nullptr,
                nullptr, c.t_bot, c.t_top, 7, s);
  ctx_mkp(x, x->ua.as<double>(), x->va.as<double>(), x->wa.as<double>());
  return NSE_CUDA(cudaGetLastError()) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

int nse_poisson(nse_ctx* x) {
  if (!x) return NSE_ERR_ARG;
  ctx_poisson64(x, F(x, NSE_PHI), false);
  return NSE_CUDA(cudaGetLastError()) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

// ------------------------------------------------------------- autotuner --
// The partitioned line passes have several launch shapes that give the same
// values: y/z lines 16, 8 or 32 lines per CTA (the y/z line-to-warp mapping:
// with L lines per CTA a warp holds min(L, 32) lines of 32/L partitions), and
// x lines one or two per warp iteration.  (The TMA tiles of the FP64 y/z
// lines are a further shape, set only by NSE_FLAG_LINES_TMA.)  Before a context's first step (outside any stream capture)
// every candidate of every pass is timed on a scratch copy of the pass's
// field (CUDA events, one warm-up and three timed runs, the fastest kept).
// Choices are kept per grid and form for the process, so the cases of an
// ensemble that share a grid are timed once.  NSE_FLAG_NO_AUTOTUNE keeps
// the fixed shapes (16 lines per CTA, two x lines per warp iteration);
// NSE_FLAG_LINES_TMA sets the TMA tiles for every FP64 y/z pass.

static int x_nl_candidates(const nse_ctx* x) { return x_rows_per_lane(x->d.nx) <= 8 ? 2 : 1; }

static void autotune_lines(nse_ctx* x) {
  if (x->tuned || !x->part) return;
  const int flags = x->cfg.flags;
  if (flags & NSE_FLAG_LINES_TMA) {
    for (int dir = 1; dir <= 2; ++dir)
      for (int comp = 0; comp < 4; ++comp) x->yzshape[dir][comp] = x->mixed ? 0 : 2;
    x->tuned = true;
    return;
  }
  if (flags & NSE_FLAG_NO_AUTOTUNE) {
    x->tuned = true;
    return;
  }
  cudaStream_t s = x->stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  const Dims& d = x->d;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  const int form = x->mixed ? (x->lines64 ? 2 : 1) : 0;
  size_t fbytes = d.ntot * (x->mixed ? sizeof(float) : sizeof(double));
  for (int comp = 0; comp < 4; ++comp) {
    void* src = comp == 0 ? x->ua.p : comp == 1 ? x->va.p : comp == 2 ? x->wa.p : x->uT.p;
    for (int dir = 0; dir < 3; ++dir) {
      char key[96];
      snprintf(key, sizeof(key), "%d %d %d %d %d %d", d.nx, d.ny, d.nz, dir,
               line_kind(dir, comp), form);
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
          if (dir == 0) x->xnl[comp] = it->second;
          else x->yzshape[dir][comp] = it->second;
          continue;
        }
      }
      std::vector<int> cand;
      if (dir == 0) {
        if (x_nl_candidates(x) < 2) continue;
        cand = {2, 1};
        // the staged loads (one warp per line, M = nx/32 even)
        const int M = x_rows_per_lane(d.nx);
        if (d.nx % 32 == 0 && (M == 4 || M == 6 || M == 8)) {
          cand.push_back(3);
          cand.push_back(4);
        }
      } else if (x->mixed) {
        cand = {0, 1, 3};
      } else {
        cand = {0, 1, 3, 2};  // 2: the FP64 TMA tiles
      }
      int best = cand[0];
      float best_ms = 1e30f;
      for (int c : cand) {
        cudaMemcpyAsync(x->sa.p, src, fbytes, cudaMemcpyDeviceToDevice, s);
        LineArgs la = line_args(x, comp);
        la.ft = 0.0;
        la.fb = 0.0;
        if (dir == 0) la.xnl = c;
        else la.yzshape = c;
        auto run = [&]() {
          if (x->mixed)
            launch_lines_part_f32(dir, line_kind(dir, comp), d, x->sa.as<float>(), nullptr, la,
                                  x->ptab_f[dir][comp].as<float>(),
                                  x->slots[dir][comp].as<int>(), x->ids[dir][comp].as<int>(),
                                  x->nmasked[dir][comp], x->pmtab_f[dir][comp].as<float>(),
                                  x->lines64 ? x->ptab[dir][comp].as<double>() : nullptr,
                                  x->lines64 ? x->pmtab[dir][comp].as<double>() : nullptr, s);
          else
            launch_lines_part(dir, line_kind(dir, comp), d, x->sa.as<double>(), la,
                              x->ptab[dir][comp].as<double>(), x->slots[dir][comp].as<int>(),
                              x->ids[dir][comp].as<int>(), x->nmasked[dir][comp],
                              x->pmtab[dir][comp].as<double>(), s);
        };
        run();
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r) run();
        cudaEventRecord(e1, s);
        float ms = 1e30f;
        if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) ==
                                                           cudaSuccess && ms < best_ms) {
          best_ms = ms;
          best = c;
        }
        tune_log(key, c, ms);
      }
      if (dir == 0) x->xnl[comp] = best;
      else x->yzshape[dir][comp] = best;
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune[key] = best;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  x->tuned = true;
}

// The fast right-hand-side kernel's launch shapes (tile height, ring depth,
// CTAs per SM; every shape computes each cell the same way) are timed the same
// way before the first step: the four AB2 histories, which the kernel reads
// and rewrites, are copied to scratch fields first, so the timing runs change
// no state (their outputs go to the step's work fields, which the step's own
// right-hand side then overwrites).
static void autotune_rhs(nse_ctx* x, const StepParams& sp) {
  if (x->rhs_tuned) return;
  if (x->cfg.flags & (NSE_FLAG_NO_AUTOTUNE | NSE_FLAG_EXACT)) {
    x->rhs_tuned = true;
    return;
  }
  cudaStream_t s = x->stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  const Dims& d = x->d;
  char key[96];
  snprintf(key, sizeof(key), "rhs %d %d %d %d %d", d.nx, d.ny, d.nz, x->mixed ? 1 : 0,
           x->math64 ? 1 : 0);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      x->rhs_shape = it->second;
      x->rhs_tuned = true;
      return;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  const size_t hb = d.ntot * (x->mixed ? sizeof(float) : sizeof(double));
  // the fourth history copy gets a buffer of its own, released after the
  // timing: phi must not serve as scratch, because the Poisson solve never
  // writes some of its ghost entries (as in the reference) and the
  // correction's face pass reads them
  DBuf extra;
  if (!extra.ensure(hb)) {  // no room: keep the default shape, report nothing
    nse_clear_error();
    cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    x->rhs_tuned = true;
    return;
  }
  void* hist[4] = {x->sa.p, x->sb.p, x->tmp.p, extra.p};
  const int hid[4] = {NSE_U_PRE, NSE_V_PRE, NSE_W_PRE, NSE_T_PRE};
  for (int q = 0; q < 4; ++q)
    cudaMemcpyAsync(hist[q], x->f[hid[q]].p, hb, cudaMemcpyDeviceToDevice, s);
  const double *u = F(x, NSE_U), *v = F(x, NSE_V), *w = F(x, NSE_W), *T = F(x, NSE_T);
  const double* c1 = F(x, NSE_CELLVALUE);
  int best = 0;
  float best_ms = 1e30f;
  const int nshape = 7;  // shapes 4-6: the TMA rings
  for (int shape = 0; shape < nshape; ++shape) {
    auto run = [&]() {
      if (x->mixed)
        launch_rhs_f32(d, x->g, x->rg, sp, u, v, w, T, F32(x, NSE_U_TA), F32(x, NSE_V_TA),
                       F32(x, NSE_W_TA), (float*)hist[0], (float*)hist[1], (float*)hist[2],
                       (float*)hist[3], c1, x->ua.as<float>(), x->va.as<float>(),
                       x->wa.as<float>(), x->uT.as<float>(), x->math64, s, shape);
      else
        launch_rhs_fast(d, x->g, x->rg, sp, u, v, w, T, F(x, NSE_U_TA), F(x, NSE_V_TA),
                        F(x, NSE_W_TA), (double*)hist[0], (double*)hist[1], (double*)hist[2],
                        (double*)hist[3], c1, x->ua.as<double>(), x->va.as<double>(),
                        x->wa.as<double>(), x->uT.as<double>(), s, shape);
    };
    run();
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; ++r) run();
    cudaEventRecord(e1, s);
    float ms = 1e30f;
    if (cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best_ms) {
      best_ms = ms;
      best = shape;
    }
    tune_log(key, shape, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  extra.release();
  x->rhs_shape = best;
  x->rhs_tuned = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
}

// one time step in the mixed-precision form: FP64 state u, v, w, T, p;
// FP32 right-hand side, line sweeps and transforms
static void ctx_step_f32(nse_ctx* x) {
  const Dims& d = x->d;
  const nse_config& c = x->cfg;
  cudaStream_t s = x->stream;
  StepParams sp;
  sp.dt = c.dt; sp.Re = c.Re; sp.Sc = c.Sc; sp.eta = c.eta;
  sp.force = c.body_force; sp.source = c.heat_source;
  sp.tbot = c.t_bot; sp.ttop = c.t_top; sp.tsolid = c.t_solid;
  sp.rho_cp = c.rho_cp; sp.thc = c.thc; sp.l = x->l;
  double *u = F(x, NSE_U), *v = F(x, NSE_V), *w = F(x, NSE_W), *p = F(x, NSE_P);
  double* T = F(x, NSE_T);
  const double* c1 = F(x, NSE_CELLVALUE);
  float *ua = x->ua.as<float>(), *va = x->va.as<float>(), *wa = x->wa.as<float>();
  float* uT = x->uT.as<float>();
  mark(x, PH_BC);
  launch_set_bc(d, u, v, w, p, T, c.t_bot, c.t_top, 31, s);
  mark(x, PH_RHS);
  autotune_rhs(x, sp);
  launch_rhs_f32(d, x->g, x->rg, sp, u, v, w, T, F32(x, NSE_U_TA), F32(x, NSE_V_TA),
                 F32(x, NSE_W_TA), F32(x, NSE_U_PRE), F32(x, NSE_V_PRE), F32(x, NSE_W_PRE),
                 F32(x, NSE_T_PRE), c1, ua, va, wa, uT, x->math64, s, x->rhs_shape);
  refresh_line_flags(x, s);
  autotune_lines(x);
  float* fa[3] = {ua, va, wa};
  auto run_on = [&](cudaStream_t st, int dir, int comp, float* f, double* out, double ft,
                    double fb) {
    LineArgs la = line_args(x, comp);
    line_shape(x, dir, comp, la);
    la.ft = ft;
    la.fb = fb;
    launch_lines_part_f32(dir, line_kind(dir, comp), d, f, out, la,
                          x->ptab_f[dir][comp].as<float>(), x->slots[dir][comp].as<int>(),
                          x->ids[dir][comp].as<int>(), x->nmasked[dir][comp],
                          x->pmtab_f[dir][comp].as<float>(),
                          x->lines64 ? x->ptab[dir][comp].as<double>() : nullptr,
                          x->lines64 ? x->pmtab[dir][comp].as<double>() : nullptr, st);
  };
  auto run = [&](int dir, int comp, float* f, double* out, double ft, double fb) {
    run_on(s, dir, comp, f, out, ft, fb);
  };
  // the four components' chains on concurrent streams, as in the FP64 form
  if (concurrent(x)) {
    mark(x, PH_YVEL);
    NSE_CUDA(cudaEventRecord(x->lfork, s));
    for (int q = 0; q < 3; ++q) NSE_CUDA(cudaStreamWaitEvent(x->side[q], x->lfork, 0));
    cudaStream_t cs[4] = {s, x->side[0], x->side[1], x->side[2]};
    for (int comp = 0; comp < 3; ++comp) {
      run_on(cs[comp], 1, comp, fa[comp], nullptr, 0.0, 0.0);
      run_on(cs[comp], 2, comp, fa[comp], nullptr, 0.0, 0.0);
      run_on(cs[comp], 0, comp, fa[comp], nullptr, 0.0, 0.0);
    }
    run_on(cs[3], 1, 3, uT, nullptr, 2.0 * c.t_bot, 2.0 * c.t_top);
    run_on(cs[3], 0, 3, uT, nullptr, 0.0, 0.0);
    run_on(cs[3], 2, 3, uT, T, 0.0, 0.0);
    // the temperature chain sets T's ghosts itself and rejoins after MKP
    launch_set_bc_f32(d, nullptr, nullptr, nullptr, nullptr, T, c.t_bot, c.t_top, 16, cs[3]);
    for (int q = 0; q < 3; ++q) NSE_CUDA(cudaEventRecord(x->ljoin[q], x->side[q]));
    for (int q = 0; q < 2; ++q) NSE_CUDA(cudaStreamWaitEvent(s, x->ljoin[q], 0));
    for (int ph = PH_ZVEL; ph <= PH_ZT; ++ph) mark(x, ph);
    mark(x, PH_BC2);
    launch_set_bc_f32(d, ua, va, wa, p, T, c.t_bot, c.t_top, 1 | 2 | 4 | 8, s);
    ctx_mkp_f32(x, ua, va, wa);
    NSE_CUDA(cudaStreamWaitEvent(s, x->ljoin[2], 0));
    if (x->prof_n < x->prof_cap) x->prof_n++;
    x->l += 1;
    return;
  } else {
    mark(x, PH_YVEL);
    for (int comp = 0; comp < 3; ++comp) run(1, comp, fa[comp], nullptr, 0.0, 0.0);
    mark(x, PH_ZVEL);
    for (int comp = 0; comp < 3; ++comp) run(2, comp, fa[comp], nullptr, 0.0, 0.0);
    mark(x, PH_XVEL);
    for (int comp = 0; comp < 3; ++comp) run(0, comp, fa[comp], nullptr, 0.0, 0.0);
    // solve_t: y, x, z; the z sweep writes the new temperature (interior) to
    // the FP64 state
    mark(x, PH_YT);
    run(1, 3, uT, nullptr, 2.0 * c.t_bot, 2.0 * c.t_top);
    mark(x, PH_XT);
    run(0, 3, uT, nullptr, 0.0, 0.0);
    mark(x, PH_ZT);
    run(2, 3, uT, T, 0.0, 0.0);
  }
  mark(x, PH_BC2);
  launch_set_bc_f32(d, ua, va, wa, p, T, c.t_bot, c.t_top, 31, s);
  ctx_mkp_f32(x, ua, va, wa);
  if (x->prof_n < x->prof_cap) x->prof_n++;
  x->l += 1;
}

// one time step, nse_dominik.f:290-446
static void ctx_step(nse_ctx* x) {
  if (x->mixed) {
    ctx_step_f32(x);
    return;
  }
  const Dims& d = x->d;
  const nse_config& c = x->cfg;
  cudaStream_t s = x->stream;
  StepParams sp;
  sp.dt = c.dt; sp.Re = c.Re; sp.Sc = c.Sc; sp.eta = c.eta;
  sp.force = c.body_force; sp.source = c.heat_source;
  sp.tbot = c.t_bot; sp.ttop = c.t_top; sp.tsolid = c.t_solid;
  sp.rho_cp = c.rho_cp; sp.thc = c.thc; sp.l = x->l;
  double *u = F(x, NSE_U), *v = F(x, NSE_V), *w = F(x, NSE_W), *p = F(x, NSE_P);
  double* T = F(x, NSE_T);
  const double* c1 = F(x, NSE_CELLVALUE);
  double *ua = x->ua.as<double>(), *va = x->va.as<double>(), *wa = x->wa.as<double>();
  double* uT = x->uT.as<double>();
  LineScratch sc{x->sa.as<double>(), x->sb.as<double>()};
  // :290 set_bc(u,v,w,p,T)
  mark(x, PH_BC);
  launch_set_bc(d, u, v, w, p, T, c.t_bot, c.t_top, 31, s);
  mark(x, PH_RHS);
  // :299-396 explicit terms, AB2, set_bc(u_a,...) and the penalised updates
  if (!(c.flags & NSE_FLAG_EXACT) && !x->rec) autotune_rhs(x, sp);
  if (c.flags & NSE_FLAG_EXACT)
    launch_rhs_fused(d, x->g, sp, u, v, w, T, F(x, NSE_U_TA), F(x, NSE_V_TA), F(x, NSE_W_TA),
                     F(x, NSE_U_PRE), F(x, NSE_V_PRE), F(x, NSE_W_PRE), F(x, NSE_T_PRE), c1,
                     ua, va, wa, uT, s);
  else
    launch_rhs_fast(d, x->g, x->rg, sp, u, v, w, T, F(x, NSE_U_TA), F(x, NSE_V_TA),
                    F(x, NSE_W_TA), F(x, NSE_U_PRE), F(x, NSE_V_PRE), F(x, NSE_W_PRE),
                    F(x, NSE_T_PRE), c1, ua, va, wa, uT, s, x->rhs_shape);
  // :397 solve_u_temp: per component y, z, x line solves
  // (timed per direction: all y solves, then z, then x of the three fields;
  // the fields are independent, so this order gives the same values as
  // the reference's per-field y, z, x order)
  refresh_line_flags(x, s);
  if (!x->rec) autotune_lines(x);
  const bool exact = (c.flags & NSE_FLAG_EXACT) != 0;
  auto lines = exact ? launch_lines_exact : launch_lines_fast;
  double* fa[3] = {ua, va, wa};
  size_t fbytes = d.ntot * sizeof(double);
  // (on the stream of the component's chain, so each copy sees its pass's input)
  auto record_on = [&](cudaStream_t st, int comp, int pass, const double* f) {
    if (x->rec)
      NSE_CUDA(cudaMemcpyAsync(x->rec[4 * comp + pass], f, fbytes, cudaMemcpyDeviceToDevice, st));
  };
  auto record = [&](int comp, int pass, const double* f) { record_on(s, comp, pass, f); };
  auto run_on = [&](cudaStream_t st, int dir, int comp, double* f, int tab, double ft,
                    double fb) {
    record_on(st, comp,
              comp == 3 ? (dir == 1 ? 0 : (dir == 0 ? 1 : 2)) : (dir == 1 ? 0 : (dir == 2 ? 1 : 2)),
              f);
    LineArgs la = line_args(x, comp);
    line_shape(x, dir, comp, la);
    la.ft = ft;
    la.fb = fb;
    if (x->part)
      launch_lines_part(dir, line_kind(dir, comp), d, f, la, x->ptab[dir][comp].as<double>(),
                        x->slots[dir][comp].as<int>(), x->ids[dir][comp].as<int>(),
                        x->nmasked[dir][comp], x->pmtab[dir][comp].as<double>(), st);
    else
      lines(dir, line_kind(dir, comp), d, f, la, x->tab[tab], x->slots[dir][comp].as<int>(),
            x->mtab[dir][comp].as<double>(), st);
  };
  auto run = [&](int dir, int comp, double* f, int tab, double ft, double fb) {
    run_on(s, dir, comp, f, tab, ft, fb);
  };
  // The four components' chains are independent (each pass reads and writes
  // its own field with read-only tables): u on the context's stream, v, w
  // and T on side streams (an adjoint replay's recording copies go on the
  // same chains).  Profiled steps (each phase timed on its own) and
  // NSE_FLAG_ONE_STREAM keep the serial order.
  if (x->part && !exact && concurrent(x)) {
    mark(x, PH_YVEL);
    NSE_CUDA(cudaEventRecord(x->lfork, s));
    for (int q = 0; q < 3; ++q) NSE_CUDA(cudaStreamWaitEvent(x->side[q], x->lfork, 0));
    cudaStream_t cs[4] = {s, x->side[0], x->side[1], x->side[2]};
    for (int comp = 0; comp < 3; ++comp) {
      run_on(cs[comp], 1, comp, fa[comp], comp == 1 ? TB_Y_V : TB_Y_U, 0.0, 0.0);
      run_on(cs[comp], 2, comp, fa[comp], TB_Z_V, 0.0, 0.0);
      run_on(cs[comp], 0, comp, fa[comp], TB_X_V, 0.0, 0.0);
    }
    run_on(cs[3], 1, 3, uT, TB_Y_T, 2.0 * c.t_bot, 2.0 * c.t_top);
    run_on(cs[3], 0, 3, uT, TB_X_T, 0.0, 0.0);
    run_on(cs[3], 2, 3, uT, TB_Z_T, 0.0, 0.0);
    for (int comp = 0; comp < 4; ++comp) record_on(cs[comp], comp, 3, comp < 3 ? fa[comp] : uT);
    std::swap(x->f[NSE_T], x->uT);
    T = F(x, NSE_T);
    // MKP needs u*, v*, w* only: the temperature chain also sets T's ghosts
    // (the T part of set_bc, which reads interior cells only) and rejoins
    // at the end of the step, so it overlaps the projection
    launch_set_bc(d, nullptr, nullptr, nullptr, nullptr, T, c.t_bot, c.t_top, 16, cs[3]);
    for (int q = 0; q < 3; ++q) NSE_CUDA(cudaEventRecord(x->ljoin[q], x->side[q]));
    for (int q = 0; q < 2; ++q) NSE_CUDA(cudaStreamWaitEvent(s, x->ljoin[q], 0));
    for (int ph = PH_ZVEL; ph <= PH_ZT; ++ph) mark(x, ph);
    mark(x, PH_BC2);
    launch_set_bc(d, ua, va, wa, p, T, c.t_bot, c.t_top, 1 | 2 | 4 | 8, s);
    ctx_mkp(x, ua, va, wa);
    NSE_CUDA(cudaStreamWaitEvent(s, x->ljoin[2], 0));
    if (x->prof_n < x->prof_cap) x->prof_n++;
    x->l += 1;
    return;
  }
  mark(x, PH_YVEL);
  for (int comp = 0; comp < 3; ++comp)
    run(1, comp, fa[comp], comp == 1 ? TB_Y_V : TB_Y_U, 0.0, 0.0);
  mark(x, PH_ZVEL);
  for (int comp = 0; comp < 3; ++comp) run(2, comp, fa[comp], TB_Z_V, 0.0, 0.0);
  mark(x, PH_XVEL);
  for (int comp = 0; comp < 3; ++comp) run(0, comp, fa[comp], TB_X_V, 0.0, 0.0);
  // :419 solve_t: y, x, z
  mark(x, PH_YT);
  run(1, 3, uT, TB_Y_T, 2.0 * c.t_bot, 2.0 * c.t_top);
  mark(x, PH_XT);
  run(0, 3, uT, TB_X_T, 0.0, 0.0);
  mark(x, PH_ZT);
  run(2, 3, uT, TB_Z_T, 0.0, 0.0);
  for (int comp = 0; comp < 3; ++comp) record(comp, 3, fa[comp]);
  record(3, 3, uT);
  // :429-437 T = u_T (interior); the ghosts are rewritten by the next set_bc
  std::swap(x->f[NSE_T], x->uT);
  T = F(x, NSE_T);
  // :441 set_bc(u_temp,v_temp,w_temp,p,T)
  mark(x, PH_BC2);
  launch_set_bc(d, ua, va, wa, p, T, c.t_bot, c.t_top, 31, s);
  // :446 MKP
  ctx_mkp(x, ua, va, wa);
  if (x->prof_n < x->prof_cap) x->prof_n++;
  x->l += 1;
}

}  // extern "C"

// internal hooks of the adjoint driver (adjoint.cu)
namespace nse {
bool ctx_info(nse_ctx* x, CtxInfo& out) {
  if (!x) return false;
  out.d = x->d;
  out.g = x->g;
  out.rg = x->rg;
  out.cfg = &x->cfg;
  out.s = x->stream;
  out.pp = &x->pb.pp;
  out.mixed = x->mixed;
  return true;
}
double* ctx_field(nse_ctx* x, int id) { return F(x, id); }
int ctx_get_l(nse_ctx* x) { return x->l; }
void ctx_set_l(nse_ctx* x, int l) { x->l = l; }
void ctx_step_rec(nse_ctx* x, double* const* rec) {
  x->rec = rec;
  ctx_step(x);
  x->rec = nullptr;
}
// the step's line solve of (dir, comp) applied to the field f with zero wall
// values (the linear part of the pass), on stream s; FP64 contexts
void ctx_line_solve(nse_ctx* x, int dir, int comp, double* f, cudaStream_t s) {
  refresh_line_flags(x, s);
  LineArgs la = line_args(x, comp);
    line_shape(x, dir, comp, la);
  la.ft = 0.0;
  la.fb = 0.0;
  const Dims& d = x->d;
  if (x->part) {
    launch_lines_part(dir, line_kind(dir, comp), d, f, la, x->ptab[dir][comp].as<double>(),
                      x->slots[dir][comp].as<int>(), x->ids[dir][comp].as<int>(),
                      x->nmasked[dir][comp], x->pmtab[dir][comp].as<double>(), s);
    return;
  }
  static const int ytab[4] = {TB_Y_U, TB_Y_V, TB_Y_U, TB_Y_T};
  const int tab = dir == 1 ? ytab[comp] : (dir == 2 ? (comp == 3 ? TB_Z_T : TB_Z_V)
                                                    : (comp == 3 ? TB_X_T : TB_X_V));
  auto lines = (x->cfg.flags & NSE_FLAG_EXACT) ? launch_lines_exact : launch_lines_fast;
  lines(dir, line_kind(dir, comp), d, f, la, x->tab[tab], x->slots[dir][comp].as<int>(),
        x->mtab[dir][comp].as<double>(), s);
}
}  // namespace nse

extern "C" {

// One step as a replay of a captured CUDA graph of one step.  The step's
// launches depend on the host-side state only through the step counter
// (l == 1 is the Euler start) and the temperature buffer pair (the FP64 form
// swaps T and its work buffer every step), so from the third step on a step
// is the replay of the graph captured from the same starting buffer.  The
// first two steps, steps after the mask changed, profiled and recorded steps,
// and steps on a stream that is being captured run eagerly (false).  The
// capture leaves the host-side state of the step behind (counter, buffer
// pair) and is launched at once; a replay sets that state the same way.
// Returns 1 (replayed), 0 (step eagerly) or -1 (a CUDA error).  A launch
// shape, a masked line list's length or a table's place that differs from
// the capture drops the graphs (a new mask is tabulated by an eager step).
static int step_replay(nse_ctx* x) {
  if (x->sg_off || x->l < 3 || x->mask_dirty || x->prof_n < x->prof_cap || x->rec) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(x->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return 0;
  const unsigned long long sig = shape_sig(x);
  if (sig != x->sg_sig) {
    drop_step_graphs(x);
    x->sg_sig = sig;
  }
  void* t0 = x->f[NSE_T].p;
  int q = -1;
  for (int k = 0; k < 2; ++k)
    if (x->sg[k] && x->sg_t[k] == t0) q = k;
  if (q >= 0) {
    if (!NSE_CUDA(cudaGraphLaunch(x->sg[q], x->stream))) return -1;
    count_launches(x->sg_nk[q]);
    x->f[NSE_T] = x->sg_T[q];
    x->uT = x->sg_uT[q];
    x->l += 1;
    return 1;
  }
  q = x->sg[0] ? 1 : 0;
  if (x->sg[q]) {
    cudaGraphExecDestroy(x->sg[q]);
    x->sg[q] = nullptr;
  }
  const int l0 = x->l;
  const DBuf T0 = x->f[NSE_T], uT0 = x->uT;
  if (cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    x->sg_off = true;
    return 0;
  }
  const long long k0 = g_launches.load();
  ctx_step(x);
  const long long nk = g_launches.load() - k0;  // counted once: the launch below
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(x->stream, &g);
  cudaGraphExec_t ex = nullptr;
  const bool ok = ce == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    // nothing ran: put the host-side state back and step eagerly
    cudaGetLastError();
    count_launches(-nk);
    x->l = l0;
    x->f[NSE_T] = T0;
    x->uT = uT0;
    x->sg_off = true;
    return 0;
  }
  if (!NSE_CUDA(cudaGraphLaunch(ex, x->stream))) {
    cudaGraphExecDestroy(ex);
    count_launches(-nk);
    x->l = l0;
    x->f[NSE_T] = T0;
    x->uT = uT0;
    return -1;
  }
  x->sg[q] = ex;
  x->sg_nk[q] = nk;
  x->sg_t[q] = t0;
  x->sg_T[q] = x->f[NSE_T];
  x->sg_uT[q] = x->uT;
  return 1;
}

int nse_step(nse_ctx* x, int nsteps) {
  if (!x || nsteps < 0) return NSE_ERR_ARG;
  for (int n = 0; n < nsteps; ++n) {
    const int r = step_replay(x);
    if (r < 0) return status_or(NSE_ERR_CUDA);
    if (r == 0) ctx_step(x);
    if (!NSE_CUDA(cudaGetLastError())) return status_or(NSE_ERR_CUDA);
    if (x->cfg.flags & 1) {  // check for non-finite values after every step
      double m[6];
      int st = nse_monitor(x, m);
      if (st != NSE_OK) return st;
      if (m[5] > 0) {
        set_error(NSE_ERR_NONFINITE, "nse_step: %g non-finite cells after step %d", m[5],
                  x->l - 1);
        return NSE_ERR_NONFINITE;
      }
    }
  }
  return NSE_OK;
}

int nse_levelset(nse_ctx* x, const double* phi0, double* phi_out, int nnn, double dtau,
                 double width) {
  if (!x || !phi0 || nnn < 0) return NSE_ERR_ARG;
  const Dims& d = x->d;
  cudaStream_t s = x->stream;
  // phi0 staged in the tmp work buffer, phi computed in NSE_PHI with ua as
  // the ping-pong buffer
  if (!NSE_CUDA(cudaMemcpyAsync(x->tmp.p, phi0, d.ntot * sizeof(double), cudaMemcpyHostToDevice, s)))
    return status_or(NSE_ERR_CUDA);
  x->mask_dirty = true;
  if (!run_levelset(d, x->g, x->tmp.as<double>(), F(x, NSE_PHI), x->ua.as<double>(),
                    F(x, NSE_CELLVALUE), nnn, dtau, width, s))
    return status_or(NSE_ERR_CUDA);
  // keep the level set: NSE_PHI is the Poisson work field of the steps
  if (!x->lsphi.ensure(d.ntot * sizeof(double)) ||
      !NSE_CUDA(cudaMemcpyAsync(x->lsphi.p, x->f[NSE_PHI].p, d.ntot * sizeof(double),
                                cudaMemcpyDeviceToDevice, s)))
    return status_or(NSE_ERR_CUDA);
  if (phi_out &&
      !NSE_CUDA(cudaMemcpyAsync(phi_out, x->f[NSE_PHI].p, d.ntot * sizeof(double),
                                cudaMemcpyDeviceToHost, s)))
    return status_or(NSE_ERR_CUDA);
  // the Poisson work field goes back to zero: MKP's PHI is a separate array
  // in the reference (mkp.f:21), and the ghost entries its solve never writes
  // (read by the correction's face pass) must not keep level-set values
  if (!NSE_CUDA(cudaMemsetAsync(x->f[NSE_PHI].p, 0, d.ntot * sizeof(double), s)))
    return status_or(NSE_ERR_CUDA);
  return NSE_CUDA(cudaStreamSynchronize(s)) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

// ----------------------------------------------- reference output files --
static bool download_vec(nse_ctx* x, int id, std::vector<double>& v) {
  v.resize(id == NSE_CELLVALUE ? x->d.ncell : x->d.ntot);
  return nse_ctx_download(x, id, v.data()) == NSE_OK;
}
static bool download_lsphi(nse_ctx* x, std::vector<double>& v) {
  v.assign(x->d.ntot, 0.0);
  if (!x->lsphi.p) return true;
  return NSE_CUDA(cudaMemcpyAsync(v.data(), x->lsphi.p, x->d.ntot * sizeof(double),
                                  cudaMemcpyDeviceToHost, x->stream)) &&
         NSE_CUDA(cudaStreamSynchronize(x->stream));
}

int nse_ctx_write_output(nse_ctx* x, const char* root) {
  if (!x || !root) return NSE_ERR_ARG;
  const Dims& d = x->d;
  std::vector<double> u, v, w, p, T, uta, vta, wta, divu, phi, cv;
  bool ok = download_vec(x, NSE_U, u) && download_vec(x, NSE_V, v) &&
            download_vec(x, NSE_W, w) && download_vec(x, NSE_P, p) &&
            download_vec(x, NSE_T, T) && download_vec(x, NSE_U_TA, uta) &&
            download_vec(x, NSE_V_TA, vta) && download_vec(x, NSE_W_TA, wta) &&
            download_vec(x, NSE_DIVU, divu) && download_lsphi(x, phi);
  if (!ok) return status_or(NSE_ERR_CUDA);
  // cellvalue(:,:,:,1) is the mask; columns 2..4 its face averages, built
  // on the device as set_immersed_boundary does at the first step
  DBuf cv4;
  const size_t nc = d.ncell;
  ok = cv4.ensure(4 * nc * sizeof(double)) &&
       NSE_CUDA(cudaMemcpyAsync(cv4.p, x->f[NSE_CELLVALUE].p, nc * sizeof(double),
                                cudaMemcpyDeviceToDevice, x->stream));
  if (ok) {
    launch_build_face_masks(d, cv4.as<double>(), x->stream);
    cv.resize(4 * nc);
    ok = NSE_CUDA(cudaMemcpyAsync(cv.data(), cv4.p, 4 * nc * sizeof(double),
                                  cudaMemcpyDeviceToHost, x->stream)) &&
         NSE_CUDA(cudaStreamSynchronize(x->stream));
  }
  cv4.release();
  if (!ok) return status_or(NSE_ERR_CUDA);
  if (!write_output_files(root, d.nx, d.ny, d.nz, u.data(), v.data(), w.data(), p.data(),
                          x->hx.data(), x->hy.data(), x->hz.data(), T.data(), cv.data(),
                          uta.data(), vta.data(), wta.data(), phi.data(), divu.data()))
    return status_or(NSE_ERR_ARG);
  return NSE_OK;
}

int nse_ctx_write_field(nse_ctx* x, const char* path, double tid, const char* grid_path) {
  if (!x || !path) return NSE_ERR_ARG;
  const Dims& d = x->d;
  std::vector<double> u, v, w, p, T, uta, vta, wta, phi;
  bool ok = download_vec(x, NSE_U, u) && download_vec(x, NSE_V, v) &&
            download_vec(x, NSE_W, w) && download_vec(x, NSE_P, p) &&
            download_vec(x, NSE_T, T) && download_vec(x, NSE_U_TA, uta) &&
            download_vec(x, NSE_V_TA, vta) && download_vec(x, NSE_W_TA, wta) &&
            download_lsphi(x, phi);
  if (!ok) return status_or(NSE_ERR_CUDA);
  if (!write_field_file(path, true, tid, d.nx, d.ny, d.nz, u.data(), v.data(), w.data(),
                        p.data(), T.data(), phi.data(), uta.data(), vta.data(), wta.data()))
    return status_or(NSE_ERR_ARG);
  if (grid_path && !write_grid_file(grid_path, d.nx, d.ny, d.nz, x->hx.data(), x->hy.data(),
                                    x->hz.data())) {
    set_error(NSE_ERR_ARG, "cannot write %s", grid_path);
    return NSE_ERR_ARG;
  }
  return NSE_OK;
}

int nse_ctx_read_field(nse_ctx* x, const char* path) {
  if (!x || !path) return NSE_ERR_ARG;
  const Dims& d = x->d;
  const size_t n = d.ntot;
  std::vector<double> u(n), v(n), w(n), p(n), T(n), phi(n), uta(n), vta(n), wta(n);
  if (!read_field_file(path, d.nx, d.ny, d.nz, u.data(), v.data(), w.data(), p.data(),
                       T.data(), phi.data(), uta.data(), vta.data(), wta.data()))
    return status_or(NSE_ERR_ARG);
  const int ids[8] = {NSE_U, NSE_V, NSE_W, NSE_P, NSE_T, NSE_U_TA, NSE_V_TA, NSE_W_TA};
  const double* src[8] = {u.data(), v.data(), w.data(), p.data(), T.data(),
                          uta.data(), vta.data(), wta.data()};
  for (int q = 0; q < 8; ++q) {
    int st = nse_ctx_upload(x, ids[q], src[q]);
    if (st != NSE_OK) return st;
  }
  if (!x->lsphi.ensure(n * sizeof(double)) ||
      !NSE_CUDA(cudaMemcpyAsync(x->lsphi.p, phi.data(), n * sizeof(double),
                                cudaMemcpyHostToDevice, x->stream)) ||
      !NSE_CUDA(cudaStreamSynchronize(x->stream)))
    return status_or(NSE_ERR_CUDA);
  return NSE_OK;
}

int nse_monitor(nse_ctx* x, double out[6]) {
  if (!x || !out) return NSE_ERR_ARG;
  double* m = x->mon.as<double>();
  if (x->mixed)
    launch_monitor_f32(x->d, x->g, F(x, NSE_U), F(x, NSE_V), F(x, NSE_W), F(x, NSE_T),
                       F32(x, NSE_DIVU), m, x->stream);
  else
    launch_monitor(x->d, x->g, F(x, NSE_U), F(x, NSE_V), F(x, NSE_W), F(x, NSE_T),
                   F(x, NSE_DIVU), m, x->stream);
  if (!NSE_CUDA(cudaMemcpyAsync(out, m, 6 * sizeof(double), cudaMemcpyDeviceToHost, x->stream)))
    return status_or(NSE_ERR_CUDA);
  return NSE_CUDA(cudaStreamSynchronize(x->stream)) ? NSE_OK : status_or(NSE_ERR_CUDA);
}

int nse_ctx_profile(nse_ctx* x, int max_steps) {
  if (!x || max_steps < 0) return NSE_ERR_ARG;
  if (!NSE_CUDA(cudaStreamSynchronize(x->stream))) return status_or(NSE_ERR_CUDA);
  for (cudaEvent_t e : x->ev) cudaEventDestroy(e);
  x->ev.assign((size_t)max_steps * (PH_COUNT + 1), nullptr);
  for (auto& e : x->ev)
    if (!NSE_CUDA(cudaEventCreate(&e))) return status_or(NSE_ERR_CUDA);
  x->prof_cap = max_steps;
  x->prof_n = 0;
  return NSE_OK;
}

int nse_ctx_phase_times(nse_ctx* x, double* ms, int nphase, int* nsteps) {
  if (!x || !ms || nphase < PH_COUNT) return NSE_ERR_ARG;
  if (!NSE_CUDA(cudaStreamSynchronize(x->stream))) return status_or(NSE_ERR_CUDA);
  for (int p = 0; p < PH_COUNT; ++p) ms[p] = 0.0;
  for (int st = 0; st < x->prof_n; ++st)
    for (int p = 0; p < PH_COUNT; ++p) {
      float t = 0.f;
      cudaEvent_t a = x->ev[(size_t)st * (PH_COUNT + 1) + p];
      cudaEvent_t b = x->ev[(size_t)st * (PH_COUNT + 1) + p + 1];
      if (!NSE_CUDA(cudaEventElapsedTime(&t, a, b))) return status_or(NSE_ERR_CUDA);
      ms[p] += t;
    }
  if (nsteps) *nsteps = x->prof_n;
  x->prof_n = 0;
  return NSE_OK;
}

int nse_ctx_set_line_shapes(nse_ctx* x, int yz_shape, int x_lines) {
  if (!x || yz_shape < 0 || yz_shape > 3 || x_lines < 1 || x_lines > 4) return NSE_ERR_ARG;
  for (int dir = 1; dir <= 2; ++dir)
    for (int comp = 0; comp < 4; ++comp) x->yzshape[dir][comp] = yz_shape;
  for (int comp = 0; comp < 4; ++comp) x->xnl[comp] = x_lines;
  x->tuned = true;
  return NSE_OK;
}

int nse_ctx_set_shapes(nse_ctx* x, int rhs_shape, int corr_shape) {
  if (!x || rhs_shape < -1 || rhs_shape > 6 || corr_shape < -1 || corr_shape > 15)
    return NSE_ERR_ARG;
  if (rhs_shape >= 0) {
    x->rhs_shape = rhs_shape;
    x->rhs_tuned = true;
  }
  if (corr_shape >= 0) {
    x->corr_shape = corr_shape;
    x->corr_tuned = true;
  }
  return NSE_OK;
}

int nse_ctx_launch_shapes(nse_ctx* x, int* out) {
  if (!x || !out) return NSE_ERR_ARG;
  for (int dir = 1; dir <= 2; ++dir)
    for (int comp = 0; comp < 4; ++comp) out[(dir - 1) * 4 + comp] = x->yzshape[dir][comp];
  for (int comp = 0; comp < 4; ++comp) out[8 + comp] = x->xnl[comp] ? x->xnl[comp] : 2;
  out[12] = x->rhs_shape;
  out[13] = x->corr_shape;
  out[14] = x->mid_chunks;
  return NSE_OK;
}

int nse_sync(nse_ctx* x) {
  if (!x) return NSE_ERR_ARG;
  if (!NSE_CUDA(cudaStreamSynchronize(x->stream))) return status_or(NSE_ERR_CUDA);
  if (spn_wait_error()) {
    set_error(NSE_ERR_CUDA, "nse_sync: the spectral solve's wait for its tile copy gave up");
    return NSE_ERR_CUDA;
  }
  if (line_wait_error()) {
    set_error(NSE_ERR_CUDA, "nse_sync: a line kernel's wait for its tile copy gave up");
    return NSE_ERR_CUDA;
  }
  if (ring_wait_error()) {
    set_error(NSE_ERR_CUDA, "nse_sync: a right-hand-side or correction ring wait gave up");
    return NSE_ERR_CUDA;
  }
  return NSE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- ensemble --
// Independent cases stepped together: each case runs on one of `nstreams`
// streams so small grids overlap on the GPU, and after the first step (the
// Euler start, which also builds the line tables of the mask) the steps are
// replayed from a CUDA graph that holds two steps of every case (two, so the
// FP64 form's temperature buffer swap returns to its starting pair and the
// graph can be replayed as is).
struct nse_ensemble {
  std::vector<nse_ctx*> cases;
  std::vector<cudaStream_t> saved;  // the cases' streams before the ensemble
  std::vector<cudaStream_t> streams;
  cudaStream_t origin = nullptr;
  bool own_origin = true;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // each case's temperature buffer when the graph was captured: the FP64
  // form swaps it with the work buffer every step, so a replay is valid only
  // after an even number of eager steps since the capture
  std::vector<void*> tbuf;
  long long nk = 0;  // kernels in the graph (counted once per replay)
};

namespace nse {

// origin waits for every case stream (eager work before a replay)
static bool ens_join_into_origin(nse_ensemble* e) {
  for (size_t i = 0; i < e->streams.size(); ++i)
    if (!NSE_CUDA(cudaEventRecord(e->join[i], e->streams[i])) ||
        !NSE_CUDA(cudaStreamWaitEvent(e->origin, e->join[i], 0)))
      return false;
  return true;
}
// every case stream waits for origin (eager work after a replay)
static bool ens_fork_from_origin(nse_ensemble* e) {
  if (!NSE_CUDA(cudaEventRecord(e->fork, e->origin))) return false;
  for (cudaStream_t st : e->streams)
    if (!NSE_CUDA(cudaStreamWaitEvent(st, e->fork, 0))) return false;
  return true;
}

static bool ens_eager_step(nse_ensemble* e) {
  for (nse_ctx* x : e->cases) {
    ctx_step(x);
    if (!NSE_CUDA(cudaGetLastError())) return false;
  }
  return true;
}

static bool ens_capture(nse_ensemble* e) {
  std::vector<int> l0;
  for (nse_ctx* x : e->cases) l0.push_back(x->l);
  e->tbuf.clear();
  for (nse_ctx* x : e->cases) e->tbuf.push_back(x->f[NSE_T].p);
  if (!NSE_CUDA(cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeRelaxed))) return false;
  const long long k0 = g_launches.load();
  bool ok = ens_fork_from_origin(e);
  for (int st = 0; ok && st < 2; ++st)
    for (nse_ctx* x : e->cases) ctx_step(x);
  e->nk = g_launches.load() - k0;
  count_launches(-e->nk);  // counted by each replay instead
  ok = ok && ens_join_into_origin(e);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(e->origin, &g);
  for (size_t i = 0; i < e->cases.size(); ++i) e->cases[i]->l = l0[i];  // nothing ran yet
  if (!ok || !NSE_CUDA(ce)) {
    if (g) cudaGraphDestroy(g);
    return false;
  }
  e->graph = g;
  return NSE_CUDA(cudaGraphInstantiate(&e->exec, g, 0));
}

}  // namespace nse

extern "C" {

int nse_ensemble_create(nse_ctx** cases, int n, int nstreams, nse_ensemble** out) {
  nse_clear_error();
  if (!cases || n < 1 || !out) {
    set_error(NSE_ERR_ARG, "nse_ensemble_create: bad arguments");
    return NSE_ERR_ARG;
  }
  *out = nullptr;
  for (int i = 0; i < n; ++i)
    if (!cases[i] || (cases[i]->cfg.flags & NSE_FLAG_CHECK_FINITE)) {
      set_error(NSE_ERR_ARG, "nse_ensemble_create: case %d is null or checks every step", i);
      return NSE_ERR_ARG;
    }
  nse_ensemble* e = new nse_ensemble();
  const int ns = std::max(1, std::min(nstreams, n));
  bool ok = NSE_CUDA(cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking)) &&
            NSE_CUDA(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
  e->streams.assign(ns, nullptr);
  e->join.assign(ns, nullptr);
  for (int i = 0; ok && i < ns; ++i)
    ok = NSE_CUDA(cudaStreamCreateWithFlags(&e->streams[i], cudaStreamNonBlocking)) &&
         NSE_CUDA(cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming));
  for (int i = 0; ok && i < n; ++i) {
    // finish what the case has queued on its own stream first
    ok = NSE_CUDA(cudaStreamSynchronize(cases[i]->stream));
    e->cases.push_back(cases[i]);
    e->saved.push_back(cases[i]->stream);
    cases[i]->stream = e->streams[i % ns];
  }
  if (!ok) {
    nse_ensemble_destroy(e);
    return status_or(NSE_ERR_CUDA);
  }
  *out = e;
  return NSE_OK;
}

int nse_ensemble_step(nse_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return NSE_ERR_ARG;
  bool ok = true;
  while (ok && nsteps > 0) {
    // eager: the first step of a case, a mask being (re)tabulated, profiled
    // steps, a temperature buffer out of the captured parity, or one step left
    bool eager = nsteps < 2;
    for (nse_ctx* x : e->cases)
      eager = eager || x->l <= 1 || x->mask_dirty || x->prof_n < x->prof_cap;
    if (!eager && e->exec)
      for (size_t i = 0; i < e->cases.size(); ++i)
        eager = eager || e->cases[i]->f[NSE_T].p != e->tbuf[i];
    if (eager) {
      ok = ens_eager_step(e);
      --nsteps;
      continue;
    }
    if (!e->exec) ok = ens_capture(e);
    ok = ok && ens_join_into_origin(e);
    for (; ok && nsteps >= 2; nsteps -= 2) {
      ok = NSE_CUDA(cudaGraphLaunch(e->exec, e->origin));
      if (ok) count_launches(e->nk);
      for (nse_ctx* x : e->cases) x->l += 2;
    }
    ok = ok && ens_fork_from_origin(e);
  }
  return ok ? NSE_OK : status_or(NSE_ERR_CUDA);
}

int nse_ensemble_set_stream(nse_ensemble* e, void* stream) {
  if (!e || !stream) return NSE_ERR_ARG;
  if (!NSE_CUDA(cudaStreamSynchronize(e->origin))) return status_or(NSE_ERR_CUDA);
  if (e->own_origin) cudaStreamDestroy(e->origin);
  e->own_origin = false;
  e->origin = (cudaStream_t)stream;
  return NSE_OK;
}

int nse_ensemble_sync(nse_ensemble* e) {
  if (!e) return NSE_ERR_ARG;
  bool ok = NSE_CUDA(cudaStreamSynchronize(e->origin));
  for (cudaStream_t st : e->streams) ok = ok && NSE_CUDA(cudaStreamSynchronize(st));
  return ok ? NSE_OK : status_or(NSE_ERR_CUDA);
}

int nse_ensemble_destroy(nse_ensemble* e) {
  if (!e) return NSE_OK;
  if (e->origin) cudaStreamSynchronize(e->origin);
  for (cudaStream_t st : e->streams)
    if (st) cudaStreamSynchronize(st);
  for (size_t i = 0; i < e->cases.size(); ++i) e->cases[i]->stream = e->saved[i];
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  for (cudaStream_t st : e->streams)
    if (st) cudaStreamDestroy(st);
  if (e->origin && e->own_origin) cudaStreamDestroy(e->origin);
  delete e;
  return NSE_OK;
}

}  // extern "C"
