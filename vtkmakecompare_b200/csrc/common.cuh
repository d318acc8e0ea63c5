// common.cuh -- shared definitions for the libnsegpu.so kernels and host glue.
//
// Device layout = the reference layout, so the C-ABI never re-lays out data:
//   padded field (0:nx+1,0:ny+1,0:nz+1) FP64, x fastest: idx = i + sx*j + sy*k
//   mask c1 (1:nx,1:ny,1:nz) FP64 (column 1 of the reference's cellvalue)
// Kernels of this library are compiled without FMA contraction except the FFT
// file, so every stencil/line-solver expression rounds like the reference's
// Fortran build (left-to-right evaluation, one rounding per operation).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/nsegpu.h"

namespace nse {

// ------------------------------------------------------------ dimensions --
struct Dims {
  int nx, ny, nz;
  long sx, sy;  // strides of j and k in a padded field
  long ntot;    // (nx+2)(ny+2)(nz+2)
  long ncell;   // nx*ny*nz
  __host__ __device__ long P(long i, long j, long k) const { return i + sx * j + sy * k; }
  // mask index (1-based i,j,k), column n = 1
  __host__ __device__ long C(long i, long j, long k) const {
    return (i - 1) + (long)nx * ((j - 1) + (long)ny * (k - 1));
  }
};

inline Dims make_dims(int nx, int ny, int nz) {
  Dims d;
  d.nx = nx; d.ny = ny; d.nz = nz;
  d.sx = nx + 2;
  d.sy = (long)(nx + 2) * (ny + 2);
  d.ntot = d.sy * (nz + 2);
  d.ncell = (long)nx * ny * nz;
  return d;
}

// grid spacing arrays on the device, each n+2 long (index 0..n+1)
struct GridDev {
  const double *dx, *dy, *dz, *dx12, *dy12, *dz12;
};

// reciprocals of the grid spacings (fast form of the resident step)
struct GridRcp {
  const double *rdx, *rdy, *rdz, *rdx12, *rdy12, *rdz12;
};

// physical parameters of one step
struct StepParams {
  double dt, Re, Sc, eta;
  double force, source, tbot, ttop, tsolid;
  double rho_cp, thc;  // uniform material properties (resident path)
  int l;               // reference step counter (1 = Euler start)
};

// ------------------------------------------------------------ host errors --
void set_error(int status, const char* fmt, ...);
bool cuda_ok(cudaError_t e, const char* what);
#define NSE_CUDA(call) ::nse::cuda_ok((call), #call)

// device buffer owned by the library
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool ensure(size_t n);  // grow-only
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// fixed-size per-device work arena for the legacy (host-array) entry points
DBuf& arena(int slot);
cudaStream_t legacy_stream();
bool ensure_device();
// counts every kernel launch issued by the library (nse_launch_count)
void count_launch();

// host <-> device copies of a sub-box of a padded field (entries i0..i1,
// j0..j1, k0..k1 inclusive), used so a legacy call writes back exactly the
// entries the reference routine writes
bool copy_box_d2h(double* host, const double* dev, const Dims& d, int i0, int i1, int j0,
                  int j1, int k0, int k1, cudaStream_t s);
bool copy_box_h2d(double* dev, const double* host, const Dims& d, int i0, int i1, int j0,
                  int j1, int k0, int k1, cudaStream_t s);

// ------------------------------------------ reference output files (host) --
// fortran_io.cu: OUTPUT / OUTFIELD / READFIELD files of nse_dominik.f:2606-2794
bool write_output_files(const std::string& root, int nx, int ny, int nz, const double* u,
                        const double* v, const double* w, const double* p, const double* x,
                        const double* y, const double* z, const double* T,
                        const double* cellvalue, const double* u_ta, const double* v_ta,
                        const double* w_ta, const double* phi, const double* divu);
bool write_grid_file(const std::string& path, int nx, int ny, int nz, const double* x,
                     const double* y, const double* z);
bool write_field_file(const std::string& path, bool with_time, double tid, int nx, int ny,
                      int nz, const double* u, const double* v, const double* w,
                      const double* p, const double* T, const double* phi,
                      const double* u_ta, const double* v_ta, const double* w_ta);
bool read_field_file(const std::string& path, int nx, int ny, int nz, double* u, double* v,
                     double* w, double* p, double* T, double* phi, double* u_ta, double* v_ta,
                     double* w_ta);
bool ensure_dir_public(const std::string& dir);

// --------------------------------------------------------- kernel launchers --
// boundary conditions (nse_dominik.f:611-753); which: bit0 u, bit1 v, bit2 w,
// bit3 p, bit4 T
void launch_set_bc(const Dims& d, double* u, double* v, double* w, double* p, double* T,
                   double tbot, double ttop, int which, cudaStream_t s);

// single routines of the step (tier 2), all on interior cells
void launch_convect(const Dims& d, const GridDev& g, const double* u, const double* v,
                    const double* w, double* u_v, double* v_v, double* w_v, double dt,
                    double force, cudaStream_t s);
void launch_convect_scalar(const Dims& d, const GridDev& g, const double* u,
                           const double* v, const double* w, const double* T,
                           const double* rcp, double* u_vT, double dt, double source,
                           cudaStream_t s);
void launch_conduction(const Dims& d, const GridDev& g, const double* u, const double* v,
                       const double* w, double* u_d, double* v_d, double* w_d, double Re,
                       double dt, cudaStream_t s);
void launch_diffusion_scalar(const Dims& d, const GridDev& g, const double* T,
                             const double* thc, const double* rcp, double* u_dT, double Re,
                             double Sc, double dt, cudaStream_t s);
void launch_build_face_masks(const Dims& d, double* cellvalue4, cudaStream_t s);
void launch_ib_forcing(const Dims& d, const double* cellvalue4, const double* u_ta,
                       const double* v_ta, const double* w_ta, double* u_l, double* v_l,
                       double* w_l, double* T_l, double eta, double dt, cudaStream_t s);
void launch_explicit(const Dims& d, const double* u_v, double* u_pre, const double* u_d,
                     double* u_a, const double* v_v, double* v_pre, const double* v_d,
                     double* v_a, const double* w_v, double* w_pre, const double* w_d,
                     double* w_a, const double* u_l, const double* v_l, const double* w_l,
                     int l, cudaStream_t s);
void launch_explicit_T(const Dims& d, const double* u_vT, const double* u_dT, double* u_T,
                       double* T_pre, const double* T_l, int l, cudaStream_t s);
void launch_penalize(const Dims& d, const double* base, double* a, const double* mask,
                     double eta, double dt, double tsolid, cudaStream_t s);

// fused right-hand side of the resident step: convect + conduction + scalar
// terms + immersed-boundary forcing + AB2 + penalised implicit update;
// writes u_a,v_a,w_a,u_T and the AB2 histories (interior cells)
void launch_rhs_fused(const Dims& d, const GridDev& g, const StepParams& sp,
                      const double* u, const double* v, const double* w, const double* T,
                      const double* u_ta, const double* v_ta, const double* w_ta,
                      double* u_pre, double* v_pre, double* w_pre, double* T_pre,
                      const double* c1, double* u_a, double* v_a, double* w_a,
                      double* u_T, cudaStream_t s);

// same terms in the fast form (reciprocal metrics, FMA, mask-free cells skip
// the immersed-boundary loads); k_rhs_fast.cu
// nonzero (and cleared) when a TMA ring wait of the RHS or correction gave up
// (1) or a launch found its buffers misaligned (2)
int ring_wait_error();
void launch_rhs_fast(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                     const double* u, const double* v, const double* w, const double* T,
                     const double* u_ta, const double* v_ta, const double* w_ta,
                     double* u_pre, double* v_pre, double* w_pre, double* T_pre,
                     const double* c1, double* u_a, double* v_a, double* w_a, double* u_T,
                     cudaStream_t s, int shape = 0);

// ADI line solves; mask is c1 (nx,ny,nz); comp: 0 u (c2), 1 v (c3), 2 w (c4)
struct LineScratch {
  double* a;  // >= ntot doubles
  double* b;  // >= ntot doubles
};
void launch_ysolve_vel(const Dims& d, const GridDev& g, double* f, const double* c1,
                       int comp, double Re, double dt, double eta, const LineScratch& sc,
                       cudaStream_t s);
void launch_zsolve_vel(const Dims& d, const GridDev& g, double* f, const double* c1,
                       int comp, double Re, double dt, double eta, const LineScratch& sc,
                       cudaStream_t s);
void launch_xsolve_vel(const Dims& d, const GridDev& g, double* f, const double* c1,
                       int comp, double Re, double dt, double eta, const LineScratch& sc,
                       cudaStream_t s);
// tier-2 variant: mask given as the cellvalue column of the component;
// dir 0 x, 1 y, 2 z
void launch_vel_line_col(const Dims& d, const GridDev& g, double* f, const double* column,
                         int dir, int comp, double Re, double dt, double eta,
                         const LineScratch& sc, cudaStream_t s);
// temperature solves; rcp/thc padded fields or NULL for uniform values
void launch_ysolve_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0,
                     double Re, double Sc, double dt, double eta, double ft, double fb,
                     const LineScratch& sc, cudaStream_t s);
void launch_zsolve_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0,
                     double Re, double Sc, double dt, double eta, const LineScratch& sc,
                     cudaStream_t s);
void launch_xsolve_T(const Dims& d, const GridDev& g, double* f, const double* c1,
                     const double* rcp, const double* thc, double rcp0, double thc0,
                     double Re, double Sc, double dt, double eta, const LineScratch& sc,
                     cudaStream_t s);
// single-system routines (tier 1/2), one GPU thread each
void launch_single_ul(double* f, double* lsc, int kind, int n, const GridDev& g, double Re,
                      double Sc, double dt, double eta, double ft, double fb, const double* cu,
                      const double* ll, const double* rr, cudaStream_t s);
void launch_single_cyc(double* f, double* gsc, double* zsc, int kind, int n, const GridDev& g,
                       double Re, double Sc, double dt, double eta, double ft, double fb,
                       const double* cu, const double* ll, const double* rr, cudaStream_t s);
void launch_cyclic_general(const double* a, const double* b, const double* c, double alpha,
                           double beta, const double* r, double* x, double* bb, double* gam,
                           double* z, int n, cudaStream_t s);
void launch_tdma(const double* a, const double* b, const double* c, const double* r, double* u,
                 double* gam, int n, cudaStream_t s);
void launch_tridiag(double* A, double* B, int NN, int ncomp, cudaStream_t s);
void launch_trid2(const double* A0, double* Amod, double* B, int M, int N, cudaStream_t s);

// Poisson / projection (mkp.f)
struct PoissonPlan {
  int nx, ny, nz, H, Hp;      // H = nx/2+1 spectral columns, Hp = padded pitch
  double* spec;               // complex [nz][ny][Hp] (interleaved)
  double* scr;                // real [nz][ny][Hp] Thomas scratch
  const double* AC;           // [3][ny] (column-major AC(1:ny,3))
  const double* KXZ;          // [nz+1][H]
  const double* twx;          // twiddles exp(-2 pi i k/nx), k<nx (complex)
  const double* twz;          // twiddles exp(-2 pi i k/nz)
  const float* twx_f;         // the same twiddles rounded to FP32
  const float* twz_f;
  const double* spn_im;       // SPN pivot reciprocals [nz][ny][Hp] (null: none)
  int spn_cp = 0;             // 1: the two-ended SPN stages by cp.async, not TMA tiles
  const double* rAC3 = nullptr;  // 1/AC3 [ny] for SP0B's marching (null: computed inline)
};
bool poisson_plan_tables(int nx, int ny, int nz, const double* dx, const double* dy,
                         const double* dz, const double* dy12, double xl, double zl,
                         double* AC_host, double* KXZ_host, double* twx_host,
                         double* twz_host);
// forward real 2-D FFT per y-plane.  src_mode 0: samples from a padded field
// (P2S, sample (i,k) = FP(i,J,k)); 1: samples = divergence of u*,v*,w* / dt
// at cell (i==0?nx:i, J, k==0?nz:k) (MKP RHS + periodic fill fused)
// src_mode 1 forms the divergence right-hand side; with rg given it multiplies
// by the tabulated reciprocal spacings instead of dividing (fast form)
// j0, nj: window of planes J = j0+1 .. j0+nj (nj = 0: all planes)
void launch_fft_fwd_x(const PoissonPlan& pp, const Dims& d, const double* FP,
                      const double* ut, const double* vt, const double* wt,
                      const GridDev& g, double dt, int src_mode, cudaStream_t s,
                      const GridRcp* rg = nullptr, int j0 = 0, int nj = 0);
void launch_fft_z(const PoissonPlan& pp, bool inverse, cudaStream_t s, int j0 = 0, int nj = 0);
// divergence right-hand side of mkp.f:90-97 (reciprocal spacings) into the
// P2S sample layout of `out`, for the forward x pass in src_mode 0
void launch_div_src(const Dims& d, const GridRcp& rg, const double* ut, const double* vt,
                    const double* wt, double dt, double* out, cudaStream_t s);
void launch_div_src32(const Dims& d, const GridRcp& rg, const float* ut, const float* vt,
                      const float* wt, double dt, double* out, cudaStream_t s);

void launch_spn(const PoissonPlan& pp, bool do_spn, bool do_sp0b, cudaStream_t s);
// SPN pivot tables of the two-ended elimination (0 from spn_split: no
// tables for this plan) and the table-driven SPN + SP0B of the fast form
int spn_split(const PoissonPlan& pp);
void launch_spn_tables(const PoissonPlan& pp, double* im, cudaStream_t s);
void launch_spn_fast(const PoissonPlan& pp, cudaStream_t s);
int poisson_mid_groups(const PoissonPlan& pp);
void launch_poisson_mid(const PoissonPlan& pp, int nchunk, cudaStream_t s);
bool launch_spn_transposed(const PoissonPlan& pp, const double* rdy, const double* dy,
                           cudaStream_t s);

void launch_spn_fast_f32(const PoissonPlan& pp, cudaStream_t s);
void launch_spn_view(int H, int ny, int nz, double* base, long sj, long sk, double* sc,
                     long scj, long sck, const double* AC, const double* KXZ, bool do_spn,
                     bool do_sp0b, cudaStream_t s);
// inverse x transform into padded FP for J=1..NY with the S2P wrap fill
void launch_fft_inv_x(const PoissonPlan& pp, const Dims& d, double* FP, cudaStream_t s,
                      int j0 = 0, int nj = 0);
void launch_phibc(const Dims& d, double* PHI, cudaStream_t s);
// k_poisson2d.cu: the three-pass solve for NX = NZ = 256 (FP64).  P2S of
// every plane (one cluster of 8 CTAs per plane), SPN + SP0B partitioned over
// 16 lanes per system (ny = 16 m, 3 <= m <= 16), S2P + PHIBC.
bool poisson3_ok(const PoissonPlan& pp);
bool spn_part_ok(const PoissonPlan& pp);
void launch_p2s256(const PoissonPlan& pp, const Dims& d, const double* FP, cudaStream_t s);
void launch_spn_part(const PoissonPlan& pp, cudaStream_t s);
void launch_s2p256_phibc(const PoissonPlan& pp, const Dims& d, double* FP, cudaStream_t s);
// SPN + SP0B through TMA tiles (ny = 16 m); false when it does not apply
bool launch_spn_tma(const PoissonPlan& pp, cudaStream_t s);
int spn_wait_error();
// spectrum <-> reference PHIT layout (0:nx/2,0:ny+1,0:nz+1)
void launch_spec_to_phit(const PoissonPlan& pp, double* phit, cudaStream_t s);
void launch_phit_to_spec(const PoissonPlan& pp, const double* phit, cudaStream_t s);
// gradient + correction of mkp.f:141-217
void launch_correct(const Dims& d, const GridDev& g, const double* PHI, const double* ut,
                    const double* vt, const double* wt, double* p, double* u, double* v,
                    double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                    double* v_ep2, double* w_ep2, double* divu, double dt, cudaStream_t s);

void launch_correct_fast(const Dims& d, const GridRcp& rg, const double* PHI, const double* ut,
                         const double* vt, const double* wt, double* p, double* u, double* v,
                         double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                         double* v_ep2, double* w_ep2, double* divu, double dt, cudaStream_t s);

void launch_correct_pipe(const Dims& d, const GridRcp& rg, const double* PHI, const double* ut,
                         const double* vt, const double* wt, double* p, double* u, double* v,
                         double* w, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
                         double* v_ep2, double* w_ep2, double* divu, double dt, cudaStream_t s,
                         int shape = 0);

// level set (set_levelset.f)
void launch_levelset_iter(const Dims& d, const GridDev& g, const double* phi0,
                          const double* phi, double* phi_new, double dtau, cudaStream_t s);
void launch_levelset_bc(const Dims& d, double* phi, cudaStream_t s);
void launch_levelset_mask(const Dims& d, const GridDev& g, const double* phi,
                          double* cellvalue1, double width, cudaStream_t s);

// reductions for nse_monitor
void launch_monitor(const Dims& d, const GridDev& g, const double* u, const double* v,
                    const double* w, const double* T, const double* divu, double* out6,
                    cudaStream_t s);

// resident context internals shared with the adjoint driver (runtime.cu)
struct CtxInfo {
  Dims d;
  GridDev g;
  GridRcp rg;
  const nse_config* cfg;
  cudaStream_t s;
  const PoissonPlan* pp;
  bool mixed;
};
bool ctx_info(nse_ctx* x, CtxInfo& out);
double* ctx_field(nse_ctx* x, int id);
int ctx_get_l(nse_ctx* x);
void ctx_set_l(nse_ctx* x, int l);
// one step of the context; with rec given, the line-solve passes record their
// inputs and outputs (16 padded fields, see nse_ctx::rec)
void ctx_step_rec(nse_ctx* x, double* const* rec);
// the line solve of (dir, comp) of the step on the field f (ft = fb = 0)
void ctx_line_solve(nse_ctx* x, int dir, int comp, double* f, cudaStream_t s);

}  // namespace nse
