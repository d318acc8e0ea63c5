// k_adjoint.cuh -- launchers of the transposed kernels (k_adjoint.cu) used by
// the adjoint driver (adjoint.cu) and the adjoint.f drop-ins.
#pragma once
#include "common.cuh"

namespace nse {

// grid spacings by axis: d[0..2] = dx, dy, dz; d12[0..2] = dx12, dy12, dz12;
// r, r12 their reciprocals (the transposed kernels multiply by them; the
// adjoint.f drop-ins divide, as the reference does, and leave them null)
struct AdjGrid {
  const double* d[3];
  const double* d12[3];
  const double* r[3];
  const double* r12[3];
};
inline AdjGrid adj_grid(const GridDev& g, const GridRcp* rg = nullptr) {
  AdjGrid a;
  a.d[0] = g.dx; a.d[1] = g.dy; a.d[2] = g.dz;
  a.d12[0] = g.dx12; a.d12[1] = g.dy12; a.d12[2] = g.dz12;
  a.r[0] = rg ? rg->rdx : nullptr; a.r[1] = rg ? rg->rdy : nullptr;
  a.r[2] = rg ? rg->rdz : nullptr;
  a.r12[0] = rg ? rg->rdx12 : nullptr; a.r12[1] = rg ? rg->rdy12 : nullptr;
  a.r12[2] = rg ? rg->rdz12 : nullptr;
  return a;
}

// adjoint of u, v, w, T at the start of a step from the adjoints of the
// explicit terms (A: of u_d / u_dT, B: of u_v / u_vT); vel, T with SET_BC.
// Field 0 runs on s, fields 1..3 on side[0..2] when side is given (the
// caller orders them)
void launch_adj_explicit(const Dims& D, const AdjGrid& g, const double* const vel[3],
                         const double* T, double* const A[4], double* const B[4], double dt,
                         double Re, double Sc, double R, double L, double* const out[4],
                         cudaStream_t s, const cudaStream_t* side = nullptr);
// penalised updates, AB2 and immersed-boundary forcing transposed
void launch_adj_point(const Dims& D, double* const A[4], double* const B[4],
                      double* const bar_pre[4], double* const bar_ta[3],
                      const double* const ta[3], const double* const rin[4], const double* c1,
                      double* const cbar[4], double eta, double dt, double tsolid, int l,
                      cudaStream_t s);
// diagonal scalings around the step's own line solve that make it the
// transposed solve (A^-T = D A^-1 D^-1, D = diag(alpha w)); out = false
// before the solve, true after (with the mask gradient of the pass)
void launch_adj_line_scale(const Dims& D, const AdjGrid& g, int dir, int comp, bool out,
                           double* xb, const double* rin, const double* xout, const double* c1,
                           double* cbar, double dt, double eta, cudaStream_t s, int next = -1);
// MKP transposed: phi_bar at the P2S samples, transposed SPN/SP0B on the
// spectrum, divergence transposed
void launch_adj_phibar(const Dims& D, const AdjGrid& g, const double* const ub[3],
                       const double* const tab[3], double dt, double* xs, cudaStream_t s);
void launch_adj_spn(const PoissonPlan& pp, cudaStream_t s);
void launch_adj_div(const Dims& D, const AdjGrid& g, double* const ub[3], const double* rb,
                    double dt, cudaStream_t s);
// objective: area-weighted wall heat flux at the y = y0 wall and its adjoint
void launch_wall_flux(const Dims& D, const AdjGrid& g, const double* T, double tb, double thc,
                      double xl, double zl, double w, double* J, cudaStream_t s);
void launch_adj_wall_flux(const Dims& D, const AdjGrid& g, double* Tb, double thc, double xl,
                          double zl, double w, cudaStream_t s);
void launch_weighted_sum(const Dims& D, const double* W, const double* f, double* J,
                         cudaStream_t s);
void launch_add_weights(const Dims& D, const double* W, double* fb, cudaStream_t s);
void launch_adj_face_fold(const Dims& D, double* c1b, const double* c2b, const double* c3b,
                          const double* c4b, cudaStream_t s);
// adjoint.f routines (drop-ins)
void launch_set_adj_convect(const Dims& D, const AdjGrid& g, const double* u, const double* v,
                            const double* w, const double* uf, const double* vf,
                            const double* wf, double* u_v, double* v_v, double* w_v, double dt,
                            cudaStream_t s);
void launch_set_adj_cscalar(const Dims& D, const AdjGrid& g, const double* T, const double* R,
                            const double* uf, const double* vf, const double* wf,
                            double* u_vT, double dt, cudaStream_t s);
void launch_set_adj_ns_scalar(const Dims& D, const AdjGrid& g, const double* T,
                              const double* Tf, double* u_s, double* v_s, double* w_s,
                              double dt, cudaStream_t s);

}  // namespace nse
