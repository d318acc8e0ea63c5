// adjoint.cu -- host driver of the discrete adjoint of the resident time
// step (nse_adjoint_*): gradient of a time-averaged wall heat flux with
// respect to the penalisation mask c1 and to the initial state.
//
// Forward: nsteps steps of the context (FP64 form), the state (u, v, w, T,
// u_ta, v_ta, w_ta and the AB2 histories) copied to device memory every
// `checkpoint_every` steps.  Reverse: per checkpoint segment, last first,
// the segment is replayed from its checkpoint with every step recording the
// state it starts from and the inputs and outputs of its line-solve passes;
// then its steps are reversed one by one with the transposed kernels of
// k_adjoint.cu; the transposed line solves are the step's own line solves
// between diagonal scalings.  Device memory: (ceil(nsteps/ckpt) * 11 +
// ckpt * 23 + 36) padded fields.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "k_adjoint.cuh"

using namespace nse;

namespace {

// state fields, in the order of the adjoint state
const int kState[11] = {NSE_U,     NSE_V,     NSE_W,     NSE_T,     NSE_U_TA, NSE_V_TA,
                        NSE_W_TA,  NSE_U_PRE, NSE_V_PRE, NSE_W_PRE, NSE_T_PRE};
enum { S_U = 0, S_V, S_W, S_T, S_UTA, S_VTA, S_WTA, S_UP, S_VP, S_WP, S_TP, NS };
const int kSeg = 7;   // u, v, w, T, u_ta, v_ta, w_ta at the start of a recorded step
const int kRec = 16;  // line-pass inputs and outputs of a recorded step
// work fields
enum { W_B = 0, W_O = 4, W_XS = 8, W_RB = 9, W_ST = 10, NW = 14 };

int state_index(int field) {
  for (int q = 0; q < NS; ++q)
    if (kState[q] == field) return q;
  return -1;
}

}  // namespace

struct nse_adjoint {
  nse_ctx* x = nullptr;
  nse_adjoint_config cfg{};
  CtxInfo ci{};
  size_t F = 0;  // doubles per padded field
  int nck = 0;
  DBuf ck, seg, rec, fin, bar, work, cbar, wts, J;
  std::vector<int> ck_l;
  int fin_l = 0;
  bool has_w[NS] = {};
  double* barp[NS] = {};
  double* outp[4] = {};
  // side streams of components 1..3 and the fork/join events
  cudaStream_t side[3] = {};
  cudaEvent_t fork = nullptr, join[3] = {};
  double* field(const DBuf& b, size_t idx) const { return b.as<double>() + idx * F; }
};

namespace {

bool copy_fields(nse_adjoint* a, double* dst_base, const int* ids, int n, bool to_ctx) {
  const size_t fb = a->F * sizeof(double);
  for (int q = 0; q < n; ++q) {
    double* cf = ctx_field(a->x, ids[q]);
    double* bf = dst_base + (size_t)q * a->F;
    if (!NSE_CUDA(cudaMemcpyAsync(to_ctx ? cf : bf, to_ctx ? bf : cf, fb,
                                  cudaMemcpyDeviceToDevice, a->ci.s)))
      return false;
  }
  return true;
}

// forward run: checkpoints, objective accumulated on the device, final state kept
bool run_forward(nse_adjoint* a) {
  const CtxInfo& ci = a->ci;
  const nse_config& c = *ci.cfg;
  const AdjGrid g = adj_grid(ci.g, &ci.rg);
  const int N = a->cfg.nsteps, K = a->cfg.checkpoint_every, n0 = a->cfg.avg_from;
  const double w = 1.0 / (double)(N - n0 + 1);
  double* J = a->J.as<double>();
  if (!NSE_CUDA(cudaMemsetAsync(J, 0, 2 * sizeof(double), ci.s))) return false;
  for (int n = 1; n <= N; ++n) {
    if ((n - 1) % K == 0) {
      const int m = (n - 1) / K;
      a->ck_l[m] = ctx_get_l(a->x);
      if (!copy_fields(a, a->field(a->ck, (size_t)m * NS), kState, NS, false)) return false;
    }
    ctx_step_rec(a->x, nullptr);
    if (n >= n0)
      launch_wall_flux(ci.d, g, ctx_field(a->x, NSE_T), c.t_bot, c.thc, c.xl, c.zl, w, J, ci.s);
  }
  for (int q = 0; q < NS; ++q)
    if (a->has_w[q])
      launch_weighted_sum(ci.d, a->field(a->wts, q), ctx_field(a->x, kState[q]), J, ci.s);
  a->fin_l = ctx_get_l(a->x);
  if (!copy_fields(a, a->fin.as<double>(), kState, NS, false)) return false;
  return NSE_CUDA(cudaGetLastError());
}

// one step reversed: a->barp holds the adjoint of the state after the step
// on entry and of the state before it on return
void adjoint_step(nse_adjoint* a, double* sg, double* const* rc, int l) {
  const CtxInfo& ci = a->ci;
  const nse_config& c = *ci.cfg;
  const Dims& D = ci.d;
  const AdjGrid g = adj_grid(ci.g, &ci.rg);
  cudaStream_t s = ci.s;
  double** bar = a->barp;
  const double* c1 = ctx_field(a->x, NSE_CELLVALUE);
  double* cb[4];
  for (int q = 0; q < 4; ++q) cb[q] = a->cbar.as<double>() + (size_t)q * D.ncell;
  double* wk[NW];
  for (int q = 0; q < NW; ++q) wk[q] = a->field(a->work, q);
  auto SG = [&](int q) { return sg + (size_t)q * a->F; };
  // MKP (mkp.f:88-217) transposed
  double* ub[3] = {bar[S_U], bar[S_V], bar[S_W]};
  const double* ubc[3] = {bar[S_U], bar[S_V], bar[S_W]};
  const double* tab[3] = {bar[S_UTA], bar[S_VTA], bar[S_WTA]};
  launch_adj_phibar(D, g, ubc, tab, c.dt, wk[W_XS], s);
  launch_fft_fwd_x(*ci.pp, D, wk[W_XS], nullptr, nullptr, nullptr, ci.g, 1.0, 0, s);
  launch_fft_z(*ci.pp, false, s);
  if (!launch_spn_transposed(*ci.pp, ci.rg.rdy, ci.g.dy, s)) launch_adj_spn(*ci.pp, s);
  launch_fft_z(*ci.pp, true, s);
  launch_fft_inv_x(*ci.pp, D, wk[W_RB], s);
  launch_adj_div(D, g, ub, wk[W_RB], c.dt, s);
  // line passes in reverse (velocity y, z, x; temperature y, x, z forward);
  // the four components are independent: component 0 on the context's
  // stream, 1..3 on side streams forked from it and joined back
  NSE_CUDA(cudaEventRecord(a->fork, s));
  for (int q = 0; q < 3; ++q) NSE_CUDA(cudaStreamWaitEvent(a->side[q], a->fork, 0));
  for (int comp = 0; comp < 4; ++comp) {
    cudaStream_t cs = comp == 0 ? s : a->side[comp - 1];
    const int vdirs[3] = {1, 2, 0}, tdirs[3] = {1, 0, 2};
    const int* dirs = comp == 3 ? tdirs : vdirs;
    double* cbar = comp == 3 ? cb[0] : cb[comp + 1];
    // scale for the last pass, then each solve's output scaling also
    // prepares the input of the pass before it (one kernel between solves)
    launch_adj_line_scale(D, g, dirs[2], comp, false, bar[comp], nullptr, nullptr, c1, nullptr,
                          c.dt, c.eta, cs);
    for (int p = 2; p >= 0; --p) {
      ctx_line_solve(a->x, dirs[p], comp, bar[comp], cs);
      launch_adj_line_scale(D, g, dirs[p], comp, true, bar[comp], rc[4 * comp + p],
                            rc[4 * comp + p + 1], c1, cbar, c.dt, c.eta, cs,
                            p > 0 ? dirs[p - 1] : -1);
    }
    if (comp > 0) NSE_CUDA(cudaEventRecord(a->join[comp - 1], cs));
  }
  for (int q = 0; q < 3; ++q) NSE_CUDA(cudaStreamWaitEvent(s, a->join[q], 0));
  // penalised updates, AB2, immersed-boundary forcing
  double* A[4] = {bar[S_U], bar[S_V], bar[S_W], bar[S_T]};
  double* B[4] = {wk[W_B], wk[W_B + 1], wk[W_B + 2], wk[W_B + 3]};
  double* pre[4] = {bar[S_UP], bar[S_VP], bar[S_WP], bar[S_TP]};
  double* bta[3] = {bar[S_UTA], bar[S_VTA], bar[S_WTA]};
  const double* ta[3] = {SG(4), SG(5), SG(6)};
  const double* rin[4] = {rc[0], rc[4], rc[8], rc[12]};
  launch_adj_point(D, A, B, pre, bta, ta, rin, c1, cb, c.eta, c.dt, c.t_solid, l, s);
  // explicit terms at the start state (SET_BC applied to a copy)
  const size_t fb = a->F * sizeof(double);
  for (int q = 0; q < 4; ++q)
    NSE_CUDA(cudaMemcpyAsync(wk[W_ST + q], SG(q), fb, cudaMemcpyDeviceToDevice, s));
  launch_set_bc(D, wk[W_ST], wk[W_ST + 1], wk[W_ST + 2], nullptr, wk[W_ST + 3], c.t_bot,
                c.t_top, 1 | 2 | 4 | 16, s);
  const double* vel[3] = {wk[W_ST], wk[W_ST + 1], wk[W_ST + 2]};
  NSE_CUDA(cudaEventRecord(a->fork, s));
  for (int q = 0; q < 3; ++q) NSE_CUDA(cudaStreamWaitEvent(a->side[q], a->fork, 0));
  launch_adj_explicit(D, g, vel, wk[W_ST + 3], A, B, c.dt, c.Re, c.Sc, c.rho_cp, c.thc,
                      a->outp, s, a->side);
  for (int q = 0; q < 3; ++q) {
    NSE_CUDA(cudaEventRecord(a->join[q], a->side[q]));
    NSE_CUDA(cudaStreamWaitEvent(s, a->join[q], 0));
  }
  for (int q = 0; q < 4; ++q) std::swap(bar[q], a->outp[q]);
}

}  // namespace

extern "C" {

int nse_adjoint_create(nse_ctx* x, const nse_adjoint_config* cfg, nse_adjoint** out) {
  nse_clear_error();
  if (!x || !cfg || !out) {
    set_error(NSE_ERR_ARG, "nse_adjoint_create: null argument");
    return NSE_ERR_ARG;
  }
  *out = nullptr;
  CtxInfo ci;
  ctx_info(x, ci);
  if (ci.mixed) {
    set_error(NSE_ERR_ARG, "nse_adjoint_create: the adjoint differentiates the FP64 step; "
                           "the context is NSE_MIXED");
    return NSE_ERR_ARG;
  }
  const nse_adjoint_config& c = *cfg;
  if (c.nsteps < 1 || c.checkpoint_every < 1 || c.avg_from < 1 || c.avg_from > c.nsteps) {
    set_error(NSE_ERR_ARG, "nse_adjoint_create: need nsteps >= 1, checkpoint_every >= 1, "
                           "1 <= avg_from <= nsteps (got %d %d %d)",
              c.nsteps, c.checkpoint_every, c.avg_from);
    return NSE_ERR_ARG;
  }
  nse_adjoint* a = new nse_adjoint();
  a->x = x;
  a->cfg = c;
  a->cfg.checkpoint_every = std::min(c.checkpoint_every, c.nsteps);
  a->ci = ci;
  a->F = (size_t)ci.d.ntot;
  a->nck = (c.nsteps + a->cfg.checkpoint_every - 1) / a->cfg.checkpoint_every;
  a->ck_l.assign(a->nck, 0);
  const size_t fb = a->F * sizeof(double);
  const size_t K = a->cfg.checkpoint_every;
  bool ok = a->ck.ensure((size_t)a->nck * NS * fb) && a->seg.ensure(K * kSeg * fb) &&
            a->rec.ensure(K * kRec * fb) && a->fin.ensure(NS * fb) && a->bar.ensure(NS * fb) &&
            a->work.ensure(NW * fb) && a->cbar.ensure(4 * ci.d.ncell * sizeof(double)) &&
            a->J.ensure(2 * sizeof(double));
  ok = ok && NSE_CUDA(cudaMemset(a->work.p, 0, NW * fb));
  for (int q = 0; ok && q < 3; ++q)
    ok = NSE_CUDA(cudaStreamCreateWithFlags(&a->side[q], cudaStreamNonBlocking)) &&
         NSE_CUDA(cudaEventCreateWithFlags(&a->join[q], cudaEventDisableTiming));
  ok = ok && NSE_CUDA(cudaEventCreateWithFlags(&a->fork, cudaEventDisableTiming));
  if (!ok) {
    nse_adjoint_destroy(a);
    if (nse_last_status() == NSE_OK)
      set_error(NSE_ERR_NOMEM, "nse_adjoint_create: out of device memory");
    return nse_last_status();
  }
  *out = a;
  return NSE_OK;
}

int nse_adjoint_destroy(nse_adjoint* a) {
  if (!a) return NSE_OK;
  cudaStreamSynchronize(a->ci.s);
  for (int q = 0; q < 3; ++q) {
    if (a->side[q]) cudaStreamSynchronize(a->side[q]);
    if (a->side[q]) cudaStreamDestroy(a->side[q]);
    if (a->join[q]) cudaEventDestroy(a->join[q]);
  }
  if (a->fork) cudaEventDestroy(a->fork);
  for (DBuf* b : {&a->ck, &a->seg, &a->rec, &a->fin, &a->bar, &a->work, &a->cbar, &a->wts, &a->J})
    b->release();
  delete a;
  return NSE_OK;
}

int nse_adjoint_set_weight(nse_adjoint* a, int field, const double* host) {
  if (!a) return NSE_ERR_ARG;
  const int q = state_index(field);
  if (q < 0) {
    set_error(NSE_ERR_ARG, "nse_adjoint_set_weight: field %d is not a state field", field);
    return NSE_ERR_ARG;
  }
  if (!host) {
    a->has_w[q] = false;
    return NSE_OK;
  }
  const size_t fb = a->F * sizeof(double);
  if (!a->wts.ensure(NS * fb)) return nse_last_status();
  if (!NSE_CUDA(cudaMemcpy(a->field(a->wts, q), host, fb, cudaMemcpyHostToDevice)))
    return NSE_ERR_CUDA;
  a->has_w[q] = true;
  return NSE_OK;
}

int nse_adjoint_objective(nse_adjoint* a, double* J) {
  if (!a) return NSE_ERR_ARG;
  ctx_info(a->x, a->ci);  // the context's stream may have changed
  if (!run_forward(a)) return nse_last_status() != NSE_OK ? nse_last_status() : NSE_ERR_CUDA;
  double h[2];
  if (!NSE_CUDA(cudaMemcpyAsync(h, a->J.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, a->ci.s)) ||
      !NSE_CUDA(cudaStreamSynchronize(a->ci.s)))
    return NSE_ERR_CUDA;
  if (J) *J = h[0];
  return NSE_OK;
}

int nse_adjoint_gradient(nse_adjoint* a, double* J, double* grad_c1) {
  if (!a) return NSE_ERR_ARG;
  const int st = nse_adjoint_objective(a, J);
  if (st != NSE_OK) return st;
  const CtxInfo& ci = a->ci;
  const nse_config& c = *ci.cfg;
  const Dims& D = ci.d;
  const AdjGrid g = adj_grid(ci.g, &ci.rg);
  cudaStream_t s = ci.s;
  const size_t fb = a->F * sizeof(double);
  const int N = a->cfg.nsteps, K = a->cfg.checkpoint_every, n0 = a->cfg.avg_from;
  const double w = 1.0 / (double)(N - n0 + 1);
  for (int q = 0; q < NS; ++q) a->barp[q] = a->field(a->bar, q);
  for (int q = 0; q < 4; ++q) a->outp[q] = a->field(a->work, W_O + q);
  if (!NSE_CUDA(cudaMemsetAsync(a->bar.p, 0, NS * fb, s)) ||
      !NSE_CUDA(cudaMemsetAsync(a->cbar.p, 0, 4 * D.ncell * sizeof(double), s)))
    return NSE_ERR_CUDA;
  for (int q = 0; q < 4; ++q)
    if (!NSE_CUDA(cudaMemsetAsync(a->outp[q], 0, fb, s))) return NSE_ERR_CUDA;
  for (int q = 0; q < NS; ++q)
    if (a->has_w[q]) launch_add_weights(D, a->field(a->wts, q), a->barp[q], s);
  std::vector<double*> recp((size_t)K * kRec);
  for (size_t q = 0; q < recp.size(); ++q) recp[q] = a->field(a->rec, q);
  const int segIds[kSeg] = {NSE_U, NSE_V, NSE_W, NSE_T, NSE_U_TA, NSE_V_TA, NSE_W_TA};
  for (int m = a->nck - 1; m >= 0; --m) {
    const int first = m * K + 1, last = std::min(N, first + K - 1);
    if (!copy_fields(a, a->field(a->ck, (size_t)m * NS), kState, NS, true)) return NSE_ERR_CUDA;
    ctx_set_l(a->x, a->ck_l[m]);
    for (int n = first; n <= last; ++n) {
      const int r = n - first;
      if (!copy_fields(a, a->field(a->seg, (size_t)r * kSeg), segIds, kSeg, false))
        return NSE_ERR_CUDA;
      ctx_step_rec(a->x, recp.data() + (size_t)r * kRec);
    }
    for (int n = last; n >= first; --n) {
      const int r = n - first;
      if (n >= n0) launch_adj_wall_flux(D, g, a->barp[S_T], c.thc, c.xl, c.zl, w, s);
      adjoint_step(a, a->field(a->seg, (size_t)r * kSeg), recp.data() + (size_t)r * kRec,
                   a->ck_l[m] + r);
    }
    if (!NSE_CUDA(cudaGetLastError())) return NSE_ERR_CUDA;
  }
  double* cb = a->cbar.as<double>();
  launch_adj_face_fold(D, cb, cb + D.ncell, cb + 2 * D.ncell, cb + 3 * D.ncell, s);
  // leave the context at the end of the forward run
  if (!copy_fields(a, a->fin.as<double>(), kState, NS, true)) return NSE_ERR_CUDA;
  ctx_set_l(a->x, a->fin_l);
  if (grad_c1 &&
      !NSE_CUDA(cudaMemcpyAsync(grad_c1, cb, D.ncell * sizeof(double), cudaMemcpyDeviceToHost, s)))
    return NSE_ERR_CUDA;
  if (!NSE_CUDA(cudaStreamSynchronize(s))) return NSE_ERR_CUDA;
  return NSE_OK;
}

int nse_adjoint_download(nse_adjoint* a, int field, double* host) {
  if (!a || !host) return NSE_ERR_ARG;
  const int q = state_index(field);
  if (q < 0 || !a->barp[q]) {
    set_error(NSE_ERR_ARG, "nse_adjoint_download: field %d has no adjoint (run "
                           "nse_adjoint_gradient first)", field);
    return NSE_ERR_ARG;
  }
  if (!NSE_CUDA(cudaMemcpyAsync(host, a->barp[q], a->F * sizeof(double), cudaMemcpyDeviceToHost,
                                a->ci.s)) ||
      !NSE_CUDA(cudaStreamSynchronize(a->ci.s)))
    return NSE_ERR_CUDA;
  return NSE_OK;
}

}  // extern "C"
