// k_rhs_fast.cu -- fused right-hand side of the resident step, fast form.
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
// A CTA covers 32 x 8 cells of an (x,y) tile and marches over KCHUNK planes
// in z so the k-1, k, k+1 planes are re-read from L1.
#include "common.cuh"

namespace nse {

#define LD(p, i) __ldg((p) + (i))

constexpr int KCHUNK = 8;

__global__ void __launch_bounds__(256, 2) k_rhs_fast(
    Dims d, GridDev g, GridRcp rg, StepParams sp, const double* __restrict__ U,
    const double* __restrict__ V, const double* __restrict__ W, const double* __restrict__ T,
    const double* __restrict__ U_TA, const double* __restrict__ V_TA,
    const double* __restrict__ W_TA, double* __restrict__ U_PRE, double* __restrict__ V_PRE,
    double* __restrict__ W_PRE, double* __restrict__ T_PRE, const double* __restrict__ C1,
    double* __restrict__ U_A, double* __restrict__ V_A, double* __restrict__ W_A,
    double* __restrict__ U_T) {
  const int I = 1 + blockIdx.x * 32 + threadIdx.x;
  const int J = 1 + blockIdx.y * 8 + threadIdx.y;
  if (I > d.nx || J > d.ny) return;
  const int k0 = 1 + blockIdx.z * KCHUNK;
  const int k1 = min(d.nz, k0 + KCHUNK - 1);
  const double DT = sp.dt;
  const double a1 = (sp.l == 1) ? 1.0 : 1.5, a2 = (sp.l == 1) ? 0.0 : -0.5;
  const double kd = DT / sp.Re * 0.5;
  const double r0 = sp.rho_cp, rr0 = 1.0 / sp.rho_cp, l0 = sp.thc;
  const double kT = 0.5 / sp.Re / sp.Sc / sp.rho_cp * DT;
  // x and y metrics of this column
  const double dx = LD(g.dx, I), dxp = LD(g.dx, I + 1), dxm = LD(g.dx, I - 1);
  const double rx = LD(rg.rdx, I), rxp = LD(rg.rdx, I + 1);
  const double rx12 = LD(rg.rdx12, I), rx12m = LD(rg.rdx12, I - 1);
  const double dy = LD(g.dy, J), dyp = LD(g.dy, J + 1), dym = LD(g.dy, J - 1);
  const double ry = LD(rg.rdy, J), ryp = LD(rg.rdy, J + 1);
  const double ry12 = LD(rg.rdy12, J), ry12m = LD(rg.rdy12, J - 1);
  const long sx = d.sx, sy = d.sy;
  const long nxny = (long)d.nx * d.ny;
  for (int K = k0; K <= k1; ++K) {
    const long c = d.P(I, J, K);
    const double dz = LD(g.dz, K), dzp = LD(g.dz, K + 1), dzm = LD(g.dz, K - 1);
    const double rz = LD(rg.rdz, K), rzp = LD(rg.rdz, K + 1);
    const double rz12 = LD(rg.rdz12, K), rz12m = LD(rg.rdz12, K - 1);
    // neighbourhood
    const double uc = LD(U, c), uxp = LD(U, c + 1), uxm = LD(U, c - 1), uyp = LD(U, c + sx),
                 uym = LD(U, c - sx), uzp = LD(U, c + sy), uzm = LD(U, c - sy),
                 uxmyp = LD(U, c - 1 + sx), uxmzp = LD(U, c - 1 + sy);
    const double vc = LD(V, c), vxp = LD(V, c + 1), vxm = LD(V, c - 1), vyp = LD(V, c + sx),
                 vym = LD(V, c - sx), vzp = LD(V, c + sy), vzm = LD(V, c - sy),
                 vxpym = LD(V, c + 1 - sx), vymzp = LD(V, c - sx + sy);
    const double wc = LD(W, c), wxp = LD(W, c + 1), wxm = LD(W, c - 1), wyp = LD(W, c + sx),
                 wym = LD(W, c - sx), wzp = LD(W, c + sy), wzm = LD(W, c - sy),
                 wxpzm = LD(W, c + 1 - sy), wypzm = LD(W, c + sx - sy);
    const double tc = LD(T, c), txp = LD(T, c + 1), txm = LD(T, c - 1), typ = LD(T, c + sx),
                 tym = LD(T, c - sx), tzp = LD(T, c + sy), tzm = LD(T, c - sy);
    // masks (set_immersed_boundary :1037-1080)
    const long m = d.C(I, J, K);
    const double cc1 = LD(C1, m);
    const double c2 = (I < d.nx) ? (cc1 + LD(C1, m + 1)) * 0.50 : cc1;
    const double c3 = (J < d.ny) ? (cc1 + LD(C1, m + d.nx)) * 0.50 : cc1;
    const double c4 = (K < d.nz) ? (cc1 + LD(C1, m + nxny)) * 0.50 : cc1;
    const bool solid = (c2 != 0.0) || (c3 != 0.0) || (c4 != 0.0) || (cc1 != 0.0);
    // u
    {
      double s1 = uc + uxp, s2 = uc + uxm;
      double U1 = (s1 * s1 - s2 * s2) * rx12;
      double U2 = ((vxp * dxp + vc * dx) * (uyp + uc) - (vxpym * dxp + vym * dx) * (uc + uym)) *
                  rx12 * ry;
      double U3 = ((wxp * dxp + wc * dx) * (uzp + uc) - (wxpzm * dxp + wzm * dx) * (uc + uzm)) *
                  rx12 * rz;
      double uv = 0.25 * (-U1 - U2 - U3) * DT + sp.force * DT;
      double L = ((uxp - uc) * rxp - (uc - uxm) * rx) * rx12 +
                 ((uyp - uc) * ry12 - (uc - uym) * ry12m) * ry +
                 ((uzp - uc) * rz12 - (uc - uzm) * rz12m) * rz;
      double ua = a1 * uv + a2 * U_PRE[c] + kd * L;
      U_PRE[c] = uv;
      if (solid && c2 != 0.0) {
        ua += sp.eta * c2 * LD(U_TA, c) * DT;
        U_A[c] = (uc + ua) / (1.0 + sp.eta * c2 * DT);
      } else {
        U_A[c] = uc + ua;
      }
    }
    // v
    {
      double V1 = ((uyp * dyp + uc * dy) * (vxp + vc) - (uxmyp * dyp + uxm * dy) * (vc + vxm)) *
                  ry12 * rx;
      double s1 = vc + vyp, s2 = vc + vym;
      double V2 = (s1 * s1 - s2 * s2) * ry12;
      double V3 = ((wyp * dyp + wc * dy) * (vzp + vc) - (wypzm * dyp + wzm * dy) * (vc + vzm)) *
                  ry12 * rz;
      double vv = 0.25 * (-V1 - V2 - V3) * DT;
      double L = ((vxp - vc) * rx12 - (vc - vxm) * rx12m) * rx +
                 ((vyp - vc) * ryp - (vc - vym) * ry) * ry12 +
                 ((vzp - vc) * rz12 - (vc - vzm) * rz12m) * rz;
      double va = a1 * vv + a2 * V_PRE[c] + kd * L;
      V_PRE[c] = vv;
      if (solid && c3 != 0.0) va += sp.eta * c3 * LD(V_TA, c) * DT;
      if (J == d.ny) va = 0.0;  // set_bc(u_a,v_a,...) zeroes v_a(:,ny,:)
      if (solid && c3 != 0.0) V_A[c] = (vc + va) / (1.0 + sp.eta * c3 * DT);
      else V_A[c] = vc + va;
    }
    // w
    {
      double W1 = ((uzp * dzp + uc * dz) * (wxp + wc) - (uxmzp * dzp + uxm * dz) * (wc + wxm)) *
                  rz12 * rx;
      double W2 = ((vzp * dzp + vc * dz) * (wyp + wc) - (vymzp * dzp + vym * dz) * (wc + wym)) *
                  rz12 * ry;
      double s1 = wc + wzp, s2 = wc + wzm;
      double W3 = (s1 * s1 - s2 * s2) * rz12;
      double wv = 0.25 * (-W1 - W2 - W3) * DT;
      double L = ((wxp - wc) * rx12 - (wc - wxm) * rx12m) * rx +
                 ((wyp - wc) * ry12 - (wc - wym) * ry12m) * ry +
                 ((wzp - wc) * rzp - (wc - wzm) * rz) * rz12;
      double wa = a1 * wv + a2 * W_PRE[c] + kd * L;
      W_PRE[c] = wv;
      if (solid && c4 != 0.0) {
        wa += sp.eta * c4 * LD(W_TA, c) * DT;
        W_A[c] = (wc + wa) / (1.0 + sp.eta * c4 * DT);
      } else {
        W_A[c] = wc + wa;
      }
    }
    // T
    {
      double UT = (-((r0 * txm * dx + r0 * tc * dxm) * uxm) * 0.5 * rx12m +
                   ((r0 * tc * dxp + r0 * txp * dx) * uc) * 0.5 * rx12) *
                  rx;
      double VT = (-((r0 * tym * dy + r0 * tc * dym) * vym) * 0.5 * ry12m +
                   ((r0 * tc * dyp + r0 * typ * dy) * vc) * 0.5 * ry12) *
                  ry;
      double WT = (-((r0 * tzm * dz + r0 * tc * dzm) * wzm) * 0.5 * rz12m +
                   ((r0 * tc * dzp + r0 * tzp * dz) * wc) * 0.5 * rz12) *
                  rz;
      double vt = (-UT - VT - WT) * DT * rr0 + sp.source * DT;
      double D1 = (l0 * (txp - tc) * rx12 - l0 * (tc - txm) * rx12m) * rx;
      double D2 = (l0 * (typ - tc) * ry12 - l0 * (tc - tym) * ry12m) * ry;
      double D3 = (l0 * (tzp - tc) * rz12 - l0 * (tc - tzm) * rz12m) * rz;
      double ut = a1 * vt + a2 * T_PRE[c] + kT * (D1 + D2 + D3);
      T_PRE[c] = vt;
      if (cc1 != 0.0) {
        double pen = sp.eta * cc1 * DT;
        U_T[c] = (tc + ut + pen * sp.tsolid) / (1.0 + pen);
      } else {
        U_T[c] = tc + ut;
      }
    }
  }
}

void launch_rhs_fast(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                     const double* u, const double* v, const double* w, const double* T,
                     const double* u_ta, const double* v_ta, const double* w_ta,
                     double* u_pre, double* v_pre, double* w_pre, double* T_pre,
                     const double* c1, double* u_a, double* v_a, double* w_a, double* u_T,
                     cudaStream_t s) {
  dim3 block(32, 8, 1);
  dim3 grid((d.nx + 31) / 32, (d.ny + 7) / 8, (d.nz + KCHUNK - 1) / KCHUNK);
  count_launch();
  k_rhs_fast<<<grid, block, 0, s>>>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre, v_pre,
                                    w_pre, T_pre, c1, u_a, v_a, w_a, u_T);
}

}  // namespace nse
