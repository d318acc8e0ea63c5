/*
 * nse_oracle.h -- CPU oracle for the fractional-step Navier-Stokes + heat hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++17/OpenMP restatement of the
 * reference Fortran routines (DominikHenzel/vtkmakeCompare: mkp.f, tridiag.f,
 * periodic_implicit.f, p2s_fftw2d.f, set_levelset.f and the step routines of
 * nse_dominik.f).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it, and only as the checker or the
 * timed CPU baseline.  The product library (libnsegpu.so) never links it.
 *
 * Every routine keeps the reference's argument meaning and floating-point
 * operation order (left-to-right Fortran evaluation, no FMA contraction:
 * build with -ffp-contract=off).  Arrays use the reference layout:
 * a padded field is Fortran column-major (0:nx+1,0:ny+1,0:nz+1), x fastest.
 *
 * Parity status of the FFT (p2s/s2p): the reference calls FFTW3 (not vendored,
 * version unpinned).  The oracle computes the transform FFTW documents
 * (unnormalised DFT, r2c half spectrum, c2r of the Hermitian extension) with
 * its own mixed-radix FFT; the tests pin it against numpy.fft and a direct
 * O(N^2) DFT.  Parity against FFTW itself is unpinned.
 */
#ifndef NSE_ORACLE_H
#define NSE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* grid (nse_dominik.f:553-607) and the tanh-stretched y variant */
void or_set_c(int nx, int ny, int nz, double* x, double* x12, double* y, double* y12,
              double* z, double* z12, double* dx, double* dx12, double* dy, double* dy12,
              double* dz, double* dz12, double xl, double yl, double zl);
void or_set_c_stretched(int nx, int ny, int nz, double* x, double* x12, double* y,
                        double* y12, double* z, double* z12, double* dx, double* dx12,
                        double* dy, double* dy12, double* dz, double* dz12, double xl,
                        double yl, double zl, double y0, double gamma);

/* step routines of nse_dominik.f */
void or_set_bc(double* u, double* v, double* w, double* p, int nx, int ny, int nz,
               double* T, double tbot, double ttop);
void or_set_convect(const double* u, double* u_v, const double* v, double* v_v,
                    const double* w, double* w_v, double dt, int nx, int ny, int nz,
                    const double* dx, const double* dy, const double* dz,
                    const double* dx12, const double* dy12, const double* dz12,
                    double force);
void or_set_convection_for_scalar(const double* u, const double* v, const double* w,
                                  double dt, int nx, int ny, int nz, const double* dx,
                                  const double* dy, const double* dz, const double* dx12,
                                  const double* dy12, const double* dz12, const double* T,
                                  double* u_vT, const double* rhoCp, double source);
void or_set_conduction(const double* u, double* u_d, const double* v, double* v_d,
                       const double* w, double* w_d, double Re, double dt, int nx, int ny,
                       int nz, const double* dx, const double* dy, const double* dz,
                       const double* dx12, const double* dy12, const double* dz12);
void or_set_diffusion_for_scalar(double Re, double dt, int nx, int ny, int nz,
                                 const double* dx, const double* dy, const double* dz,
                                 const double* dx12, const double* dy12,
                                 const double* dz12, const double* T, double* u_dT,
                                 double Sc, const double* thc, const double* rhoCp);
void or_set_immersed_boundary(double eta, int nx, int ny, int nz, double dt, double* u_l,
                              double* v_l, double* w_l, double* T_l, double* cellvalue,
                              const double* u_ta, const double* v_ta, const double* w_ta,
                              int l);
void or_set_explicit(const double* u_v, double* u_pre, const double* u_d, double* u_a,
                     const double* v_v, double* v_pre, const double* v_d, double* v_a,
                     const double* w_v, double* w_pre, const double* w_d, double* w_a,
                     const double* u_l, const double* v_l, const double* w_l, int nx,
                     int ny, int nz, int l);
void or_set_explicit_for_tempreture(const double* u_vT, const double* u_dT, double* u_T,
                                    double* T_pre, const double* T_l, int nx, int ny,
                                    int nz, int l);

/* line solvers */
void or_implicit_uy(double* SUY, int ny, const double* dy, const double* dy12, double Re,
                    double dt, double ft, double fb, double eta, const double* CUY);
void or_implicit_vy(double* SVY, int ny, const double* dy, const double* dy12, double Re,
                    double dt, double ft, double fb, double eta, const double* CVY);
void or_implicit_ty(double* STY, int ny, const double* dy, const double* dy12, double Re,
                    double Sc, double dt, const double* lly, const double* rry, double ft,
                    double fb, const double* CUY, double eta);
void or_implicit_tx(double* STX, int nx, const double* dx, const double* dx12, double Re,
                    double Sc, double dt, const double* llx, const double* rrx, double ft,
                    double fb, double eta, const double* CUX);
void or_implicit_solver(double* SUX, int nx, const double* dx, const double* dx12,
                        double Re, double dt, double ft, double fb, double eta,
                        const double* CUX);
void or_tdma(const double* a, const double* b, const double* c, const double* r, double* u,
             int n);
void or_cyclic(const double* a, const double* b, const double* c, double alpha,
               double beta, const double* r, double* x, int n);
void or_solve_u_temp(double* u_a, double* v_a, double* w_a, int nx, int ny, int nz,
                     const double* dx, const double* dy, const double* dz,
                     const double* dx12, const double* dy12, const double* dz12, double Re,
                     double dt, double eta, const double* cellvalue, const double* u,
                     const double* v, const double* w);
void or_solve_t(double* u_T, int nx, int ny, int nz, const double* dx, const double* dy,
                const double* dz, const double* dx12, const double* dy12,
                const double* dz12, double Re, double Sc, double dt, const double* rhoCp,
                const double* thc, const double* cellvalue, double eta, double ft_y,
                double fb_y);

/* tridiag.f */
void or_tridiag(double* A, double* B, int NN);
void or_trid2(double* A, double* B, int M, int N);
void or_ctridiag(double* A, double* B /* complex interleaved */, int NN);

/* p2s_fftw2d.f, mkp.f */
void or_p2s(const double* FP, double* FPT /* complex interleaved */, int NX, int NY, int NZ);
void or_s2p(const double* FPT, double* FP, int NX, int NY, int NZ);
void or_spn(int NX, int NY, int NZ, const double* AC, const double* KXZ, double* PHIT);
void or_sp0b(int NX, int NY, int NZ, const double* AC, double* PHIT);
void or_phibc(int NX, int NY, int NZ, double* PHI);
void or_mkp_coeffs(int nx, int ny, int nz, const double* dx, const double* dy,
                   const double* dz, const double* dy12, double xl, double zl, double* AC,
                   double* KXZ);
void or_mkp(double* p, const double* u_temp, const double* v_temp, const double* w_temp,
            double dt, const double* dx, const double* dy, const double* dz,
            const double* dx12, const double* dy12, const double* dz12, double Re, int nx,
            int ny, int nz, double* u_ta, double* v_ta, double* w_ta, double* u_ep2,
            double* v_ep2, double* w_ep2, double* divu, double* u, double* v, double* w,
            double xl, double zl, double* phi_work);

/* set_levelset.f */
void or_set_levelset(int nx, int ny, int nz, const double* dx, const double* dx12,
                     const double* dy12, const double* dz12, const double* phi0,
                     double* phi, double* cellvalue, int nnn, double dtau, double width);

/* one time step of nse_dominik.f:261-446 (diagnostics and file output omitted) */
typedef struct or_state {
  int nx, ny, nz, l;
  double dt, Re, Sc, eta, xl, zl;
  double force, source, tbot, ttop, tsolid;
  double *dx, *dy, *dz, *dx12, *dy12, *dz12;
  double *u, *v, *w, *p, *T;
  double *u_ta, *v_ta, *w_ta, *u_pre, *v_pre, *w_pre, *T_pre;
  double *divu, *u_ep2, *v_ep2, *w_ep2;
  double *cellvalue, *rhoCp, *thc;
  double *u_v, *v_v, *w_v, *u_d, *v_d, *w_d, *u_a, *v_a, *w_a;
  double *u_l, *v_l, *w_l, *u_temp, *v_temp, *w_temp;
  double *u_vT, *u_dT, *u_T, *T_l, *phi_work;
} or_state;
void or_step(or_state* s);

/* timing mode: 1 keeps the reference's per-line dense (n+2)^2 matrix zeroing in the
 * y-line solvers (nse_dominik.f:1519-1523,1596-1600,1800-1804); 0 skips it. */
void or_set_faithful(int on);
int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
