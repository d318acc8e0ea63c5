/*
 * c_driver.c -- a C restatement of the reference driver's time loop
 * (nse_dominik.f:246-257 and :290-446) that calls libnsegpu.so only through
 * the prototypes of include/nsegpu.h, the way the Fortran driver would call
 * the reference's own subroutines.  It is compiled by tests/test_c_driver.py
 * (gcc, -Wall -Werror) so that a mismatch between the header and what a C
 * caller passes fails the build, and its output is compared with the CPU
 * oracle's restatement of the same loop.
 *
 *   c_driver IN OUT
 *
 * IN holds: int32 nx, ny, nz, nsteps; float64 dt, Re, Sc, eta, xl, yl, zl;
 * then the padded fields u, v, w, T (each (nx+2)(ny+2)(nz+2) float64,
 * x fastest) and the cell mask c1 (nx*ny*nz float64).  OUT receives u, v,
 * w, p, T after nsteps steps.  Reference parameters: body force and heat
 * source 1 (hard-coded in SET_CONVECT / SET_CONVECTION_FOR_SCALAR), walls at
 * T = 0, rhoCp = thc = 1 (nse_dominik.f:190-191), uniform grid (SET_C).
 * Exit status 0 on success, 1 on an I/O error, 2 on a library error.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nsegpu.h"

static double* field(long n, double fill) {
  double* a = (double*)malloc((size_t)n * sizeof(double));
  for (long q = 0; q < n; ++q) a[q] = fill;
  return a;
}

static int failed(const char* where) {
  if (nse_last_status() != NSE_OK) {
    fprintf(stderr, "c_driver: %s: %s\n", where, nse_last_error());
    return 1;
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: c_driver IN OUT\n");
    return 1;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) return 1;
  int hdr[4];
  double par[7];
  if (fread(hdr, sizeof(int), 4, in) != 4 || fread(par, sizeof(double), 7, in) != 7) return 1;
  int nx = hdr[0], ny = hdr[1], nz = hdr[2], nsteps = hdr[3];
  double dt = par[0], Re = par[1], Sc = par[2], eta = par[3];
  double xl = par[4], yl = par[5], zl = par[6];
  const long n = (long)(nx + 2) * (ny + 2) * (nz + 2);
  const long nc = (long)nx * ny * nz;

  double *u = field(n, 0), *v = field(n, 0), *w = field(n, 0), *T = field(n, 0);
  double* cellvalue = field(4 * nc, 0);
  if (fread(u, sizeof(double), n, in) != (size_t)n || fread(v, sizeof(double), n, in) != (size_t)n ||
      fread(w, sizeof(double), n, in) != (size_t)n || fread(T, sizeof(double), n, in) != (size_t)n ||
      fread(cellvalue, sizeof(double), nc, in) != (size_t)nc)
    return 1;
  fclose(in);

  /* the arrays of the reference main that the step touches */
  double *p = field(n, 0), *u_v = field(n, 0), *v_v = field(n, 0), *w_v = field(n, 0);
  double *u_d = field(n, 0), *v_d = field(n, 0), *w_d = field(n, 0);
  double *u_a = field(n, 0), *v_a = field(n, 0), *w_a = field(n, 0);
  double *u_l = field(n, 0), *v_l = field(n, 0), *w_l = field(n, 0), *T_l = field(n, 0);
  double *u_ta = field(n, 0), *v_ta = field(n, 0), *w_ta = field(n, 0);
  double *u_pre = field(n, 0), *v_pre = field(n, 0), *w_pre = field(n, 0), *T_pre = field(n, 0);
  double *u_ep2 = field(n, 0), *v_ep2 = field(n, 0), *w_ep2 = field(n, 0), *divu = field(n, 0);
  double *u_temp = field(n, 0), *v_temp = field(n, 0), *w_temp = field(n, 0);
  double *u_vT = field(n, 0), *u_dT = field(n, 0), *u_T = field(n, 0);
  double *rhoCp = field(n, 1.0), *thc = field(n, 1.0);
  double *x = field(nx + 2, 0), *x12 = field(nx + 2, 0), *dx = field(nx + 2, 0),
         *dx12 = field(nx + 2, 0);
  double *y = field(ny + 2, 0), *y12 = field(ny + 2, 0), *dy = field(ny + 2, 0),
         *dy12 = field(ny + 2, 0);
  double *z = field(nz + 2, 0), *z12 = field(nz + 2, 0), *dz = field(nz + 2, 0),
         *dz12 = field(nz + 2, 0);
  double cons_cell = 0.0;
  const double ompnthreads = 1.0; /* passed, as the reference does, and ignored */

  set_c_(&nx, &ny, &nz, x, x12, y, y12, z, z12, dx, dx12, dy, dy12, dz, dz12, &xl, &yl, &zl);
  if (failed("set_c")) return 2;
  /* nse_dominik.f:246-257 */
  memcpy(u_pre, u, n * sizeof(double));
  memcpy(v_pre, v, n * sizeof(double));
  memcpy(w_pre, w, n * sizeof(double));
  memcpy(T_pre, T, n * sizeof(double));

  for (int l = 1; l <= nsteps; ++l) {
    set_bc_(u, v, w, p, &nx, &ny, &nz, T); /* :290 */
    set_convect_(u, u_v, v, v_v, w, w_v, &dt, &nx, &ny, &nz, dx, dy, dz, dx12, dy12, dz12);
    set_convection_for_scalar_(u, v, w, &dt, &nx, &ny, &nz, dx, dy, dz, dx12, dy12, dz12, T,
                               u_vT, rhoCp);
    set_conduction_(u, u_d, v, v_d, w, w_d, &Re, &dt, &nx, &ny, &nz, dx, dy, dz, dx12, dy12,
                    dz12);
    set_diffusion_for_scalar_(&Re, &dt, &nx, &ny, &nz, dx, dy, dz, dx12, dy12, dz12, T, u_dT,
                              &Sc, thc, rhoCp);
    set_immersed_boundary_(&eta, &nx, &ny, &nz, &dt, u_l, v_l, w_l, dx, dy, dz, T_l,
                           cellvalue, u_ta, v_ta, w_ta, &l, &cons_cell);
    set_explicit_(u_v, u_pre, u_d, u_a, v_v, v_pre, v_d, v_a, w_v, w_pre, w_d, w_a, u_l, v_l,
                  w_l, &nx, &ny, &nz, &l);
    set_explicit_for_tempreture_(u_vT, u_dT, u_T, T_pre, T_l, &nx, &ny, &nz, &l);
    set_bc_(u_a, v_a, w_a, p, &nx, &ny, &nz, T); /* :377 */
    if (failed("explicit terms")) return 2;
    /* :387-396 penalised temperature update */
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          long c = i + (long)(nx + 2) * (j + (long)(ny + 2) * k);
          long m = (i - 1) + (long)nx * ((j - 1) + (long)ny * (k - 1));
          u_T[c] = (T[c] + u_T[c]) / (1.0 + eta * cellvalue[m] * dt);
        }
    solve_u_temp_(u_a, v_a, w_a, &nx, &ny, &nz, dx, dy, dz, dx12, dy12, dz12, &Re, &dt, &eta,
                  cellvalue, u, v, w); /* :397 */
    memcpy(u_temp, u_a, n * sizeof(double)); /* :407-417 */
    memcpy(v_temp, v_a, n * sizeof(double));
    memcpy(w_temp, w_a, n * sizeof(double));
    solve_t_(u_T, &nx, &ny, &nz, dx, dy, dz, dx12, dy12, dz12, &Re, &Sc, &dt, rhoCp, thc,
             cellvalue, &eta); /* :419 */
    if (failed("line solves")) return 2;
    for (int k = 1; k <= nz; ++k) /* :429-437 */
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          long c = i + (long)(nx + 2) * (j + (long)(ny + 2) * k);
          T[c] = u_T[c];
        }
    set_bc_(u_temp, v_temp, w_temp, p, &nx, &ny, &nz, T); /* :441 */
    mkp_(p, u_temp, v_temp, w_temp, &dt, dx, dy, dz, dx12, dy12, dz12, &Re, &nx, &ny, &nz,
         &ompnthreads, u_ta, v_ta, w_ta, u_ep2, v_ep2, w_ep2, divu, u, v, w, &xl, &zl); /* :446 */
    if (failed("mkp")) return 2;
  }

  FILE* out = fopen(argv[2], "wb");
  if (!out) return 1;
  const double* res[5] = {u, v, w, p, T};
  for (int q = 0; q < 5; ++q)
    if (fwrite(res[q], sizeof(double), n, out) != (size_t)n) return 1;
  fclose(out);
  return 0;
}
