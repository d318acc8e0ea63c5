/*
 * nsegpu.h -- C-ABI of libnsegpu.so, the B200 (sm_100a) drop-in for the
 * fractional-step hot path of DominikHenzel/vtkmakeCompare.
 *
 * Tier 1 and tier 2 are the reference's own Fortran subroutines, exported
 * under gfortran's default mangling (lower case + trailing underscore), with
 * every argument passed by reference exactly as the Fortran caller passes it.
 * Arrays are the caller's host arrays in the reference layout:
 *   padded field  REAL*8 (0:nx+1,0:ny+1,0:nz+1), column-major (x fastest)
 *   cellvalue     REAL*8 (1:nx,1:ny,1:nz,1:4)
 *   spectrum      COMPLEX*16 (0:nx/2,0:ny+1,0:nz+1), interleaved re,im
 * Each call copies its inputs to the GPU, runs CUDA kernels and copies back
 * exactly the entries the reference routine writes.  Legacy entry points
 * return nothing (as in Fortran); on failure they print one line to stderr
 * and record the error for nse_last_error().  There is no CPU fallback: a
 * missing or unusable GPU is an error.
 *
 * Tier 3 is the resident API: the fields live in HBM across time steps and
 * every function returns an nse_status.
 *
 * Not re-entrant per context; one host thread per context.
 */
#ifndef NSEGPU_H
#define NSEGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum nse_status {
  NSE_OK = 0,
  NSE_ERR_ARG = 1,        /* bad dimension or argument */
  NSE_ERR_CUDA = 2,       /* CUDA runtime error or no usable GPU */
  NSE_ERR_NOMEM = 3,      /* device allocation failed */
  NSE_ERR_NONFINITE = 4,  /* non-finite value detected in a field */
  NSE_ERR_LIMIT = 5       /* size beyond a documented limit */
} nse_status;

const char* nse_last_error(void);
int nse_last_status(void);
void nse_clear_error(void);

/* ------------------------------------------ tier 1: the drop-in files ---- */

/* p2s_fftw2d.f:5 P2S(FP,FPT,NX,NY,NZ): per y-plane J=1..NY, real 2-D DFT of
 * FP(0:NX-1,J,0:NZ-1), half spectrum scaled by 1/(NX*NZ) into
 * FPT(0:NX/2,J,0:NZ-1).  Own radix kernels (no cuFFT/FFTW). */
void p2s_(double* FP, double* FPT, const int* NX, const int* NY, const int* NZ);
/* p2s_fftw2d.f:116 S2P(FPT,FP,NX,NY,NZ): inverse (unnormalised c2r) per plane,
 * then FP(NX,J,:)=FP(0,J,:), FP(:,J,NZ)=FP(:,J,0). */
void s2p_(double* FPT, double* FP, const int* NX, const int* NY, const int* NZ);

/* tridiag.f:5 TRIDIAG(A,B,NN), :21 TRID2(A,B,M,N), :43 CTRIDIAG(A,B,NN):
 * Thomas solves without pivoting; A(NN,3) is overwritten as in the reference. */
void tridiag_(double* A, double* B, const int* NN);
void trid2_(double* A, double* B, const int* M, const int* N);
void ctridiag_(double* A, double* B, const int* NN);

/* periodic_implicit.f:1 implicit_solver(SUX,nx,dx,dx12,Re,dt,ft,fb,eta,CUX),
 * :47 TDMA(a,b,c,r,u,n), :67 cyclic(a,b,c,alpha,beta,r,x,n).  The NMAX=500
 * static limit of the reference does not apply. */
void implicit_solver_(double* SUX, const int* nx, const double* dx, const double* dx12,
                      const double* Re, const double* dt, const double* ft,
                      const double* fb, const double* eta, const double* CUX);
void tdma_(const double* a, const double* b, const double* c, const double* r, double* u,
           const int* n);
void cyclic_(const double* a, const double* b, const double* c, const double* alpha,
             const double* beta, const double* r, double* x, const int* n);

/* mkp.f:9 MKP: projection step (divergence RHS, FFT Poisson, correction).
 * ompnthreads is accepted and ignored. */
void mkp_(double* p, double* u_temp, double* v_temp, double* w_temp, const double* dt,
          const double* dx, const double* dy, const double* dz, const double* dx12,
          const double* dy12, const double* dz12, const double* Re, const int* nx,
          const int* ny, const int* nz, const void* ompnthreads, double* u_ta, double* v_ta,
          double* w_ta, double* u_ep2, double* v_ep2, double* w_ep2, double* divu,
          double* u, double* v, double* w, const double* xl, const double* zl);
/* mkp.f:223 SPN, :263 SP0B, :293 PHIBC */
void spn_(const int* NX, const int* NY, const int* NZ, const double* AC, const double* KXZ,
          double* PHIT);
void sp0b_(const int* NX, const int* NY, const int* NZ, const double* AC, double* PHIT);
void phibc_(const int* NX, const int* NY, const int* NZ, double* PHI);

/* set_levelset.f:1 set_levelset(nx,ny,nz,dx,dx12,dy12,dz12,phi0,phi,x,y,z,cellvalue):
 * 2001 reinitialisation sweeps on the GPU, mask into cellvalue(:,:,:,1), and the
 * ASCII files levelset.vtk / cellvalue1.vtk written as the reference does
 * (set NSEGPU_NO_VTK=1 to skip the files). */
void set_levelset_(const int* nx, const int* ny, const int* nz, const double* dx,
                   const double* dx12, const double* dy12, const double* dz12,
                   const double* phi0, double* phi, const double* x, const double* y,
                   const double* z, double* cellvalue);
/* set_levelset.f:202 readgrid3d(nx,ny,nz,phi0): reads structure.dat (host I/O) */
void readgrid3d_(const int* nx, const int* ny, const int* nz, double* phi0);

/* --------------------------- tier 2: step routines of nse_dominik.f ---- */
void set_c_(const int* nx, const int* ny, const int* nz, double* x, double* x12, double* y,
            double* y12, double* z, double* z12, double* dx, double* dx12, double* dy,
            double* dy12, double* dz, double* dz12, const double* xl, const double* yl,
            const double* zl);                                   /* nse_dominik.f:553 */
void set_bc_(double* u, double* v, double* w, double* p, const int* nx, const int* ny,
             const int* nz, double* T);                          /* nse_dominik.f:611 */
void set_convect_(double* u, double* u_v, double* v, double* v_v, double* w, double* w_v,
                  const double* dt, const int* nx, const int* ny, const int* nz,
                  const double* dx, const double* dy, const double* dz, const double* dx12,
                  const double* dy12, const double* dz12);     /* nse_dominik.f:757 */
void set_convection_for_scalar_(double* u, double* v, double* w, const double* dt,
                                const int* nx, const int* ny, const int* nz,
                                const double* dx, const double* dy, const double* dz,
                                const double* dx12, const double* dy12, const double* dz12,
                                double* T, double* u_vT, double* rhoCp); /* :834 */
void set_conduction_(double* u, double* u_d, double* v, double* v_d, double* w, double* w_d,
                     const double* Re, const double* dt, const int* nx, const int* ny,
                     const int* nz, const double* dx, const double* dy, const double* dz,
                     const double* dx12, const double* dy12, const double* dz12); /* :888 */
void set_diffusion_for_scalar_(const double* Re, const double* dt, const int* nx,
                               const int* ny, const int* nz, const double* dx,
                               const double* dy, const double* dz, const double* dx12,
                               const double* dy12, const double* dz12, double* T,
                               double* u_dT, const double* Sc, double* thc,
                               double* rhoCp);                   /* :950 */
void set_immersed_boundary_(const double* eta, const int* nx, const int* ny, const int* nz,
                            const double* dt, double* u_l, double* v_l, double* w_l,
                            const double* dx, const double* dy, const double* dz,
                            double* T_l, double* cellvalue, double* u_ta, double* v_ta,
                            double* w_ta, const int* l, double* cons_cell); /* :1011 */
void set_explicit_(double* u_v, double* u_pre, double* u_d, double* u_a, double* v_v,
                   double* v_pre, double* v_d, double* v_a, double* w_v, double* w_pre,
                   double* w_d, double* w_a, double* u_l, double* v_l, double* w_l,
                   const int* nx, const int* ny, const int* nz, const int* l); /* :1132 */
void set_explicit_for_tempreture_(double* u_vT, double* u_dT, double* u_T, double* T_pre,
                                  double* T_l, const int* nx, const int* ny, const int* nz,
                                  const int* l);                  /* :1291 */
void solve_u_temp_(double* u_a, double* v_a, double* w_a, const int* nx, const int* ny,
                   const int* nz, const double* dx, const double* dy, const double* dz,
                   const double* dx12, const double* dy12, const double* dz12,
                   const double* Re, const double* dt, const double* eta,
                   double* cellvalue, double* u, double* v, double* w); /* :1344 */
void solve_t_(double* u_T, const int* nx, const int* ny, const int* nz, const double* dx,
              const double* dy, const double* dz, const double* dx12, const double* dy12,
              const double* dz12, const double* Re, const double* Sc, const double* dt,
              double* rhoCp, double* thc, double* cellvalue, const double* eta); /* :1465 */
/* single-line solvers nse_dominik.f:1505 implicit_uy, :1583 implicit_vy,
 * :1725 implicit_Tx, :1784 implicit_Ty */
void implicit_uy_(double* SUY, const int* ny, const double* dy, const double* dy12,
                  const double* Re, const double* dt, const double* ft, const double* fb,
                  const double* eta, const double* CUY);
void implicit_vy_(double* SVY, const int* ny, const double* dy, const double* dy12,
                  const double* Re, const double* dt, const double* ft, const double* fb,
                  const double* eta, const double* CVY);
void implicit_tx_(double* STX, const int* nx, const double* dx, const double* dx12,
                  const double* Re, const double* Sc, const double* dt, const double* llx,
                  const double* rrx, const double* ft, const double* fb, const double* eta,
                  const double* CUX);
void implicit_ty_(double* STY, const int* ny, const double* dy, const double* dy12,
                  const double* Re, const double* Sc, const double* dt, const double* lly,
                  const double* rry, const double* ft, const double* fb, const double* CUY,
                  const double* eta);
/* line drivers of the reference's OpenMP loops, nse_dominik.f:2893 parallel_uy,
 * :2912 parallel_z, :2931 parallel_x, :2950 parallel_vy, :2969 parallel_Tx,
 * :2995 parallel_Ty, :3021 parallel_Tz: one line of the padded field (line
 * indices 1-based, mask column n of cellvalue), solved by the single-line
 * solver above; each writes the entries its reference routine writes
 * (u_a(i,0:ny+1,k); v_a(i,0:ny,k); u_a(i,j,0:nz+1); u_a(0:nx+1,j,k); u_T on
 * the interior of the line).  The end entries of the rhoCp/thc line locals,
 * which the reference leaves unset, are the fields' ghost cells. */
void parallel_uy_(const int* i, const int* k, double* u_a, const double* cellvalue,
                  const int* nx, const int* ny, const int* nz, const double* dy,
                  const double* dy12, const double* Re, const double* dt, const double* eta,
                  const int* n);
void parallel_vy_(const int* i, const int* k, double* v_a, const double* cellvalue,
                  const int* nx, const int* ny, const int* nz, const double* dy,
                  const double* dy12, const double* Re, const double* dt, const double* eta,
                  const int* n);
void parallel_z_(const int* i, const int* j, double* u_a, const double* cellvalue,
                 const int* nx, const int* ny, const int* nz, const double* dz,
                 const double* dz12, const double* Re, const double* dt, const double* eta,
                 const int* n);
void parallel_x_(const int* j, const int* k, double* u_a, const double* cellvalue,
                 const int* nx, const int* ny, const int* nz, const double* dx,
                 const double* dx12, const double* Re, const double* dt, const double* eta,
                 const int* n);
void parallel_tx_(const int* k, const int* j, const int* nx, const int* ny, const int* nz,
                  const double* rhoCp, const double* thc, double* u_T,
                  const double* cellvalue, const double* dx, const double* dx12,
                  const double* Re, const double* Sc, const double* dt, const double* eta);
void parallel_ty_(const int* i, const int* k, const int* nx, const int* ny, const int* nz,
                  const double* rhoCp, const double* thc, double* u_T,
                  const double* cellvalue, const double* dy, const double* dy12,
                  const double* Re, const double* Sc, const double* dt, const double* eta);
void parallel_tz_(const int* i, const int* j, const int* nx, const int* ny, const int* nz,
                  const double* rhoCp, const double* thc, double* u_T,
                  const double* cellvalue, const double* dz, const double* dz12,
                  const double* Re, const double* Sc, const double* dt, const double* eta);
/* OUTPUT (nse_dominik.f:2606): ./nseoutput2/{velocity,temperature,pressure,
 * divergence,gridx,gridy,gridz,gridnumber,phi,cellvalue1..4}.dat, field.u,
 * grid.u and ./temperature_check.dat, byte for byte as gfortran writes them
 * (sequential unformatted records with 4-byte length markers) */
void output_(const double* u, const double* v, const double* w, const double* p,
             const double* x, const double* y, const double* z, const int* nx, const int* ny,
             const int* nz, const double* T, const double* cellvalue, const double* u_ta,
             const double* v_ta, const double* w_ta, const double* phi, const double* divu);
/* OUTFIELD (nse_dominik.f:2726): ./field.u (time record first) and
 * ./nseoutput2/grid.u */
void outfield_(const double* x, const double* y, const double* z, const double* u,
               const double* v, const double* w, const double* p, const int* nx,
               const int* ny, const int* nz, const double* tid, const double* T,
               const double* phi, const double* u_ta, const double* v_ta,
               const double* w_ta);
/* READFIELD (nse_dominik.f:2769): ./nseoutput2/field.u into the arrays */
void readfield_(double* u, double* v, double* w, double* p, const int* nx, const int* ny,
                const int* nz, double* T, double* phi, double* u_ta, double* v_ta,
                double* w_ta);

/* Extension (no counterpart in the reference): SET_C with the y faces
 * y12(j) = y0 + yl/2 (1 + tanh(gamma(2j/ny-1))/tanh(gamma)), j=0..ny, the
 * ghost spacing mirrored; gamma = 0 gives SET_C shifted by y0. */
void nse_set_c_stretched(int nx, int ny, int nz, double* x, double* x12, double* y,
                         double* y12, double* z, double* z12, double* dx, double* dx12,
                         double* dy, double* dy12, double* dz, double* dz12, double xl,
                         double yl, double zl, double y0, double gamma);

/* No counterpart in the reference.  SPN (mkp.f:223) for callers that cannot
 * allocate GPU memory: AC (ny,3), KXZ (nx/2+1, nz+1) and the complex spectrum
 * PHIT (0:nx/2, 0:ny+1, 0:nz+1) are DEVICE pointers in the reference layouts;
 * the solve is queued on `stream` (a cudaStream_t, NULL = legacy default
 * stream) and the function returns without synchronising.  It allocates
 * nothing: its scratch is a fixed array inside the library of
 * NSE_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB, resident on every GPU that
 * loads the library until exit), so (nx/2+1)*ny*nz must not exceed it, nor
 * nz 65535 (NSE_ERR_LIMIT otherwise).  The first call on a device looks up
 * the array's device address and keeps it for the life of the process; make
 * that first call before any stream capture, and do not call this entry
 * point on a device after cudaDeviceReset.  Calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller.  A CUDA
 * error pending from the caller's earlier work is reported (NSE_ERR_CUDA)
 * and left in place.  Returns an nse_status. */
#define NSE_NOALLOC_SCRATCH_DOUBLES (2L * 1024L * 1024L)
int nse_spn_noalloc(int nx, int ny, int nz, const double* AC, const double* KXZ,
                    double* PHIT, void* stream);

/* ------------------------------------------------ tier 3: resident API ---- */
typedef struct nse_config {
  int nx, ny, nz;
  double dt, Re, Sc, eta;
  double xl, yl, zl;
  double y0;            /* y origin (0 in the reference SET_C) */
  double ystretch;      /* tanh stretching gamma in y; 0 = uniform (reference) */
  double body_force;    /* x body force; 1.0 in the reference (nse_dominik.f:785) */
  double heat_source;   /* volumetric heat source; 1.0 in the reference (:879) */
  double t_bot, t_top;  /* wall temperatures at y=y0, y=y0+yl; 0 in the reference */
  double t_solid;       /* temperature imposed in the solid; 0 in the reference */
  double rho_cp, thc;   /* uniform rhoCp and conductivity; 1 in the reference */
  int precision;        /* NSE_FP64 (plain) or NSE_MIXED */
  int flags;
} nse_config;

/* NSE_MIXED (no counterpart in the reference): u, v, w, T, p and the Poisson
 * solution stay FP64; the right-hand-side stencils and the line sweeps run
 * on FP32 intermediates; the divergence of the FP32 provisional velocity,
 * the Poisson solve (transforms, spectral recurrences, mean mode), the
 * correction and the reductions are FP64.  With NSE_FLAG_POISSON32 the
 * Poisson transforms and spectrum are FP32 instead (FP64 recurrences) with
 * one FP64 residual-refinement pass (two with NSE_FLAG_REFINE2).  u_ta, the
 * AB2 histories, u_ep2 and divu are held in FP32 (upload/download convert).
 * Needs nx = 32*M (M in 3, 4, 5, 6, 8, 16) and 12..512 cells in y and z. */
enum { NSE_FP64 = 0, NSE_MIXED = 1 };
/* nse_config.flags bits */
enum {
  NSE_FLAG_CHECK_FINITE = 1, /* nse_step checks every step for non-finite values */
  NSE_FLAG_EXACT = 4,        /* resident step rounds every operation like the reference
                                (no FMA, true divisions); default is the fast form */
  NSE_FLAG_REFINE2 = 8,      /* NSE_MIXED + NSE_FLAG_POISSON32: two refinement passes
                                instead of one */
  NSE_FLAG_POISSON64 = 16,   /* NSE_MIXED: FP64 Poisson solve (the default; kept so
                                callers that set it keep working) */
  NSE_FLAG_MATH64 = 32,      /* NSE_MIXED: FP64 arithmetic in the right-hand-side stencils
                                (their results are still stored in FP32) */
  NSE_FLAG_LINES64 = 64,     /* NSE_MIXED: FP64 arithmetic and tables in the line sweeps
                                (FP32 storage) */
  NSE_FLAG_ONE_STREAM = 128, /* everything on the context's stream, in the reference's
                                order (default: the line passes of u, v, w, T as four
                                concurrent chains on side streams; same results) */
  NSE_FLAG_POISSON3 = 256,   /* FP64 Poisson solve in three launches (each plane's 2-D
                                transform in one cluster launch, partitioned SPN; NX =
                                NZ = 256, ny = 16 m) instead of the five-launch default */
  NSE_FLAG_POISSON32 = 512,  /* NSE_MIXED: FP32 Poisson transforms and spectrum with FP64
                                residual refinement instead of the FP64 solve */
  NSE_FLAG_LINES_TMA = 1024, /* FP64 fast form: the y and z line passes stream tiles of
                                16 lines through shared memory by TMA copies (persistent
                                CTAs, next tile in flight while one is solved) */
  NSE_FLAG_NO_AUTOTUNE = 2048, /* keep the fixed line launch shapes instead of timing the
                                candidates before the first step (same values either way) */
  NSE_FLAG_SPN_TMA = 4096,   /* FP64 spectral tridiagonal solve (SPN + SP0B) through TMA
                                tiles of 16 kx columns, partitioned over 16 warps
                                (ny = 16 m), instead of the two-ended solver */
  NSE_FLAG_MID_SLICES = 8192, /* FP64 five-launch solve with NZ = 256: run the z
                                transforms and the SPN in 3 kx slices without timing the
                                slice counts (same values either way) */
  NSE_FLAG_SPN_CPASYNC = 16384 /* fast forms: the two-ended SPN stages its rows by
                                per-thread cp.async copies instead of TMA tiles of 16 kx
                                columns (same values either way) */
};

/* field ids for upload/download (padded fields unless noted) */
enum nse_field {
  NSE_U = 0, NSE_V, NSE_W, NSE_P, NSE_T,
  NSE_U_TA, NSE_V_TA, NSE_W_TA,
  NSE_U_PRE, NSE_V_PRE, NSE_W_PRE, NSE_T_PRE,
  NSE_DIVU, NSE_U_EP2, NSE_V_EP2, NSE_W_EP2,
  NSE_PHI,          /* Poisson right-hand side / solution (padded) */
  NSE_CELLVALUE,    /* (nx,ny,nz,4) mask, only column 1 is used on upload */
  NSE_NUM_FIELDS
};

typedef struct nse_ctx nse_ctx;

int nse_ctx_create(const nse_config* cfg, nse_ctx** out);
int nse_ctx_destroy(nse_ctx* ctx);
/* run subsequent work on this cudaStream_t (NULL = the context's own stream) */
int nse_ctx_set_stream(nse_ctx* ctx, void* stream);
int nse_ctx_upload(nse_ctx* ctx, int field, const double* host);
int nse_ctx_download(nse_ctx* ctx, int field, double* host);
/* grid arrays (each n+2 long) of the context, as SET_C / its stretched variant */
int nse_ctx_grid(nse_ctx* ctx, double* x, double* x12, double* y, double* y12, double* z,
                 double* z12, double* dx, double* dx12, double* dy, double* dy12,
                 double* dz, double* dz12);
/* step counter l of the reference loop (1 = first step: Euler start, masks built) */
int nse_ctx_set_step(nse_ctx* ctx, int l);
int nse_ctx_get_step(nse_ctx* ctx);
/* copy u,v,w,T into the AB2 histories (nse_dominik.f:246-257) */
int nse_start(nse_ctx* ctx);
/* nsteps time steps (nse_dominik.f:290-446), asynchronous on the context stream */
int nse_step(nse_ctx* ctx, int nsteps);
/* MKP on the resident fields, reading u,v,w (with SET_BC applied to a copy,
   as nse_dominik.f:441 does before MKP) as u_temp (asynchronous) */
int nse_project(nse_ctx* ctx);
/* Poisson solve P2S->SPN->SP0B->S2P->PHIBC in place on the NSE_PHI field */
int nse_poisson(nse_ctx* ctx);
/* level set reinitialisation + mask from a padded phi0 (host) into the
 * resident mask; phi_out (padded, host) may be NULL */
int nse_levelset(nse_ctx* ctx, const double* phi0, double* phi_out, int nnn, double dtau,
                 double width);
/* The reference's output and restart files from the resident fields (same
 * bytes as OUTPUT / OUTFIELD / READFIELD would give for the downloaded
 * arrays): root/nseoutput2/... and root/temperature_check.dat; field.u with
 * the time record at `path`, grid.u at `grid_path` (NULL: not written);
 * READFIELD's field.u (no time record) into u, v, w, p, T, the level set
 * phi and u_ta, v_ta, w_ta.  phi is the level set of the last nse_levelset
 * (zero before one); cellvalue 2..4 are the face masks of the current mask. */
int nse_ctx_write_output(nse_ctx* ctx, const char* root);
int nse_ctx_write_field(nse_ctx* ctx, const char* path, double tid, const char* grid_path);
int nse_ctx_read_field(nse_ctx* ctx, const char* path);
/* FP64 device reductions: out[0]=max|divu|, out[1]=sum|u|dx, out[2]=sum|v|dy,
 * out[3]=sum|w|dz, out[4]=sum T dx dy dz (all cells), out[5]=non-finite count */
int nse_monitor(nse_ctx* ctx, double out[6]);
int nse_sync(nse_ctx* ctx);
/* Launch shapes the autotuner chose (set before the context's first step;
 * no counterpart in the reference), out[15]: out[(dir-1)*4 + comp] for the y
 * (dir 1) and z (dir 2) line passes of u, v, w, T (0 = 16 lines per CTA, 1 =
 * 8, 3 = 32, 2 = TMA tiles of 16 lines), out[8 + comp] the x lines per warp
 * iteration (1 or 2; 3 and 4 the same through shared-memory staged loads), out[12] the right-hand-side kernel's shape (0 = 32x4 tiles with a
 * 5-plane ring in FP64 / 32x8 in FP32, 1 = 32x4 with 4 planes, 2 = 32x8 with
 * 5, 3 = 32x8 with 4; the ring filled by TMA copies (FP32 storage: the FP64
 * halo planes by TMA, the history tiles by cp.async): 4 = 32x4 with 5 planes,
 * 5 = 32x4 with 4, 6 = 32x8 with 4), out[13] the pipelined
 * correction's shape (0 = the default, 1 = 32x8 tiles with 5 planes, 2 = 32x4
 * with 4, 3 = 32x8 with 4; FP64 TMA ring: 4 = 32x4 with 4 planes, 5 = 32x4
 * with 5, 6 = 32x8 with 4, 7 = 32x4 with 7, 8 = 32x4 with 6; 16 z planes per
 * CTA: 9 = 32x4 with 5, 10 = 32x4 with 4; the TMA ring holding only what the
 * correction reads: 11 = 32x4 with 5, 12 = 32x4 with 4, 13 = as 11 with 16 z
 * planes per CTA, 14 = 32x4 with 5 and four CTAs per SM; 15 = the full TMA
 * ring with 5 planes and three CTAs), out[14] the kx
 * slices the FP64 solve's z
 * transforms and SPN run in (1 = unsliced). */
int nse_ctx_launch_shapes(nse_ctx* ctx, int* out);
/* Fix the right-hand-side and correction launch shapes (codes as above; -1
 * leaves that one to the autotuner) before the first step; every shape gives
 * the same values.  NSE_ERR_ARG for a code outside -1..6 (right-hand side)
 * or -1..15 (correction). */
int nse_ctx_set_shapes(nse_ctx* ctx, int rhs_shape, int corr_shape);
/* Fix the launch shapes of every partitioned line pass (y/z: 0..3 as in
 * nse_ctx_launch_shapes; x: 1..4 lines per warp iteration / staged loads)
 * before the first step instead of the autotuner's choice; every shape gives
 * the same values.  NSE_ERR_ARG outside those ranges. */
int nse_ctx_set_line_shapes(nse_ctx* ctx, int yz_shape, int x_lines);
/* Per-phase timing of the next max_steps steps with CUDA events on the
 * context stream (0 disables).  nse_ctx_phase_times returns, per phase, the
 * summed milliseconds over the profiled steps; phases in launch order:
 * set_bc, rhs, y-lines u/v/w, z-lines u/v/w, x-lines u/v/w, T y, T x, T z,
 * set_bc(u_temp), fft x fwd, fft z fwd, spn+sp0b, fft z inv, fft x inv,
 * phibc, refinement (mixed form), correction (17 phases).  Profiled steps
 * run every pass in order on the context's stream (no side streams), so each
 * phase is timed on its own. */
int nse_ctx_profile(nse_ctx* ctx, int max_steps);
int nse_ctx_phase_times(nse_ctx* ctx, double* ms, int nphase, int* nsteps);
/* Ensemble (no counterpart in the reference): independent cases, each a
 * context created as usual (grids, masks and precisions may differ), stepped
 * together.  Case i runs on stream i mod nstreams (owned by the ensemble;
 * nse_ensemble_destroy gives each case its own stream back).  The first step
 * of every case runs eagerly (the Euler start; it also builds the mask's
 * line tables); later steps replay a CUDA graph captured from two steps of
 * all cases, with an eager step for an odd remainder.  A case's mask and
 * parameters must not change while it belongs to an ensemble, and contexts
 * with NSE_FLAG_CHECK_FINITE are refused.  Asynchronous; nse_ensemble_sync
 * waits for all cases. */
typedef struct nse_ensemble nse_ensemble;
int nse_ensemble_create(nse_ctx** cases, int n, int nstreams, nse_ensemble** out);
int nse_ensemble_step(nse_ensemble* ens, int nsteps);
/* graph replays go to `stream` (a cudaStream_t of the caller) instead of the
 * ensemble's own; the case streams are forked from and joined into it */
int nse_ensemble_set_stream(nse_ensemble* ens, void* stream);
int nse_ensemble_sync(nse_ensemble* ens);
int nse_ensemble_destroy(nse_ensemble* ens);
/* Discrete adjoint (no counterpart in the reference, whose adjoint.f is a set
 * of unconnected routines): the exact transpose of the FP64 resident step.
 * Objective, from the context's current state over nsteps steps:
 *   J = mean over steps avg_from..nsteps of the wall heat flux at y = y0,
 *       sum_ik a_ik thc (T(i,1,k) - T(i,0,k)) / dy12(0), a_ik = dx_i dz_k/(xl zl),
 *       with the wall ghost T(i,0,k) = 2 t_bot - T(i,1,k)
 *     + sum over state fields f of <W_f, f after nsteps> (nse_adjoint_set_weight).
 * nse_adjoint_gradient returns J and dJ/dc1 (nx*ny*nz, the layout of
 * cellvalue's first column); the adjoint of the initial state is then read
 * with nse_adjoint_download (padded field; u, v, w, T, u_ta, v_ta, w_ta and
 * the AB2 histories).  The forward run is checkpointed every
 * checkpoint_every steps in device memory and replayed per segment; the
 * context is left at the state after nsteps.  FP64 contexts only. */
typedef struct nse_adjoint nse_adjoint;
typedef struct nse_adjoint_config {
  int nsteps;
  int checkpoint_every;
  int avg_from;  /* first step (1-based) of the averaging window */
} nse_adjoint_config;
int nse_adjoint_create(nse_ctx* ctx, const nse_adjoint_config* cfg, nse_adjoint** out);
/* weights (padded field, interior used) of a linear functional of the final
 * state field `field` added to J; NULL removes them */
int nse_adjoint_set_weight(nse_adjoint* adj, int field, const double* weights);
/* forward run only: J */
int nse_adjoint_objective(nse_adjoint* adj, double* J);
int nse_adjoint_gradient(nse_adjoint* adj, double* J, double* grad_c1);
int nse_adjoint_download(nse_adjoint* adj, int field, double* host);
int nse_adjoint_destroy(nse_adjoint* adj);

/* adjoint.f routines (drop-ins, same arguments): set_adj_convect adjoint.f:1,
 * set_adj_convection_for_scalar :128, set_adj_ns_scalar :185.  They compute
 * what the reference's routines compute (including their index slips); the
 * reference's set_adj_NS_scalar reads its adjoint temperature T_final from an
 * uninitialised local array, which static zero-filled storage makes zero:
 * set_adj_ns_scalar_ uses zero, nse_adj_ns_scalar takes T_final. */
void set_adj_convect_(double* u, double* u_v, double* v, double* v_v, double* w, double* w_v,
                      const double* Re, const double* dt, const int* nx, const int* ny,
                      const int* nz, const double* dx, const double* dy, const double* dz,
                      const double* dx12, const double* dy12, const double* dz12,
                      double* u_final, double* v_final, double* w_final);
void set_adj_convection_for_scalar_(double* u, double* v, double* w, const double* Re,
                                    const double* dt, const int* nx, const int* ny,
                                    const int* nz, const double* dx, const double* dy,
                                    const double* dz, const double* dx12, const double* dy12,
                                    const double* dz12, double* T, double* u_vT,
                                    double* rhoCp, double* u_final, double* v_final,
                                    double* w_final);
void set_adj_ns_scalar_(const double* dt, const int* nx, const int* ny, const int* nz,
                        const double* dx12, const double* dy12, const double* dz12, double* T,
                        double* u_s, double* v_s, double* w_s, double* u_final,
                        double* v_final, double* w_final);
int nse_adj_ns_scalar(const double* dt, int nx, int ny, int nz, const double* dx12,
                      const double* dy12, const double* dz12, const double* T,
                      const double* T_final, double* u_s, double* v_s, double* w_s);

/* Device memory the library holds at once (all its allocations: contexts,
 * ensembles, adjoints and the staging buffers of the legacy entry points),
 * capped at `bytes` (0 = no cap, the default).  An allocation beyond the cap
 * fails like an out-of-memory one: NSE_ERR_NOMEM, and a context being
 * created is released.  No counterpart in the reference. */
void nse_set_alloc_limit(long long bytes);
long long nse_alloc_bytes(void);

/* number of kernel launches this process has issued through the library */
long long nse_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
