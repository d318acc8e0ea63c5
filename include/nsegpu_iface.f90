! nsegpu_iface.f90 -- Fortran 2003 interfaces to the resident (tier 3) API of
! libnsegpu.so.  The reference subroutines themselves (MKP, P2S, S2P, SPN,
! SP0B, PHIBC, CTRIDIAG, TRIDIAG, TRID2, implicit_solver, TDMA, cyclic,
! set_levelset, readgrid3d, the step routines of nse_dominik.f with their
! parallel_* line drivers, and the adjoint.f routines set_adj_convect,
! set_adj_convection_for_scalar, set_adj_NS_scalar) need no interface:
! libnsegpu.so exports them under gfortran's mangled names (mkp_, p2s_, ...),
! so a driver that calls them links against the library instead of the
! reference object files (link line: -L<dir of libnsegpu.so> -lnsegpu, with
! the reference's mkp.f, p2s_fftw2d.f, tridiag.f, periodic_implicit.f and
! set_levelset.f left out of the link).
module nsegpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: NSE_OK = 0, NSE_FP64 = 0, NSE_MIXED = 1
  integer(c_int), parameter :: NSE_FLAG_CHECK_FINITE = 1, NSE_FLAG_EXACT = 4
  integer(c_int), parameter :: NSE_U = 0, NSE_V = 1, NSE_W = 2, NSE_P = 3, NSE_T = 4, &
       NSE_U_TA = 5, NSE_V_TA = 6, NSE_W_TA = 7, NSE_U_PRE = 8, NSE_V_PRE = 9, &
       NSE_W_PRE = 10, NSE_T_PRE = 11, NSE_DIVU = 12, NSE_U_EP2 = 13, NSE_V_EP2 = 14, &
       NSE_W_EP2 = 15, NSE_PHI = 16, NSE_CELLVALUE = 17

  type, bind(C) :: nse_adjoint_config
     integer(c_int) :: nsteps, checkpoint_every, avg_from
  end type nse_adjoint_config

  type, bind(C) :: nse_config
     integer(c_int) :: nx, ny, nz
     real(c_double) :: dt, Re, Sc, eta
     real(c_double) :: xl, yl, zl
     real(c_double) :: y0, ystretch
     real(c_double) :: body_force, heat_source
     real(c_double) :: t_bot, t_top, t_solid
     real(c_double) :: rho_cp, thc
     integer(c_int) :: precision, flags
  end type nse_config

  interface
     integer(c_int) function nse_ctx_create(cfg, ctx) bind(C, name="nse_ctx_create")
       import :: c_int, c_ptr, nse_config
       type(nse_config), intent(in) :: cfg
       type(c_ptr), intent(out) :: ctx
     end function nse_ctx_create
     integer(c_int) function nse_ctx_destroy(ctx) bind(C, name="nse_ctx_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function nse_ctx_destroy
     integer(c_int) function nse_ctx_upload(ctx, field, host) bind(C, name="nse_ctx_upload")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: field
       real(c_double), intent(in) :: host(*)
     end function nse_ctx_upload
     integer(c_int) function nse_ctx_download(ctx, field, host) bind(C, name="nse_ctx_download")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: field
       real(c_double), intent(out) :: host(*)
     end function nse_ctx_download
     integer(c_int) function nse_ctx_set_step(ctx, l) bind(C, name="nse_ctx_set_step")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: l
     end function nse_ctx_set_step
     integer(c_int) function nse_start(ctx) bind(C, name="nse_start")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function nse_start
     integer(c_int) function nse_step(ctx, nsteps) bind(C, name="nse_step")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: nsteps
     end function nse_step
     integer(c_int) function nse_project(ctx) bind(C, name="nse_project")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function nse_project
     integer(c_int) function nse_levelset(ctx, phi0, phi_out, nnn, dtau, width) &
          bind(C, name="nse_levelset")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: phi0(*)
       type(c_ptr), value :: phi_out
       integer(c_int), value :: nnn
       real(c_double), value :: dtau, width
     end function nse_levelset
     integer(c_int) function nse_monitor(ctx, out) bind(C, name="nse_monitor")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: out(6)
     end function nse_monitor
     integer(c_int) function nse_sync(ctx) bind(C, name="nse_sync")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function nse_sync
     integer(c_int) function nse_adjoint_create(ctx, cfg, adj) bind(C, name="nse_adjoint_create")
       import :: c_int, c_ptr, nse_adjoint_config
       type(c_ptr), value :: ctx
       type(nse_adjoint_config), intent(in) :: cfg
       type(c_ptr), intent(out) :: adj
     end function nse_adjoint_create
     integer(c_int) function nse_adjoint_gradient(adj, J, grad_c1) &
          bind(C, name="nse_adjoint_gradient")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: adj
       real(c_double), intent(out) :: J
       real(c_double), intent(out) :: grad_c1(*)
     end function nse_adjoint_gradient
     integer(c_int) function nse_adjoint_objective(adj, J) bind(C, name="nse_adjoint_objective")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: adj
       real(c_double), intent(out) :: J
     end function nse_adjoint_objective
     integer(c_int) function nse_adjoint_destroy(adj) bind(C, name="nse_adjoint_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: adj
     end function nse_adjoint_destroy
     type(c_ptr) function nse_last_error() bind(C, name="nse_last_error")
       import :: c_ptr
     end function nse_last_error
     subroutine nse_set_alloc_limit(bytes) bind(C, name="nse_set_alloc_limit")
       import :: c_long_long
       integer(c_long_long), value :: bytes
     end subroutine nse_set_alloc_limit
  end interface
end module nsegpu
