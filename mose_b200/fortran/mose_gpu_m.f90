!> ISO_C_BINDING interface to libmose_gpu.so (include/mose_gpu.h).
!>
!> MOSE's explicit driver calls these in place of Compute_dt, Set_Global_dt,
!> Copy_State, Fill_Ghost_Cell, Fluxes + BC_Fluxes, RK_Newstate and
!> Compute_Residual (src/lib/numerics/time/explicit/Mod_Explicit.f90:40-113).
!> Arrays keep the reference layouts: node(3,0:ni,0:nj,0:nk),
!> P(nprim,1-gc:ni+gc,1-gc:nj+gc,1-gc:nk+gc); bc records are the parsed
!> bc.txt lines.  Every entry point of include/mose_gpu.h has an interface
!> here, in the header's order; scalars passed by value in C are VALUE
!> arguments, pointers are arrays or INTENT(OUT) scalars, the context and
!> device addresses are TYPE(C_PTR).  Strings come back as C pointers
!> (mose_gpu_last_error): convert them with C_F_POINTER.
module mose_gpu_m
  use iso_c_binding
  implicit none
  private

  integer(c_int32_t), parameter, public :: MOSE_GPU_ABI_VERSION = 2
  integer(c_int), parameter, public :: MOSE_OK = 0

  type, bind(C), public :: mose_gpu_config
    integer(c_int32_t) :: abi_version
    integer(c_int32_t) :: n_rk
    real(c_double)     :: cfl
    integer(c_int32_t) :: time_accurate
    integer(c_int32_t) :: ramp_iter
    integer(c_int32_t) :: limiter
    integer(c_int32_t) :: riemann
    integer(c_int32_t) :: integration
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: ndir
    integer(c_int32_t) :: nsc
    real(c_double)     :: gamma
    real(c_double)     :: rgas
    integer(c_int32_t) :: device
    integer(c_int32_t) :: res_diter
  end type mose_gpu_config

  public :: mose_gpu_default_config, mose_gpu_create, mose_gpu_destroy, mose_gpu_last_error
  public :: mose_gpu_error_location, mose_gpu_add_block, mose_gpu_set_bcs, mose_gpu_add_series
  public :: mose_gpu_setup, mose_gpu_upload_prim, mose_gpu_download_prim, mose_gpu_upload_prim_old
  public :: mose_gpu_download_residual, mose_gpu_upload_residual, mose_gpu_download_dt, mose_gpu_upload_dt
  public :: mose_gpu_compute_dt, mose_gpu_set_global_dt, mose_gpu_copy_state, mose_gpu_fill_ghosts
  public :: mose_gpu_residual, mose_gpu_rk_stage, mose_gpu_step, mose_gpu_advance, mose_gpu_residual_norms
  public :: mose_gpu_residual_norms_noalloc, mose_gpu_noalloc_last_error, mose_gpu_set_time
  public :: mose_gpu_get_time, mose_gpu_synchronize, mose_gpu_stream, mose_gpu_time_kernels
  public :: mose_gpu_uniform_metrics, mose_gpu_launch_count, mose_gpu_download_metrics
  public :: mose_gpu_download_faces, mose_gpu_check_fast_math, mose_gpu_set_sd_limiter, mose_gpu_set_irs_beta
  public :: mose_gpu_set_viscous, mose_gpu_set_riemann_minf, mose_gpu_set_tiling, mose_gpu_get_tiling
  public :: mose_gpu_autotune, mose_gpu_set_inflow_mach, mose_gpu_adjoint_forward, mose_gpu_adjoint_backward
  public :: mose_gpu_adjoint_step, mose_gpu_upload_adjoint, mose_gpu_download_adjoint

  interface
    subroutine mose_gpu_default_config(cfg) bind(C, name="mose_gpu_default_config")
      import :: mose_gpu_config
      type(mose_gpu_config), intent(out) :: cfg
    end subroutine
    integer(c_int) function mose_gpu_create(cfg, out) bind(C, name="mose_gpu_create")
      import :: mose_gpu_config, c_ptr, c_int
      type(mose_gpu_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: out
    end function
    subroutine mose_gpu_destroy(ctx) bind(C, name="mose_gpu_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine
    type(c_ptr) function mose_gpu_last_error(ctx) bind(C, name="mose_gpu_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_error_location(ctx, b, i, j, k) bind(C, name="mose_gpu_error_location")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: b
      integer(c_int32_t), intent(out) :: i
      integer(c_int32_t), intent(out) :: j
      integer(c_int32_t), intent(out) :: k
    end function
    ! metrics: c_loc of the packed Setup_Metrics arrays (layout in mose_gpu.h),
    ! or c_null_ptr to form them on the device from the nodes
    integer(c_int) function mose_gpu_add_block(ctx, b, ni, nj, nk, node, metrics) bind(C, name="mose_gpu_add_block")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      integer(c_int32_t), value :: ni
      integer(c_int32_t), value :: nj
      integer(c_int32_t), value :: nk
      real(c_double), intent(in) :: node(*)
      type(c_ptr), value :: metrics
    end function
    integer(c_int) function mose_gpu_set_bcs(ctx, rec, dat, nbound) bind(C, name="mose_gpu_set_bcs")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: rec(15, *)
      real(c_double), intent(in) :: dat(6, *)
      integer(c_int32_t), value :: nbound
    end function
    integer(c_int) function mose_gpu_add_series(ctx, time, val, n, periodic, id) bind(C, name="mose_gpu_add_series")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: time
      real(c_double), intent(in) :: val(*)
      integer(c_int32_t), value :: n
      integer(c_int32_t), value :: periodic
      integer(c_int32_t), intent(out) :: id
    end function
    integer(c_int) function mose_gpu_setup(ctx) bind(C, name="mose_gpu_setup")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_upload_prim(ctx, b, P) bind(C, name="mose_gpu_upload_prim")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(in) :: P(*)
    end function
    integer(c_int) function mose_gpu_download_prim(ctx, b, P) bind(C, name="mose_gpu_download_prim")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(out) :: P(*)
    end function
    integer(c_int) function mose_gpu_upload_prim_old(ctx, b, PO) bind(C, name="mose_gpu_upload_prim_old")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(in) :: PO(*)
    end function
    integer(c_int) function mose_gpu_download_residual(ctx, b, R) bind(C, name="mose_gpu_download_residual")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(out) :: R(*)
    end function
    integer(c_int) function mose_gpu_upload_residual(ctx, b, R) bind(C, name="mose_gpu_upload_residual")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(in) :: R(*)
    end function
    integer(c_int) function mose_gpu_download_dt(ctx, b, dt) bind(C, name="mose_gpu_download_dt")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(out) :: dt(*)
    end function
    integer(c_int) function mose_gpu_upload_dt(ctx, b, dt) bind(C, name="mose_gpu_upload_dt")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(in) :: dt(*)
    end function
    integer(c_int) function mose_gpu_compute_dt(ctx, cfl, iter, ramp_iter, dtglobal) bind(C, name="mose_gpu_compute_dt")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: cfl
      integer(c_int32_t), value :: iter
      integer(c_int32_t), value :: ramp_iter
      real(c_double), intent(inout) :: dtglobal
    end function
    integer(c_int) function mose_gpu_set_global_dt(ctx, dtglobal) bind(C, name="mose_gpu_set_global_dt")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: dtglobal
    end function
    integer(c_int) function mose_gpu_copy_state(ctx) bind(C, name="mose_gpu_copy_state")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_fill_ghosts(ctx) bind(C, name="mose_gpu_fill_ghosts")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_residual(ctx) bind(C, name="mose_gpu_residual")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_rk_stage(ctx, irk) bind(C, name="mose_gpu_rk_stage")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: irk
    end function
    integer(c_int) function mose_gpu_step(ctx, dtglobal, time) bind(C, name="mose_gpu_step")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: dtglobal
      real(c_double), intent(out) :: time
    end function
    integer(c_int) function mose_gpu_advance(ctx, nsteps, dtglobal, time) bind(C, name="mose_gpu_advance")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsteps
      real(c_double), intent(inout) :: dtglobal
      real(c_double), intent(out) :: time
    end function
    integer(c_int) function mose_gpu_residual_norms(ctx, total) bind(C, name="mose_gpu_residual_norms")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: total(5)
    end function
    integer(c_int) function mose_gpu_residual_norms_noalloc(P, PO, ni, nj, nk, total, stream) &
        bind(C, name="mose_gpu_residual_norms_noalloc")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: P, PO          ! device addresses (reference layout of one block)
      integer(c_int32_t), value :: ni
      integer(c_int32_t), value :: nj
      integer(c_int32_t), value :: nk
      type(c_ptr), value :: total          ! device address of 5 doubles
      type(c_ptr), value :: stream
    end function
    type(c_ptr) function mose_gpu_noalloc_last_error() bind(C, name="mose_gpu_noalloc_last_error")
      import :: c_ptr
    end function
    integer(c_int) function mose_gpu_set_time(ctx, time, iter) bind(C, name="mose_gpu_set_time")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: time
      integer(c_int32_t), value :: iter
    end function
    integer(c_int) function mose_gpu_get_time(ctx, time, iter) bind(C, name="mose_gpu_get_time")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: time
      integer(c_int32_t), intent(out) :: iter
    end function
    integer(c_int) function mose_gpu_synchronize(ctx) bind(C, name="mose_gpu_synchronize")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function mose_gpu_stream(ctx) bind(C, name="mose_gpu_stream")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_time_kernels(ctx, nsteps, ms, launches) bind(C, name="mose_gpu_time_kernels")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsteps
      real(c_double), intent(out) :: ms(3)
      integer(c_int32_t), intent(out) :: launches(3)
    end function
    integer(c_int) function mose_gpu_uniform_metrics(ctx) bind(C, name="mose_gpu_uniform_metrics")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    integer(c_int64_t) function mose_gpu_launch_count(ctx) bind(C, name="mose_gpu_launch_count")
      import :: c_ptr, c_int64_t
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_download_metrics(ctx, b, vol, dl) bind(C, name="mose_gpu_download_metrics")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(out) :: vol(*)
      real(c_double), intent(out) :: dl(*)
    end function
    integer(c_int) function mose_gpu_download_faces(ctx, b, dir, N, A) bind(C, name="mose_gpu_download_faces")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      integer(c_int32_t), value :: dir
      real(c_double), intent(out) :: N(*)
      real(c_double), intent(out) :: A(*)
    end function
    integer(c_int) function mose_gpu_check_fast_math(n, seed, out) bind(C, name="mose_gpu_check_fast_math")
      import :: c_int, c_int64_t, c_double
      integer(c_int64_t), value :: n
      integer(c_int64_t), value :: seed
      real(c_double), intent(out) :: out(*)
    end function
    integer(c_int) function mose_gpu_set_sd_limiter(ctx, on) bind(C, name="mose_gpu_set_sd_limiter")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: on
    end function
    integer(c_int) function mose_gpu_set_irs_beta(ctx, beta) bind(C, name="mose_gpu_set_irs_beta")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: beta
    end function
    integer(c_int) function mose_gpu_set_viscous(ctx, model, mu, kappa, vnn) bind(C, name="mose_gpu_set_viscous")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: model
      real(c_double), value :: mu
      real(c_double), value :: kappa
      real(c_double), value :: vnn
    end function
    integer(c_int) function mose_gpu_set_riemann_minf(ctx, minf) bind(C, name="mose_gpu_set_riemann_minf")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: minf
    end function
    integer(c_int) function mose_gpu_set_tiling(ctx, tiling) bind(C, name="mose_gpu_set_tiling")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: tiling(4)
    end function
    integer(c_int) function mose_gpu_get_tiling(ctx, tiling) bind(C, name="mose_gpu_get_tiling")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: tiling(4)
    end function
    integer(c_int) function mose_gpu_autotune(ctx, steps, tiling_out, best_ms_per_step, default_ms_per_step) &
        bind(C, name="mose_gpu_autotune")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: steps
      integer(c_int32_t), intent(out) :: tiling_out(4)
      real(c_double), intent(out) :: best_ms_per_step
      real(c_double), intent(out) :: default_ms_per_step
    end function
    integer(c_int) function mose_gpu_set_inflow_mach(ctx, mach) bind(C, name="mose_gpu_set_inflow_mach")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: mach
    end function
    integer(c_int) function mose_gpu_adjoint_forward(ctx, nsteps, interval, block, face, J) &
        bind(C, name="mose_gpu_adjoint_forward")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), value :: interval
      integer(c_int32_t), value :: block
      integer(c_int32_t), value :: face
      real(c_double), intent(out) :: J
    end function
    integer(c_int) function mose_gpu_adjoint_backward(ctx, dJ_dmach) bind(C, name="mose_gpu_adjoint_backward")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: dJ_dmach
    end function
    integer(c_int) function mose_gpu_adjoint_step(ctx, dJ_dmach) bind(C, name="mose_gpu_adjoint_step")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: dJ_dmach
    end function
    integer(c_int) function mose_gpu_upload_adjoint(ctx, b, lam) bind(C, name="mose_gpu_upload_adjoint")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(in) :: lam(*)
    end function
    integer(c_int) function mose_gpu_download_adjoint(ctx, b, lam) bind(C, name="mose_gpu_download_adjoint")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(out) :: lam(*)
    end function
  end interface

end module mose_gpu_m
