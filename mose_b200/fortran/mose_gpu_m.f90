!> ISO_C_BINDING interface to libmose_gpu.so (include/mose_gpu.h).
!>
!> MOSE's explicit driver calls these in place of Compute_dt, Set_Global_dt,
!> Copy_State, Fill_Ghost_Cell, Fluxes + BC_Fluxes, RK_Newstate and
!> Compute_Residual (src/lib/numerics/time/explicit/Mod_Explicit.f90:40-113).
!> Arrays keep the reference layouts: node(3,0:ni,0:nj,0:nk),
!> P(nprim,1-gc:ni+gc,1-gc:nj+gc,1-gc:nk+gc); bc records are the parsed
!> bc.txt lines.
module mose_gpu_m
  use iso_c_binding
  implicit none
  private

  integer(c_int32_t), parameter, public :: MOSE_GPU_ABI_VERSION = 1
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
  public :: mose_gpu_add_block, mose_gpu_set_bcs, mose_gpu_add_series, mose_gpu_setup
  public :: mose_gpu_upload_prim, mose_gpu_download_prim, mose_gpu_download_residual, mose_gpu_upload_residual
  public :: mose_gpu_compute_dt, mose_gpu_set_global_dt, mose_gpu_copy_state, mose_gpu_fill_ghosts
  public :: mose_gpu_residual, mose_gpu_rk_stage, mose_gpu_step, mose_gpu_residual_norms
  public :: mose_gpu_set_time, mose_gpu_synchronize

  interface
    subroutine mose_gpu_default_config(cfg) bind(C, name="mose_gpu_default_config")
      import :: mose_gpu_config
      type(mose_gpu_config), intent(out) :: cfg
    end subroutine
    integer(c_int) function mose_gpu_create(cfg, ctx) bind(C, name="mose_gpu_create")
      import :: mose_gpu_config, c_int, c_ptr
      type(mose_gpu_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: ctx
    end function
    subroutine mose_gpu_destroy(ctx) bind(C, name="mose_gpu_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine
    type(c_ptr) function mose_gpu_last_error(ctx) bind(C, name="mose_gpu_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function mose_gpu_add_block(ctx, b, ni, nj, nk, node) bind(C, name="mose_gpu_add_block")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b, ni, nj, nk
      real(c_double), intent(in) :: node(*)
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
      real(c_double), intent(in) :: time(*), val(*)
      integer(c_int32_t), value :: n, periodic
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
      real(c_double), intent(inout) :: P(*)
    end function
    integer(c_int) function mose_gpu_download_residual(ctx, b, R) bind(C, name="mose_gpu_download_residual")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(inout) :: R(*)
    end function
    integer(c_int) function mose_gpu_upload_residual(ctx, b, R) bind(C, name="mose_gpu_upload_residual")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: b
      real(c_double), intent(in) :: R(*)
    end function
    integer(c_int) function mose_gpu_compute_dt(ctx, cfl, iter, ramp, dtglobal) bind(C, name="mose_gpu_compute_dt")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: cfl
      integer(c_int32_t), value :: iter, ramp
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
      real(c_double), intent(out) :: dtglobal, time
    end function
    integer(c_int) function mose_gpu_residual_norms(ctx, total) bind(C, name="mose_gpu_residual_norms")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: total(5)
    end function
    integer(c_int) function mose_gpu_set_time(ctx, time, iter) bind(C, name="mose_gpu_set_time")
      import :: c_ptr, c_int, c_int32_t, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: time
      integer(c_int32_t), value :: iter
    end function
    integer(c_int) function mose_gpu_synchronize(ctx) bind(C, name="mose_gpu_synchronize")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
  end interface

end module mose_gpu_m
