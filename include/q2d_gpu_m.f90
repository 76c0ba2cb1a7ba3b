! q2d_gpu_m.f90 — ISO_C_BINDING interface of the B200 explicit residual / time-update path
! (include/q2d_gpu.h) for the Q2D Fortran host.
!
! A Q2D host adds this module (for instance as src/lib/gpu/q2d_gpu_m.f90) and links with
! -L<repo>/q2d_b200/lib -lq2d_gpu. One q2d_gpu_step call replaces the body of Explicit_Step
! (src/lib/numerics/time/explicit/Mod_Explicit.f90:10-174) for one grid level; the option
! fields mirror the [Q2D-Numerics] / [Q2D-Parameters] / [Q2D-IO] / [Q2D-Sources] keys
! (Register_Numerics.f90:31-76, Register_Sim_Param.f90:26-29, Register_IO.f90:26-35) and the bc
! records mirror bc.txt (IO_BC.f90:209-402). The derived types below follow the C structs of
! q2d_gpu.h field by field (tests/test_fortran_module.py checks their order and kinds against
! the ctypes mirror of the header).
!
! Argument conventions: `nodes` is node(0:ni,0:nj)%c(1:2) flattened (x, y per node, i
! fastest); `area` is c_loc(Cross_Section) or c_null_ptr; `P` is the host's own
! blk(b)%P(1:4, -1:ni+2, -1:nj+2) passed as is; bc records keep their 1-based indices, with
! alpha = huge(1.0_c_double) for the `normal` keyword. Every function returns a Q2D_* status.
module q2d_gpu_m
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: Q2D_OK = 0, Q2D_ERR_BADARG = 1, Q2D_ERR_OOM = 2, Q2D_ERR_CUDA = 3
  integer(c_int), parameter :: Q2D_ERR_NONPHYSICAL = 4, Q2D_ERR_NAN = 5, Q2D_ERR_TIMEOUT = 6
  integer(c_int), parameter :: Q2D_ERR_UNSUPPORTED = 7, Q2D_ERR_CAPACITY = 8
  integer(c_int), parameter :: Q2D_TODO_CONTINUE = 1, Q2D_TODO_IO = 2, Q2D_TODO_END = 3
  integer(c_int), parameter :: Q2D_PREC_FP64 = 0, Q2D_PREC_FP32_FLUX = 1
  integer(c_int), parameter :: Q2D_SRC_NONE = 0, Q2D_SRC_AXI = 1, Q2D_SRC_AREA = 2
  integer(c_int), parameter :: Q2D_NOALLOC_MAX_PARTIALS = 8192, Q2D_NOALLOC_CELLS_PER_PARTIAL = 2048

  type, bind(c) :: q2d_options
    integer(c_int) :: limiter            ! flux-limiter (Q2D_LIM_*)
    integer(c_int) :: riemann            ! riemann-solver (Q2D_RIEMANN_*)
    integer(c_int) :: n_rk               ! time-scheme: 1 euler, 2 RK2, 3 RK3
    integer(c_int) :: time_accurate      ! time-accurate
    integer(c_int) :: source             ! [Q2D-Sources] active
    integer(c_int) :: precision          ! Q2D_PREC_*
    integer(c_int) :: rampa_iter         ! cfl-rise-threshold
    integer(c_int) :: res_diter          ! res-diter
    integer(c_int) :: sol_diter          ! sol-diter
    integer(c_int) :: res_relative       ! 0: absolute res-threshold; 1: drop from the first step
    integer(c_long_long) :: itermax      ! iter-threshold
    real(c_double) :: cfl                ! cfl
    real(c_double) :: res_threshold      ! res-threshold
    real(c_double) :: time_threshold     ! time-threshold
    real(c_double) :: sol_dtime          ! sol-dtime
    real(c_double) :: gas_R              ! gas constant of the phase
    real(c_double) :: gas_gamma          ! ratio of specific heats
    real(c_double) :: irs_beta           ! irs-beta; smoothing when > 0
    integer(c_int) :: shock_detector     ! MUSCL-SD: 1 or 0
    real(c_double) :: riemann_minf       ! riemann-options-Minf (AUSM+-up, AUSM+-up2)
  end type q2d_options

  type, bind(c) :: q2d_bc_rec
    integer(c_int) :: b, i, j, f, type   ! bc.txt header
    integer(c_int) :: bs, is, js, fs     ! 101 / 201: donor block, cell and face
    integer(c_int) :: d11, d12, d21, d22 ! 101 / 201: index orientation
    real(c_double) :: T0, p0, pamb, mach, alpha, rel_fac   ! 401 / 405 / 406 properties
  end type q2d_bc_rec

  type, bind(c) :: q2d_step_info
    real(c_double) :: dtglobal
    real(c_double) :: time
    integer(c_long_long) :: iter
    real(c_double) :: residual(4)
    real(c_double) :: residual0
    integer(c_int) :: todo
    integer(c_int) :: err
    integer(c_int) :: err_b, err_i, err_j, err_stage
  end type q2d_step_info

  interface
    subroutine q2d_options_default(o) bind(c)
      import; type(q2d_options), intent(out) :: o
    end subroutine
    integer(c_int) function q2d_gpu_create(ctx, o) bind(c)
      import; type(c_ptr), intent(out) :: ctx; type(q2d_options), intent(in) :: o
    end function
    integer(c_int) function q2d_gpu_add_case(ctx, case_id) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), intent(out) :: case_id
    end function
    integer(c_int) function q2d_gpu_add_block(ctx, case_id, ni, nj, nodes, area, block_id) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id, ni, nj
      real(c_double), intent(in) :: nodes(*); type(c_ptr), value :: area
      integer(c_int), intent(out) :: block_id
    end function
    integer(c_int) function q2d_gpu_set_bcs(ctx, case_id, recs, n) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id, n
      type(q2d_bc_rec), intent(in) :: recs(*)
    end function
    integer(c_int) function q2d_gpu_upload_prim(ctx, block_id, P) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: block_id
      real(c_double), intent(in) :: P(*)
    end function
    integer(c_int) function q2d_gpu_set_case_time(ctx, case_id, time) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id
      real(c_double), value :: time
    end function
    integer(c_int) function q2d_gpu_set_thermo_table(ctx, ntab, h_tab, cp_tab) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: ntab
      real(c_double), intent(in) :: h_tab(*), cp_tab(*)
    end function
    integer(c_int) function q2d_gpu_set_case_end(ctx, case_id, iter_end) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id
      integer(c_long_long), value :: iter_end
    end function
    integer(c_int) function q2d_gpu_commit(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function q2d_gpu_step(ctx, nsteps, info) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nsteps
      type(q2d_step_info), intent(out) :: info(*)
    end function
    integer(c_int) function q2d_gpu_step_async(ctx, nsteps) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nsteps
    end function
    integer(c_int) function q2d_gpu_wait(ctx, info) bind(c)
      import; type(c_ptr), value :: ctx; type(q2d_step_info), intent(out) :: info(*)
    end function
    integer(c_int) function q2d_gpu_prepare(ctx, nsteps) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nsteps
    end function
    integer(c_int) function q2d_gpu_autotune(ctx, steps, schedule, ms_per_step) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: steps
      integer(c_int), intent(out) :: schedule; real(c_float), intent(out) :: ms_per_step
    end function
    integer(c_int) function q2d_gpu_set_schedule(ctx, schedule) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: schedule
    end function
    integer(c_int) function q2d_gpu_get_schedule(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function q2d_gpu_residual_norm_noalloc(p_new, p_old, ncells, plane_stride, norms_out, &
                                                          stream) bind(c)
      import; type(c_ptr), value :: p_new, p_old, norms_out, stream
      integer(c_long_long), value :: ncells, plane_stride
    end function
    type(c_ptr) function q2d_gpu_stream(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function q2d_gpu_case_info(ctx, case_id, info) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id
      type(q2d_step_info), intent(out) :: info
    end function
    integer(c_int) function q2d_gpu_download_prim(ctx, block_id, P) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: block_id
      real(c_double), intent(inout) :: P(*)
    end function
    integer(c_int) function q2d_gpu_upload_prim_many(ctx, n, ids, P) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: n
      integer(c_int), intent(in) :: ids(*); type(c_ptr), intent(in) :: P(*)   ! c_loc(blk(b)%P)
    end function
    integer(c_int) function q2d_gpu_download_prim_many(ctx, n, ids, P) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: n
      integer(c_int), intent(in) :: ids(*); type(c_ptr), intent(in) :: P(*)   ! c_loc(blk(b)%P)
    end function
    integer(c_int) function q2d_gpu_num_cases(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_long_long) function q2d_gpu_num_cells(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function q2d_serve_create(ctx, o, device_bytes, max_cases) bind(c)
      import; type(c_ptr), intent(out) :: ctx; type(q2d_options), intent(in) :: o
      integer(c_long_long), value :: device_bytes; integer(c_int), value :: max_cases
    end function
    integer(c_int) function q2d_serve_admit(ctx, nblocks, ni, nj, nodes, areas, P, recs, nrecs, case_id) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nblocks, nrecs
      integer(c_int), intent(in) :: ni(*), nj(*)
      type(c_ptr), intent(in) :: nodes(*), areas(*), P(*)
      type(q2d_bc_rec), intent(in) :: recs(*); integer(c_int), intent(out) :: case_id
    end function
    integer(c_int) function q2d_serve_retire(ctx, case_id) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id
    end function
    integer(c_int) function q2d_serve_block_id(ctx, case_id, b, block_id) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: case_id, b
      integer(c_int), intent(out) :: block_id
    end function
    integer(c_long_long) function q2d_serve_free_cells(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_long_long) function q2d_gpu_launch_count(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    type(c_ptr) function q2d_gpu_errstr(status) bind(c)
      import; integer(c_int), value :: status
    end function
    type(c_ptr) function q2d_gpu_last_error(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    subroutine q2d_gpu_destroy(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end subroutine
  end interface
end module q2d_gpu_m
