! evolve_gpu.f90 -- ISO_C_BINDING interface of libechogpu.so for the
! ECHO-QGP Fortran host.  With -DECHO_GPU the bodies of evolve_main,
! evolve_alloc and the state hand-over around output call these bindings
! (see INTEGRATION.md for the exact edits of evolve.f90 and echo.f90).
!
! All arrays are passed as they are: v(ix1:ix2,iy1:iy2,iz1:iz2,nv) and u(...)
! are column-major with x fastest and the variable index slowest, the layout
! the library expects.  This file is not compiled in this repository (no
! Fortran compiler is available here); it is the binding a maintainer adds.
module evolve_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: ECHO_MAX_NV = 16

  type, bind(C) :: echo_params
    integer(c_int) :: nx, ny, nz
    real(c_double) :: x1, x2, y1, y2, z1, z2
    integer(c_int) :: coordinates, mhd, divclean, viscosity, bulkvis
    integer(c_int) :: recal, nrk, eqstate, algo_solver, obtained_zz
    integer(c_int) :: init_type, enable_smooth_viscosity
    integer(c_int) :: ibc(3, 2, ECHO_MAX_NV)   ! C int ibc[16][2][3]
    real(c_double) :: cfl, maxdt, maxspeed, glm_alpha, eta_over_s
    real(c_double) :: tau_pi_coeff, smooth_pressure, enezero, przero, c2p_tol
    integer(c_int) :: imex   ! this library's implicit Israel-Stewart relaxation; set 0 for the reference's explicit
    real(c_double) :: sigma_el, sigma_chiral   ! sigma_el_cond, sigma_chiral_cond (resistive runs)
  end type echo_params

  type(c_ptr), save :: echo_ctx = c_null_ptr

  interface
    integer(c_int) function echo_gpu_init(p, eos_table, n_eos, ctx) bind(C, name="echo_gpu_init")
      import :: c_int, c_ptr, c_double, echo_params
      type(echo_params), intent(in) :: p
      real(c_double), intent(in) :: eos_table(*)
      integer(c_int), value :: n_eos
      type(c_ptr), intent(out) :: ctx
    end function

    integer(c_int) function echo_gpu_upload(ctx, v, u, t) bind(C, name="echo_gpu_upload")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: v(*), u(*)
      real(c_double), value :: t
    end function

    integer(c_int) function echo_gpu_download(ctx, v, u) bind(C, name="echo_gpu_download")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: v(*), u(*)
    end function

    integer(c_int) function echo_gpu_set_tout(ctx, tout) bind(C, name="echo_gpu_set_tout")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tout
    end function

    integer(c_int) function echo_gpu_evolve_main(ctx, irk, dt, errcode) bind(C, name="echo_gpu_evolve_main")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: irk
      real(c_double), intent(out) :: dt
      integer(c_int), intent(out) :: errcode
    end function

    integer(c_int) function echo_gpu_end_step(ctx) bind(C, name="echo_gpu_end_step")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function echo_gpu_free(ctx) bind(C, name="echo_gpu_free")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    ! learned con2prim seed (ALG_SOLV = 101): weights(ECHO_MLP_NWEIGHTS) and
    ! norm(ECHO_MLP_NNORM) as echo_gpu_mlp_train writes them; before the
    ! first evolve_main
    integer(c_int) function echo_gpu_mlp_set(ctx, weights, norm) bind(C, name="echo_gpu_mlp_set")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: weights(*), norm(*)
    end function
  end interface

contains

  ! evolve_main(irk, dt) of evolve.f90:114 on the device: same arguments,
  ! run_crashed set exactly when the reference would set it
  subroutine evolve_main_gpu(irk, dt, run_crashed, errcode)
    integer, intent(in) :: irk
    real(8), intent(out) :: dt
    logical, intent(inout) :: run_crashed
    integer, intent(out) :: errcode
    integer(c_int) :: st, code
    real(c_double) :: dtc
    st = echo_gpu_evolve_main(echo_ctx, int(irk, c_int), dtc, code)
    if (st /= 0) then
      write(*,*) 'echo_gpu_evolve_main: library status ', st
      stop 2
    end if
    dt = dtc
    errcode = code
    if (code /= 0) run_crashed = .true.
  end subroutine evolve_main_gpu

end module evolve_gpu
