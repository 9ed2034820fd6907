! evolve_gpu.f90 -- ISO_C_BINDING interface of libechogpu.so for the
! ECHO-QGP Fortran host.  With -DECHO_GPU the bodies of evolve_main,
! evolve_alloc and the state hand-over around output call these bindings;
! the per-step work of echo.f90 around them (check_temp, out_vars, out_hyp,
! out_dump/out_restart) has device counterparts bound below as well.
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

  ! init()'s GLAUBER_GEOMETRIC parameters (echo_gpu_optical_glauber)
  type, bind(C) :: echo_optical_glauber
    real(c_double) :: mass_number, radius, delta, roze   ! projmass, radius, delta, roze of nuclear_data.dat
    real(c_double) :: sigma_in                           ! fm^2 (SIGMA_IN/10)
    real(c_double) :: ah, bimpact, ecenter, rhocenter
    real(c_double) :: dr, dz1, acc                       ! thickness table steps and accuracy
    real(c_double) :: deta, sigeta                       ! 3+1D plateau and Gaussian width of H(eta)
    real(c_double) :: sqrt_s, nucleon_mass               ! gamma_col = sqrt_s / (2 m)
  end type echo_optical_glauber

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

    ! check_temp (out.f90:1487-1557) on the device: max_value = the grid
    ! maximum of T (freeze_type 0) or e (1); stop = 1 when it is below temp_end
    integer(c_int) function echo_gpu_check_temp(ctx, freeze_type, temp_end, max_value, stop_flag) &
        bind(C, name="echo_gpu_check_temp")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: freeze_type
      real(c_double), value :: temp_end
      real(c_double), intent(out) :: max_value
      integer(c_int), intent(out) :: stop_flag
    end function

    ! out_vars (out.f90:232-591): the bytes of one outNNNN.dat (t, then the
    ! selected fields), precision 8 or 4; sel is a mask of ECHO_OUT_* bits
    integer(c_int) function echo_gpu_out_vars_size(ctx, sel, precision, nbytes) &
        bind(C, name="echo_gpu_out_vars_size")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: sel          ! C unsigned: the low 27 bits are used
      integer(c_int), value :: precision
      integer(c_size_t), intent(out) :: nbytes
    end function

    integer(c_int) function echo_gpu_out_vars(ctx, sel, precision, buf, nbytes, errcode) &
        bind(C, name="echo_gpu_out_vars")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: sel
      integer(c_int), value :: precision
      type(c_ptr), value :: buf             ! c_loc of an integer(1) buffer of nbytes
      integer(c_size_t), value :: nbytes
      integer(c_int), intent(out) :: errcode
    end function

    ! out_hyp (out.f90:1569-1650): hyp_init once, hyp_step at every
    ! hypersurface time, hyp_get for the n_elements rows of 8 + nv doubles
    integer(c_int) function echo_gpu_hyp_init(ctx, freeze_type, freeze_value) bind(C, name="echo_gpu_hyp_init")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: freeze_type
      real(c_double), value :: freeze_value
    end function

    integer(c_int) function echo_gpu_hyp_step(ctx, n_elements, errcode) bind(C, name="echo_gpu_hyp_step")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: n_elements
      integer(c_int), intent(out) :: errcode
    end function

    integer(c_int) function echo_gpu_hyp_get(ctx, elements) bind(C, name="echo_gpu_hyp_get")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: elements(*)   ! (8 + nv) * n_elements
    end function

    ! out_dump / out_restart (out.f90:1313-1483): the run state at a step
    ! boundary as one blob of checkpoint_size bytes
    integer(c_int) function echo_gpu_checkpoint_size(ctx, nbytes) bind(C, name="echo_gpu_checkpoint_size")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      integer(c_size_t), intent(out) :: nbytes
    end function

    integer(c_int) function echo_gpu_checkpoint(ctx, blob) bind(C, name="echo_gpu_checkpoint")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr), value :: blob            ! c_loc of an integer(1) buffer
    end function

    integer(c_int) function echo_gpu_restart(ctx, blob) bind(C, name="echo_gpu_restart")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr), value :: blob
    end function

    ! dump.dat in the reference's own layout (out_dump / out_restart):
    ! keep_old(1) once after the upload makes vold/uold complete; dump fills
    ! a buffer of dump_size bytes that the host writes to outrNNNN/dump.dat
    integer(c_int) function echo_gpu_keep_old(ctx, on) bind(C, name="echo_gpu_keep_old")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: on
    end function

    integer(c_int) function echo_gpu_dump_size(ctx, nbytes) bind(C, name="echo_gpu_dump_size")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      integer(c_size_t), intent(out) :: nbytes
    end function

    integer(c_int) function echo_gpu_dump(ctx, iout, buf, nbytes) bind(C, name="echo_gpu_dump")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: iout
      type(c_ptr), value :: buf
      integer(c_size_t), value :: nbytes
    end function

    integer(c_int) function echo_gpu_restart_dump(ctx, buf, nbytes, iout) bind(C, name="echo_gpu_restart_dump")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      type(c_ptr), value :: buf
      integer(c_size_t), value :: nbytes
      integer(c_int), intent(out) :: iout
    end function

    ! init()'s optical Glauber branch on the device: the state is uploaded at t
    integer(c_int) function echo_gpu_optical_glauber(ctx, g, t, check_mass, max_e) &
        bind(C, name="echo_gpu_optical_glauber")
      import :: c_int, c_ptr, c_double, echo_optical_glauber
      type(c_ptr), value :: ctx
      type(echo_optical_glauber), intent(in) :: g
      real(c_double), value :: t
      real(c_double), intent(out) :: check_mass, max_e
    end function

    ! the fused stage kernel on (1) or off (0); info(7) receives the choice
    integer(c_int) function echo_gpu_set_stage(ctx, fused, tx, ty, zseg, info) bind(C, name="echo_gpu_set_stage")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: fused, tx, ty, zseg
      integer(c_int), intent(out) :: info(7)
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
