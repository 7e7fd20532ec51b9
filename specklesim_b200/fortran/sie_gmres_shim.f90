! ISO_C_BINDING shim: the public procedures of the reference module
! lib_sie_solver_gmres_interface (src/lib_sie_solver_gmres_interface.f90:27-29) with the
! whole GMRES solve on the GPU (sie_solve, include/sie_gpu.h) in place of the CPU driver
! lib_math_solver_gmres_run and its per-iteration callbacks.  Compile it in place of the
! reference module, together with sie_shim.f90 in place of lib_sie_tri_mlfmm_interface;
! main.f90 links unchanged.
!
! Module globals read here are the reference's own (lib_sie_data_container,
! lib_sie_tri_data_container): restart, max_iterations, convergence_tolerance, x_initial,
! precondition_left, m_pairs, n_el, file_out_error, file_name_output_I, simulation_data.
! Differences from the reference routine (:123-211):
! - the solve is one library call, so the error file holds one line (iterations and the
!   final Arnoldi backward error) where the reference writes one per iteration;
! - precondition_left selects the library's near-field preconditioner (applied on the
!   right) in place of the left Jacobi scaling;
! - the run-parameters file (output_file_GMRES, :213-245) is not written here
!   (specklesim_b200.io writes the same file from Python).
! Not compiled in this repository's test-suite: the build image has no Fortran compiler.

module lib_sie_solver_gmres_interface
  use iso_c_binding
  use sie_gpu_c
  use lib_sie_tri_mlfmm_interface
  use lib_sie_data_container
  use lib_sie_tri_data_container
  implicit none
  private

  public :: run_ml_fmm_GMRES_tri
  public :: lib_sie_solver_GMRES_run
  public :: prerun_ml_fmm_GMRES_tri_conical_planewaves

  integer, parameter :: unit_error = 115

contains

  ! run_ml_fmm_GMRES_tri (:39-45)
  subroutine run_ml_fmm_GMRES_tri()
    call set_parameters_tri()
    call lib_sie_ml_fmm_precalculation_tri()
    call lib_sie_solver_gmres_run()
  end subroutine run_ml_fmm_GMRES_tri

  ! prerun_ml_fmm_GMRES_tri_conical_planewaves (:47-53)
  subroutine prerun_ml_fmm_GMRES_tri_conical_planewaves()
    call set_parameters_tri()
    call lib_sie_ml_fmm_precalculation_tri()
  end subroutine prerun_ml_fmm_GMRES_tri_conical_planewaves

  ! lib_sie_solver_gmres_run (:123-211): the plane-wave right-hand side, the solve from
  ! x_initial, the currents saved and written to file_name_output_I.
  subroutine lib_sie_solver_gmres_run()
    type(sie_solver_cfg) :: cfg
    type(sie_stats) :: st
    double complex, dimension(:), allocatable, target :: b, x
    type(c_ptr) :: ctx
    integer(c_int) :: rc
    integer :: i, count0, count1, rate
    double precision :: gmres_time
    ctx = sie_shim_context()
    call system_clock(count0, rate)
    call lib_sie_ml_fmm_get_vector_b_tri(b)
    allocate(x(2 * m_pairs))
    x = x_initial
    call sie_solver_default(cfg)
    cfg%restart = restart
    cfg%max_iterations = max_iterations
    cfg%tolerance = convergence_tolerance
    cfg%use_initial_guess = 1
    if (precondition_left) then
      call sie_check(sie_set_preconditioner(ctx, SIE_PRECOND_NEAR), 'sie_set_preconditioner')
      file_out_error = trim(file_out_error)//'_LeftP.txt'
    else
      file_out_error = trim(file_out_error)//'_NoP.txt'
    end if
    rc = sie_solve(ctx, c_loc(b), c_loc(x), 1_c_int, cfg, st)
    if (rc /= SIE_ERR_NOCONV) call sie_check(rc, 'sie_solve')
    call system_clock(count1, rate)
    gmres_time = (count1 - count0) / real(rate) / 60
    print '("GMRES-Time = ",f15.3," mins.")', gmres_time
    open (unit=unit_error, file=file_out_error, action="write", status='replace')
    write (unit_error, '(1(i10, tr5), 1(es19.12, tr5))') st%iterations, st%backward_error_arnoldi
    close (unit_error)
    call lib_sie_ml_fmm_save_vector_x_tri(x)
    open (unit=206, file=file_name_output_I, action="write", status='replace')
    write (206, *) 'n_el,', n_el
    write (206, *) 'm_pairs', m_pairs
    do i = 1, m_pairs * 2
      write (206, '(201(es19.12, tr5))') simulation_data%vector_x(i)
    end do
    close (206)
  end subroutine lib_sie_solver_gmres_run

end module lib_sie_solver_gmres_interface
