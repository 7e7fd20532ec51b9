! ISO_C_BINDING shim: the public procedures of the reference module
! lib_sie_tri_mlfmm_interface (src/lib_sie_tri_mlfmm_interface.f90:18-26) with the
! B200 library (include/sie_gpu.h) behind them.  Compile this file in place of the
! reference module; lib_sie_solver_gmres_interface and main.f90 link unchanged, and
! the GMRES driver keeps calling the same callbacks (lib_sie_solver_gmres_interface.f90:60-80).
!
! Module globals read here are the reference's own (lib_sie_data_container,
! lib_sie_tri_data_container): struc_tri, m_pairs, illumination_p, eps_r1, eps_r2,
! calc_p, pre_types, ng, tree_s_opt, truncation_number_default, x_initial,
! simulation_data.  A non-zero status prints the library's message and stops, which is
! how the reference reports errors.
!
! Not compiled in this repository's test-suite: the build image has no Fortran compiler.
! The C entry points it binds are exercised through ctypes by tests/test_gpu_parity.py.

module sie_gpu_c
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: SIE_OK = 0
  integer(c_int), parameter :: SIE_ERR_NOCONV = 6
  integer(c_int), parameter :: SIE_PMCHWT = 1
  integer(c_int), parameter :: SIE_ICTF = 3
  integer(c_int), parameter :: SIE_FP64 = 0
  integer(c_int), parameter :: SIE_PRECOND_NEAR = 1

  type, bind(C) :: sie_config
    real(c_double) :: lambda
    real(c_double) :: eps_r1_re, eps_r1_im
    real(c_double) :: eps_r2_re, eps_r2_im
    integer(c_int) :: formulation
    integer(c_int) :: ngp
    integer(c_int) :: tree_s_opt
    integer(c_int) :: truncation_number
    integer(c_int) :: normal_convention
    integer(c_int) :: fix_itbn
    integer(c_int) :: device
    integer(c_int) :: dense
  end type sie_config

  type, bind(C) :: sie_solver_cfg
    integer(c_int) :: restart
    integer(c_int) :: max_iterations
    real(c_double) :: tolerance
    integer(c_int) :: use_initial_guess
    integer(c_int) :: precision
    integer(c_int) :: inner_restart
    real(c_double) :: inner_tolerance
    real(c_double) :: time_limit_s
  end type sie_solver_cfg

  type, bind(C) :: sie_stats
    integer(c_int) :: iterations
    integer(c_int) :: inner_iterations
    integer(c_int) :: matvecs
    integer(c_int) :: converged
    real(c_double) :: backward_error_arnoldi
    real(c_double) :: backward_error_true
    real(c_double) :: seconds
  end type sie_stats

  interface
    subroutine sie_config_default(cfg) bind(C, name="sie_config_default")
      import :: sie_config
      type(sie_config), intent(out) :: cfg
    end subroutine
    function sie_last_error() bind(C, name="sie_last_error") result(p)
      import :: c_ptr
      type(c_ptr) :: p
    end function
    function sie_init(cfg, verts, nv, tris, nt, ctx) bind(C, name="sie_init") result(rc)
      import :: c_int, c_double, c_ptr, sie_config
      type(sie_config), intent(in) :: cfg
      real(c_double), intent(in) :: verts(*)
      integer(c_int), value :: nv
      integer(c_int), intent(in) :: tris(*)
      integer(c_int), value :: nt
      type(c_ptr), intent(out) :: ctx
      integer(c_int) :: rc
    end function
    function sie_setup(ctx) bind(C, name="sie_setup") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function
    function sie_matvec(ctx, x, y, nrhs, precision) bind(C, name="sie_matvec") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, x, y
      integer(c_int), value :: nrhs, precision
      integer(c_int) :: rc
    end function
    function sie_rhs_planewave(ctx, k_in, e_in, nrhs, b) bind(C, name="sie_rhs_planewave") result(rc)
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: k_in(3), e_in(3)
      integer(c_int), value :: nrhs
      type(c_ptr), value :: b
      integer(c_int) :: rc
    end function
    function sie_precondition_left(ctx, v1, v2) bind(C, name="sie_precondition_left") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, v1, v2
      integer(c_int) :: rc
    end function
    subroutine sie_solver_default(cfg) bind(C, name="sie_solver_default")
      import :: sie_solver_cfg
      type(sie_solver_cfg), intent(out) :: cfg
    end subroutine
    function sie_matvec_adjoint(ctx, x, y, nrhs) bind(C, name="sie_matvec_adjoint") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, x, y
      integer(c_int), value :: nrhs
      integer(c_int) :: rc
    end function
    function sie_grad(ctx, x, k_in, e_in, pts, npts, cfg, dJdz, J, stats) bind(C, name="sie_grad") result(rc)
      import :: c_int, c_double, c_ptr, sie_solver_cfg, sie_stats
      type(c_ptr), value :: ctx, x
      real(c_double), intent(in) :: k_in(3), e_in(3)
      type(c_ptr), value :: pts
      integer(c_int), value :: npts
      type(sie_solver_cfg), intent(in) :: cfg
      type(c_ptr), value :: dJdz
      real(c_double), intent(out) :: J
      type(sie_stats), intent(out) :: stats
      integer(c_int) :: rc
    end function
    function sie_set_inner_operator(ctx, inner) bind(C, name="sie_set_inner_operator") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, inner
      integer(c_int) :: rc
    end function
    function sie_solve(ctx, b, x, nrhs, cfg, stats) bind(C, name="sie_solve") result(rc)
      import :: c_int, c_ptr, sie_solver_cfg, sie_stats
      type(c_ptr), value :: ctx
      type(c_ptr), value :: b, x
      integer(c_int), value :: nrhs
      type(sie_solver_cfg), intent(in) :: cfg
      type(sie_stats), intent(out) :: stats
      integer(c_int) :: rc
    end function
    function sie_set_preconditioner(ctx, kind) bind(C, name="sie_set_preconditioner") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: kind
      integer(c_int) :: rc
    end function
    function sie_solve_direct(ctx, b, x, nrhs) bind(C, name="sie_solve_direct") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, b, x
      integer(c_int), value :: nrhs
      integer(c_int) :: rc
    end function
    function sie_solve_direct_mixed(ctx, b, x, nrhs, tolerance, &
        max_refinements, stats) bind(C, name="sie_solve_direct_mixed") result(rc)
      import :: c_int, c_double, c_ptr, sie_stats
      type(c_ptr), value :: ctx, b, x
      integer(c_int), value :: nrhs
      real(c_double), value :: tolerance
      integer(c_int), value :: max_refinements
      type(sie_stats), intent(out) :: stats
      integer(c_int) :: rc
    end function
    function sie_release_factors(ctx) bind(C, name="sie_release_factors") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function
    function sie_farfield(ctx, x, pts, npts, E, H, intensity) bind(C, name="sie_farfield") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, x, pts
      integer(c_int), value :: npts
      type(c_ptr), value :: E, H, intensity
      integer(c_int) :: rc
    end function
    function sie_field_interior(ctx, x, pts, npts, eps_r_re, eps_r_im, &
        E, H) bind(C, name="sie_field_interior") result(rc)
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx, x, pts
      integer(c_int), value :: npts
      real(c_double), value :: eps_r_re, eps_r_im
      type(c_ptr), value :: E, H
      integer(c_int) :: rc
    end function
    function sie_free(ctx) bind(C, name="sie_free") result(rc)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function
  end interface

contains

  subroutine sie_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    integer :: n
    if (rc == SIE_OK) return
    call c_f_pointer(sie_last_error(), msg, [1024])
    n = 0
    do while (n < 1024)
      if (msg(n + 1) == c_null_char) exit
      n = n + 1
    end do
    print *, 'B200 SIE library: ', what, ' failed (status ', rc, '): ', msg(1:n)
    stop
  end subroutine sie_check

end module sie_gpu_c


module lib_sie_tri_mlfmm_interface
  use iso_c_binding
  use sie_gpu_c
  use lib_sie_data_container
  use lib_sie_tri_data_container
  implicit none
  private

  public :: lib_sie_ml_fmm_calculate_vector_b_tri
  public :: lib_sie_ml_fmm_get_vector_b_tri
  public :: lib_sie_ml_fmm_get_init_vector_x_tri
  public :: lib_sie_ml_fmm_precalculation_tri
  public :: lib_sie_ml_fmm_run_tri
  public :: lib_sie_ml_fmm_save_vector_x_tri
  public :: run_MLFMM_one_forward_tri
  public :: lib_sie_ml_fmm_preconditioner_left
  ! additions with no counterpart in the reference module: the adjoint product and the
  ! shape gradient of the far-field intensity
  public :: lib_sie_ml_fmm_adjoint_tri
  public :: lib_sie_ml_fmm_grad_z_tri
  ! the fill and dense LU solve of the reference's normal solver, on the GPU
  public :: lib_sie_ml_fmm_solve_direct_tri
  ! the fields at observation points, outside and inside the body, on the GPU
  public :: lib_sie_ml_fmm_fields_tri
  ! the library context, for the GMRES-interface shim (sie_gmres_shim.f90)
  public :: sie_shim_context

  type(c_ptr), save :: m_ctx = c_null_ptr

contains

  function sie_shim_context() result(ctx)
    type(c_ptr) :: ctx
    ctx = m_ctx
  end function sie_shim_context

  ! The library's settings and mesh from the reference's module globals, as the
  ! precalculation (:59-92) takes them; dense = 1 asks for the assembled matrix.
  subroutine shim_open(dense, ctx)
    integer(c_int), intent(in) :: dense
    type(c_ptr), intent(inout) :: ctx
    type(sie_config) :: cfg
    real(c_double), allocatable :: verts(:)
    integer(c_int), allocatable :: tris(:)
    integer :: i, nv, nt
    nv = size(struc_tri%points)
    nt = size(struc_tri%elements)
    allocate(verts(3 * nv), tris(3 * nt))
    do i = 1, nv
      verts(3 * i - 2:3 * i) = struc_tri%points(i)%point
    end do
    do i = 1, nt
      tris(3 * i - 2:3 * i) = struc_tri%elements(i)%corners(1:3) - 1
    end do
    call sie_config_default(cfg)
    cfg%lambda = illumination_p%lambda
    cfg%eps_r1_re = real(eps_r1, c_double)
    cfg%eps_r1_im = aimag(eps_r1)
    cfg%eps_r2_re = real(eps_r2, c_double)
    cfg%eps_r2_im = aimag(eps_r2)
    cfg%formulation = SIE_ICTF
    if (pre_types%formulation == 'PMCHWT') cfg%formulation = SIE_PMCHWT
    cfg%ngp = ng
    cfg%tree_s_opt = tree_s_opt
    cfg%truncation_number = truncation_number_default
    cfg%normal_convention = calc_p(7)
    cfg%dense = dense
    if (c_associated(ctx)) call sie_check(sie_free(ctx), 'sie_free')
    call sie_check(sie_init(cfg, verts, nv, tris, nt, ctx), 'sie_init')
    call sie_check(sie_setup(ctx), 'sie_setup')
  end subroutine shim_open

  ! lib_sie_ml_fmm_precalculation_tri (:59-92): mesh, tree, near field, RT, TL, diagonal.
  subroutine lib_sie_ml_fmm_precalculation_tri()
    call shim_open(0_c_int, m_ctx)
  end subroutine lib_sie_ml_fmm_precalculation_tri

  subroutine run_MLFMM_one_forward_tri()
    call lib_sie_ml_fmm_precalculation_tri()
    call lib_sie_ml_fmm_run_tri()
  end subroutine run_MLFMM_one_forward_tri

  ! lib_sie_ml_fmm_run_tri (:164-188): one forward product with the initial vector.
  subroutine lib_sie_ml_fmm_run_tri()
    double complex, dimension(:), allocatable :: x, b
    call lib_sie_ml_fmm_get_init_vector_x_tri(x)
    allocate(b(2 * m_pairs))
    call lib_sie_ml_fmm_calculate_vector_b_tri(x, b)
  end subroutine lib_sie_ml_fmm_run_tri

  ! lib_sie_ml_fmm_get_init_vector_x_tri (:190-239), file branch disabled as in the reference.
  subroutine lib_sie_ml_fmm_get_init_vector_x_tri(vector_x)
    double complex, dimension(:), allocatable, intent(inout) :: vector_x
    if (allocated(vector_x)) deallocate(vector_x)
    allocate(vector_x(2 * m_pairs))
    vector_x = x_initial
  end subroutine lib_sie_ml_fmm_get_init_vector_x_tri

  ! lib_sie_ml_fmm_save_vector_x_tri (:241-261)
  subroutine lib_sie_ml_fmm_save_vector_x_tri(vector_x)
    double complex, dimension(:), allocatable, intent(in) :: vector_x
    double complex, dimension(:), allocatable :: buffer_x
    allocate(buffer_x(size(vector_x)))
    buffer_x = vector_x
    call move_alloc(buffer_x, simulation_data%vector_x)
  end subroutine lib_sie_ml_fmm_save_vector_x_tri

  ! lib_sie_ml_fmm_get_vector_b_tri (:263-276): plane-wave right-hand side.
  subroutine lib_sie_ml_fmm_get_vector_b_tri(vector_b)
    double complex, dimension(:), allocatable, target, intent(inout) :: vector_b
    if (allocated(vector_b)) deallocate(vector_b)
    allocate(vector_b(2 * m_pairs))
    call sie_check(sie_rhs_planewave(m_ctx, illumination_p%k_in, illumination_p%E_in, 1_c_int, &
                                     c_loc(vector_b)), 'sie_rhs_planewave')
  end subroutine lib_sie_ml_fmm_get_vector_b_tri

  ! lib_sie_ml_fmm_calculate_vector_b_tri (:285-319): the GMRES matvec callback.
  subroutine lib_sie_ml_fmm_calculate_vector_b_tri(vector_x, vector_b)
    double complex, dimension(:), allocatable, target, intent(in) :: vector_x
    double complex, dimension(:), allocatable, target, intent(inout) :: vector_b
    call sie_check(sie_matvec(m_ctx, c_loc(vector_x), c_loc(vector_b), 1_c_int, SIE_FP64), &
                   'sie_matvec')
  end subroutine lib_sie_ml_fmm_calculate_vector_b_tri

  ! lib_sie_ml_fmm_preconditioner_left (:323-339)
  subroutine lib_sie_ml_fmm_preconditioner_left(vector_1, vector_2)
    double complex, dimension(:), allocatable, target, intent(in) :: vector_1
    double complex, dimension(:), allocatable, target, intent(out) :: vector_2
    allocate(vector_2(size(vector_1)))
    call sie_check(sie_precondition_left(m_ctx, c_loc(vector_1), c_loc(vector_2)), &
                   'sie_precondition_left')
  end subroutine lib_sie_ml_fmm_preconditioner_left

  ! vector_y = Z^H vector_x (FP64), the operator of an adjoint solve
  subroutine lib_sie_ml_fmm_adjoint_tri(vector_x, vector_y)
    double complex, dimension(:), allocatable, target, intent(in) :: vector_x
    double complex, dimension(:), allocatable, target, intent(inout) :: vector_y
    call sie_check(sie_matvec_adjoint(m_ctx, c_loc(vector_x), c_loc(vector_y), 1_c_int), &
                   'sie_matvec_adjoint')
  end subroutine lib_sie_ml_fmm_adjoint_tri

  ! dJ/dz of every vertex for J = sum of far-field intensities at the points pts(3, npts),
  ! at the solution vector_x of the plane wave (k_in, e_in); adjoint solve with FP64 GMRES
  ! (restart, max_iterations, tolerance)
  subroutine lib_sie_ml_fmm_grad_z_tri(vector_x, k_in, e_in, pts, restart, max_iterations, tolerance, &
                                       dJdz, J)
    double complex, dimension(:), allocatable, target, intent(in) :: vector_x
    real(c_double), intent(in) :: k_in(3), e_in(3)
    real(c_double), dimension(:, :), allocatable, target, intent(in) :: pts
    integer, intent(in) :: restart, max_iterations
    double precision, intent(in) :: tolerance
    real(c_double), dimension(:), allocatable, target, intent(inout) :: dJdz
    double precision, intent(out) :: J
    type(sie_solver_cfg) :: cfg
    type(sie_stats) :: st
    integer(c_int) :: rc
    call sie_solver_default(cfg)
    cfg%restart = restart
    cfg%max_iterations = max_iterations
    cfg%tolerance = tolerance
    rc = sie_grad(m_ctx, c_loc(vector_x), k_in, e_in, c_loc(pts), int(size(pts, 2), c_int), cfg, &
                  c_loc(dJdz), J, st)
    if (rc /= SIE_ERR_NOCONV) call sie_check(rc, 'sie_grad')
  end subroutine lib_sie_ml_fmm_grad_z_tri

  ! The impedance fill and solver_LU of lib_sie_tri_solver_normal_I
  ! (src/lib_sie_tri_solver_normal.f90:87-138, ZGESV at src/lib_sie_math.f90:649-676) on
  ! the GPU: a dense context from the same module globals, the plane-wave right-hand side
  ! and the direct solve.  mixed = .false. factorises the FP64 matrix; mixed = .true.
  ! factorises it in complex64 on the tensor cores and refines in FP64 until
  ! ||b - Z x|| <= tolerance ||b||.  On return vector_b holds the solution, as VV_EH of
  ! solver_LU does; the context and its factors are freed.
  subroutine lib_sie_ml_fmm_solve_direct_tri(vector_b, mixed, tolerance)
    double complex, dimension(:), allocatable, target, intent(inout) :: vector_b
    logical, intent(in) :: mixed
    double precision, intent(in) :: tolerance
    double complex, dimension(:), allocatable, target :: vector_x
    type(c_ptr) :: ctx
    type(sie_stats) :: st
    integer(c_int) :: rc
    ctx = c_null_ptr
    call shim_open(1_c_int, ctx)
    if (allocated(vector_b)) deallocate(vector_b)
    allocate(vector_b(2 * m_pairs), vector_x(2 * m_pairs))
    call sie_check(sie_rhs_planewave(ctx, illumination_p%k_in, illumination_p%E_in, 1_c_int, &
                                     c_loc(vector_b)), 'sie_rhs_planewave')
    if (mixed) then
      rc = sie_solve_direct_mixed(ctx, c_loc(vector_b), c_loc(vector_x), 1_c_int, &
                                  real(tolerance, c_double), 30_c_int, st)
      if (rc == SIE_ERR_NOCONV) then
        print *, 'B200 SIE library: refinement stopped at backward error ', st%backward_error_true
      else
        call sie_check(rc, 'sie_solve_direct_mixed')
      end if
    else
      call sie_check(sie_solve_direct(ctx, c_loc(vector_b), c_loc(vector_x), 1_c_int), &
                     'sie_solve_direct')
    end if
    vector_b = vector_x
    call sie_check(sie_free(ctx), 'sie_free')
  end subroutine lib_sie_ml_fmm_solve_direct_tri

  ! E(3, n) and H(3, n) at the points pts(3, n) for the currents vector_x: where media(i)
  ! is 2, the field inside the body (Integration_scattered_field_tri_within_medium,
  ! src/lib_sie_tri_calculation_mod.f90:2829-2877, in eps_r2), elsewhere the scattered
  ! field (Integration_scattered_field_tri, :2782-2825); all points in two library calls,
  ! for the point loops of lib_sie_tri_observation_field_calculation
  ! (src/lib_sie_tri_solver_normal.f90:325-420), which add the incident field and zero
  ! vanishing interior components as before.
  subroutine lib_sie_ml_fmm_fields_tri(vector_x, pts, media, E, H)
    double complex, dimension(:), allocatable, target, intent(in) :: vector_x
    real(c_double), dimension(:, :), intent(in) :: pts
    integer, dimension(:), intent(in) :: media
    double complex, dimension(:, :), intent(out) :: E, H
    real(c_double), allocatable, target :: p_in(:, :), p_out(:, :), intens(:)
    double complex, allocatable, target :: e_in(:, :), h_in(:, :), e_out(:, :), h_out(:, :)
    integer :: i, n_in, n_out, a, b
    n_in = count(media == 2)
    n_out = size(media) - n_in
    allocate(p_in(3, max(n_in, 1)), p_out(3, max(n_out, 1)), intens(max(n_out, 1)))
    allocate(e_in(3, max(n_in, 1)), h_in(3, max(n_in, 1)), e_out(3, max(n_out, 1)), h_out(3, max(n_out, 1)))
    a = 0
    b = 0
    do i = 1, size(media)
      if (media(i) == 2) then
        a = a + 1
        p_in(:, a) = pts(:, i)
      else
        b = b + 1
        p_out(:, b) = pts(:, i)
      end if
    end do
    if (n_in > 0) call sie_check(sie_field_interior(m_ctx, c_loc(vector_x), c_loc(p_in), int(n_in, c_int), &
                                 real(eps_r2, c_double), real(aimag(eps_r2), c_double), c_loc(e_in), &
                                 c_loc(h_in)), 'sie_field_interior')
    if (n_out > 0) call sie_check(sie_farfield(m_ctx, c_loc(vector_x), c_loc(p_out), int(n_out, c_int), &
                                  c_loc(e_out), c_loc(h_out), c_loc(intens)), 'sie_farfield')
    a = 0
    b = 0
    do i = 1, size(media)
      if (media(i) == 2) then
        a = a + 1
        E(:, i) = e_in(:, a)
        H(:, i) = h_in(:, a)
      else
        b = b + 1
        E(:, i) = e_out(:, b)
        H(:, i) = h_out(:, b)
      end if
    end do
  end subroutine lib_sie_ml_fmm_fields_tri

end module lib_sie_tri_mlfmm_interface
