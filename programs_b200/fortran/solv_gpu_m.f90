! solv_gpu_m.f90 -- iso_c_binding layer over libsolv_gpu.so for the
! spray-simulation host code.  Drop-in replacements of solv_cg / solv_bicg
! (spray-simulation/solv_cg.f90:7, solv_bicg.f90:7) with the same argument
! lists; the matrix comes from the same module globals (solv_data_m: pl, ng)
! and is handed to the GPU by solv_gpu_sync_matrix, which stands in for
! grd_solv (grd_solv.f90:7-24) and for every coefficient refill done by
! cfd_setup before a solve.
!
! No Fortran compiler exists on the build machines, so this module ships as
! source; the C entry points it binds are exercised from C/C++/Python
! (tests/test_abi.py checks every name bound here is exported).
module solv_gpu_m
  use iso_c_binding
  use solv_data_m
  implicit none
  private
  public :: solv_gpu_init, solv_gpu_sync_matrix, solv_gpu_sync_values, &
            solv_cg, solv_bicg, solv_gpu_final

  integer(c_intptr_t), save :: ctx = 0_c_intptr_t
  logical, save :: have_structure = .false.

  interface
    ! solv_gpu_create(solv_gpu_ctx **out, int device): out is the address
    ! of the handle, passed by value
    integer(c_int) function c_create(pctx, device) bind(c, name='solv_gpu_create')
      import :: c_ptr, c_int
      type(c_ptr), value :: pctx
      integer(c_int), value :: device
    end function
    integer(c_int) function c_destroy(h) bind(c, name='solv_gpu_destroy')
      import :: c_intptr_t, c_int
      integer(c_intptr_t), value :: h
    end function
    integer(c_int) function c_matrix_set(h, n_cell, n_face, ip, in, p, n, pl) &
        bind(c, name='solv_gpu_matrix_set')
      import :: c_intptr_t, c_int, c_double
      integer(c_intptr_t), value :: h
      integer(c_int), value :: n_cell, n_face
      integer(c_int), dimension(*) :: ip, in
      real(c_double), dimension(*) :: p, n, pl
    end function
    integer(c_int) function c_matrix_values(h, p, n, pl) bind(c, name='solv_gpu_matrix_values')
      import :: c_intptr_t, c_int, c_double
      integer(c_intptr_t), value :: h
      real(c_double), dimension(*) :: p, n, pl
    end function
    integer(c_int) function c_cg(h, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st) &
        bind(c, name='solv_gpu_cg')
      import :: c_intptr_t, c_int, c_double, c_ptr
      integer(c_intptr_t), value :: h
      integer(c_int), value :: imat, n_iter, n_vc, not_r0
      real(c_double), value :: reduc
      real(c_double), dimension(*) :: phi, res0, res0_n
      type(c_ptr), value :: st
    end function
    integer(c_int) function c_bicg(h, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st) &
        bind(c, name='solv_gpu_bicg')
      import :: c_intptr_t, c_int, c_double, c_ptr
      integer(c_intptr_t), value :: h
      integer(c_int), value :: imat, n_iter, n_vc, not_r0
      real(c_double), value :: reduc
      real(c_double), dimension(*) :: phi, res0, res0_n
      type(c_ptr), value :: st
    end function
  end interface

contains

  subroutine solv_gpu_init(device)
    integer, intent(in) :: device
    integer(c_int) :: rc
    integer(c_intptr_t), target :: h
    h = 0
    rc = c_create(c_loc(h), int(device, c_int))
    if (rc /= 0 .or. h == 0) stop 'solv_gpu_init: no CUDA device'
    ctx = h
    have_structure = .false.
  end subroutine

  subroutine solv_gpu_final()
    integer(c_int) :: rc
    if (ctx /= 0) rc = c_destroy(ctx)
    ctx = 0
  end subroutine

  ! grd_solv: structure + coefficients of the module globals ng, pl
  subroutine solv_gpu_sync_matrix()
    integer(c_int), allocatable :: ip(:), in(:)
    real(c_double), allocatable :: p(:), n(:)
    integer(c_int) :: rc
    integer :: f
    allocate(ip(size(ng)), in(size(ng)), p(size(ng)), n(size(ng)))
    do f = 1, size(ng)
      ip(f) = ng(f)%ip; in(f) = ng(f)%in
      p(f) = ng(f)%p;   n(f) = ng(f)%n
    end do
    rc = c_matrix_set(ctx, int(size(pl), c_int), int(size(ng), c_int), ip, in, p, n, pl)
    if (rc /= 0) stop 'solv_gpu_sync_matrix failed'
    have_structure = .true.
  end subroutine

  ! cfd_setup refilled ng%p, ng%n, pl on the same structure
  subroutine solv_gpu_sync_values()
    real(c_double), allocatable :: p(:), n(:)
    integer(c_int) :: rc
    integer :: f
    if (.not. have_structure) then
      call solv_gpu_sync_matrix()
      return
    end if
    allocate(p(size(ng)), n(size(ng)))
    do f = 1, size(ng)
      p(f) = ng(f)%p; n(f) = ng(f)%n
    end do
    rc = c_matrix_values(ctx, p, n, pl)
    if (rc /= 0) stop 'solv_gpu_sync_values failed'
  end subroutine

  subroutine pack_phi(phi, n_cell, n_vc, buf)
    type(phi_t), dimension(:), intent(in) :: phi
    integer, intent(in) :: n_cell, n_vc
    real(c_double), intent(out) :: buf(n_vc, n_cell)
    integer :: ip
    do ip = 1, n_cell
      buf(:, ip) = phi(ip)%vc(1:n_vc)
    end do
  end subroutine

  subroutine unpack_phi(buf, n_cell, n_vc, phi)
    integer, intent(in) :: n_cell, n_vc
    real(c_double), intent(in) :: buf(n_vc, n_cell)
    type(phi_t), dimension(:), intent(inout) :: phi
    integer :: ip
    do ip = 1, n_cell
      phi(ip)%vc(1:n_vc) = buf(:, ip)
    end do
  end subroutine

  ! same argument list as spray-simulation/solv_cg.f90:7-13
  subroutine solv_cg(imat, reduc, n_iter, phi, res0, res0_n, not_r0)
    integer, intent(in) :: imat, n_iter
    real(wp), intent(in) :: reduc
    logical, intent(in) :: not_r0
    type(phi_t), dimension(:), intent(inout) :: phi
    real(wp), dimension(:,:), intent(inout) :: res0
    real(wp), dimension(:), intent(inout) :: res0_n
    real(c_double), allocatable :: buf(:,:)
    integer(c_int) :: rc, nr
    if (size(res0, 1) /= size(pl) .or. size(res0, 2) /= size(res0_n)) &
      stop 'solv_cg (gpu): res0 must be res0(n_cell, n_vc)'
    allocate(buf(size(res0_n), size(pl)))
    call solv_gpu_sync_values()
    call pack_phi(phi, size(pl), size(res0_n), buf)
    nr = 0; if (not_r0) nr = 1
    rc = c_cg(ctx, int(imat, c_int), real(reduc, c_double), int(n_iter, c_int), &
              int(size(res0_n), c_int), buf, res0, res0_n, nr, c_null_ptr)
    if (rc /= 0 .and. rc /= 1) stop 'solv_cg (gpu) failed'
    call unpack_phi(buf, size(pl), size(res0_n), phi)
  end subroutine

  ! same argument list as spray-simulation/solv_bicg.f90:7-13
  subroutine solv_bicg(imat, reduc, n_iter, phi, res0, res0_n, not_r0)
    integer, intent(in) :: imat, n_iter
    real(wp), intent(in) :: reduc
    logical, intent(in) :: not_r0
    type(phi_t), dimension(:), intent(inout) :: phi
    real(wp), dimension(:,:), intent(inout) :: res0
    real(wp), dimension(:), intent(inout) :: res0_n
    real(c_double), allocatable :: buf(:,:)
    integer(c_int) :: rc, nr
    if (size(res0, 1) /= size(pl) .or. size(res0, 2) /= size(res0_n)) &
      stop 'solv_bicg (gpu): res0 must be res0(n_cell, n_vc)'
    allocate(buf(size(res0_n), size(pl)))
    call solv_gpu_sync_values()
    call pack_phi(phi, size(pl), size(res0_n), buf)
    nr = 0; if (not_r0) nr = 1
    rc = c_bicg(ctx, int(imat, c_int), real(reduc, c_double), int(n_iter, c_int), &
                int(size(res0_n), c_int), buf, res0, res0_n, nr, c_null_ptr)
    if (rc /= 0 .and. rc /= 1) stop 'solv_bicg (gpu) failed'
    call unpack_phi(buf, size(pl), size(res0_n), phi)
  end subroutine
end module
