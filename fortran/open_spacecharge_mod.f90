!-----------------------------------------------------------------------------------------
! open_spacecharge_mod (drop-in): the public interface of code/open_spacecharge_mod.f90 --
! mesh3d_struct, deposit_particles, space_charge_3d, space_charge_freespace,
! space_charge_cathodeimages, space_charge_rectpipe, osc_freespace_solver2,
! interpolate_field, print_mesh3d -- with the same dummy arguments and optional-argument
! defaults, the work done by libopensc_b200.so (include/opensc_gpu.h).
!
! A program that uses the reference module links against this one instead
! (gfortran fortran/open_spacecharge_core_mod.f90 fortran/open_spacecharge_mod.f90 ...
! -L<dir> -lopensc_b200).  Arrays are passed as they are: Fortran column-major with the
! field component slowest is the library's layout.  interpolate_field of one point runs on
! the host (a GPU round trip per point would cost more than the arithmetic);
! interpolate_field_batch does many points on the GPU.
!-----------------------------------------------------------------------------------------
module open_spacecharge_mod

use, intrinsic :: iso_c_binding
use, intrinsic :: iso_fortran_env
use open_spacecharge_core_mod

implicit none

integer, parameter, private :: dp = REAL64

type mesh3d_struct
  integer :: nlo(3) = [ 1,  1,  1]       ! lowest grid index in x, y, z of rho and the fields
  integer :: nhi(3) = [64, 64, 64]       ! highest grid index in x, y, z
  integer :: npad(3) = [ 1,  1,  1]      ! padding of the cyclic convolution (legacy solvers)
  real(dp) :: min(3)                     ! mesh minimum per dimension
  real(dp) :: max(3)                     ! mesh maximum per dimension
  real(dp) :: delta(3)                   ! grid spacing
  real(dp) :: gamma                      ! relativistic gamma
  real(dp) :: charge                     ! total charge on the mesh
  real(dp), allocatable, dimension(:,:,:) :: rho
  real(dp), allocatable, dimension(:,:,:) :: phi
  real(dp), allocatable, dimension(:,:,:,:) :: efield
  real(dp), allocatable, dimension(:,:,:,:) :: bfield
end type

interface
  integer(c_int) function c_deposit_particles(ctx, np, xa, ya, za, qa, total_charge, resize, mesh, rho, &
      n_outside) bind(C, name="osc_deposit_particles")
    import :: c_ptr, c_int, c_int64_t, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    integer(c_int64_t), value :: np
    real(c_double), intent(in) :: xa(*), ya(*), za(*)
    type(c_ptr), value :: qa, total_charge
    integer(c_int), value :: resize
    type(osc_mesh3d_c) :: mesh
    real(c_double) :: rho(*)
    integer(c_int64_t) :: n_outside
  end function
  integer(c_int) function c_space_charge_3d(ctx, mesh, rho, offset, at_cathode, calc_bfield, prec, efield, &
      bfield) bind(C, name="osc_space_charge_3d")
    import :: c_ptr, c_int, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    type(osc_mesh3d_c), intent(in) :: mesh
    real(c_double), intent(in) :: rho(*)
    type(c_ptr), value :: offset
    integer(c_int), value :: at_cathode, calc_bfield, prec
    real(c_double) :: efield(*), bfield(*)
  end function
  integer(c_int) function c_freespace_solver2(ctx, n, rho, gamma, delta, offset, prec, efield, phi) &
      bind(C, name="osc_freespace_solver2")
    import :: c_ptr, c_int, c_int32_t, c_double
    type(c_ptr), value :: ctx
    integer(c_int32_t), intent(in) :: n(3)
    real(c_double), intent(in) :: rho(*)
    real(c_double), value :: gamma
    real(c_double), intent(in) :: delta(3)
    type(c_ptr), value :: offset, efield, phi
    integer(c_int), value :: prec
  end function
  integer(c_int) function c_interpolate_field(ctx, mesh, efield, bfield, np, x, y, z, E, B, n_clamped) &
      bind(C, name="osc_interpolate_field")
    import :: c_ptr, c_int, c_int64_t, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    type(osc_mesh3d_c), intent(in) :: mesh
    type(c_ptr), value :: efield, bfield, E, B
    integer(c_int64_t), value :: np
    real(c_double), intent(in) :: x(*), y(*), z(*)
    integer(c_int64_t) :: n_clamped
  end function
end interface

contains

function to_c(mesh3d) result(m)
  type(mesh3d_struct), intent(in) :: mesh3d
  type(osc_mesh3d_c) :: m
  m%nlo = int(mesh3d%nlo, c_int32_t)
  m%nhi = int(mesh3d%nhi, c_int32_t)
  m%npad = int(mesh3d%npad, c_int32_t)
  m%min = mesh3d%min
  m%max = mesh3d%max
  m%delta = mesh3d%delta
  m%gamma = mesh3d%gamma
  m%charge = mesh3d%charge
end function

subroutine print_mesh3d(mesh3d)
  type(mesh3d_struct) :: mesh3d
  print *, '------------------------'
  print *, 'Mesh: '
  print *, 'nlo: ', mesh3d%nlo
  print *, 'nhi: ', mesh3d%nhi
  print *, 'min: ', mesh3d%min
  print *, 'max: ', mesh3d%max
  print *, 'delta: ', mesh3d%delta
  print *, 'gamma: ', mesh3d%gamma
  print *, 'charge: ', mesh3d%charge
  if (allocated(mesh3d%rho)) print *, 'rho allocated'
  if (allocated(mesh3d%phi)) print *, 'phi allocated'
  if (allocated(mesh3d%efield)) print *, 'efield allocated'
  if (allocated(mesh3d%bfield)) print *, 'bfield allocated'
  print *, '------------------------'
end subroutine

! The grids of the mesh with bounds nlo:nhi, (re)allocated when the bounds changed
! (code/open_spacecharge_mod.f90:193-219).
subroutine ensure_grids(mesh3d)
  type(mesh3d_struct) :: mesh3d
  integer :: i, lo(3), hi(3)
  logical :: good
  lo = mesh3d%nlo
  hi = mesh3d%nhi
  if (allocated(mesh3d%rho)) then
    good = .true.
    do i = 1, 3
      if (lbound(mesh3d%rho, i) /= lo(i) .or. ubound(mesh3d%rho, i) /= hi(i)) good = .false.
    enddo
    if (.not. good) then
      deallocate(mesh3d%rho, mesh3d%phi, mesh3d%efield, mesh3d%bfield)
    endif
  endif
  if (.not. allocated(mesh3d%rho)) then
    allocate(mesh3d%rho(lo(1):hi(1), lo(2):hi(2), lo(3):hi(3)))
    allocate(mesh3d%phi(lo(1):hi(1), lo(2):hi(2), lo(3):hi(3)))
    allocate(mesh3d%efield(lo(1):hi(1), lo(2):hi(2), lo(3):hi(3), 3))
    allocate(mesh3d%bfield(lo(1):hi(1), lo(2):hi(2), lo(3):hi(3), 3))
  endif
end subroutine

!-----------------------------------------------------------------------------------------
! code/open_spacecharge_mod.f90:156-288
subroutine deposit_particles(xa, ya, za, mesh3d, qa, total_charge, resize_mesh)
  real(dp), target :: xa(:), ya(:), za(:)
  type(mesh3d_struct) :: mesh3d
  real(dp), optional, target :: qa(:), total_charge
  logical, optional :: resize_mesh
  type(osc_mesh3d_c) :: m
  type(c_ptr) :: pq, ptc
  integer(c_int) :: resize, rc
  integer(c_int64_t) :: nout
  resize = 1
  if (present(resize_mesh)) then
    if (.not. resize_mesh) resize = 0
  endif
  if (.not. present(qa) .and. .not. present(total_charge)) then
    write(*, *) 'Error, must specify qa or total_charge'
    return
  endif
  call ensure_grids(mesh3d)
  pq = c_null_ptr
  ptc = c_null_ptr
  if (present(qa)) then
    pq = c_loc(qa(1))
  else
    ptc = c_loc(total_charge)
  endif
  m = to_c(mesh3d)
  rc = c_deposit_particles(osc_context(), int(size(xa), c_int64_t), xa, ya, za, pq, ptc, resize, m, mesh3d%rho, &
      nout)
  call osc_check(rc, 'deposit_particles')
  mesh3d%min = m%min
  mesh3d%max = m%max
  mesh3d%delta = m%delta
  mesh3d%charge = m%charge
end subroutine

! code/open_spacecharge_mod.f90:431-489
subroutine space_charge_3d(mesh3d, offset, at_cathode, calc_bfield)
  type(mesh3d_struct) :: mesh3d
  real(dp), optional, target :: offset(3)
  logical, optional :: at_cathode, calc_bfield
  integer(c_int) :: cath, bcalc
  type(c_ptr) :: poff
  cath = 0
  bcalc = 0
  if (present(at_cathode)) then
    if (at_cathode) cath = 1
  endif
  if (present(calc_bfield)) then
    if (calc_bfield) bcalc = 1
  endif
  poff = c_null_ptr
  if (present(offset)) poff = c_loc(offset(1))
  call ensure_grids(mesh3d)
  call osc_check(c_space_charge_3d(osc_context(), to_c(mesh3d), mesh3d%rho, poff, cath, bcalc, osc_precision, &
      mesh3d%efield, mesh3d%bfield), 'space_charge_3d')
end subroutine

! code/open_spacecharge_mod.f90:535-597
subroutine osc_freespace_solver2(rho, gamma, delta, efield, phi, offset)
  real(dp), intent(in), dimension(:,:,:), target :: rho
  real(dp), intent(in) :: gamma, delta(3)
  real(dp), optional, intent(out), dimension(:,:,:,:), target :: efield
  real(dp), optional, intent(out), dimension(:,:,:), target :: phi
  real(dp), intent(in), optional, target :: offset(3)
  integer(c_int32_t) :: n(3)
  type(c_ptr) :: pe, pp, po
  real(dp), allocatable, target :: rho_c(:,:,:)
  n = int(shape(rho), c_int32_t)
  pe = c_null_ptr
  pp = c_null_ptr
  po = c_null_ptr
  if (present(efield)) pe = c_loc(efield)
  if (present(phi)) pp = c_loc(phi)
  if (present(offset)) po = c_loc(offset)
  rho_c = rho  ! contiguous copy (rho may be a strided section, e.g. the flipped image charge)
  call osc_check(c_freespace_solver2(osc_context(), n, rho_c, gamma, delta, po, osc_precision, pe, pp), &
      'osc_freespace_solver2')
end subroutine

! code/open_spacecharge_mod.f90:60-75
subroutine space_charge_freespace(mesh3d, direct_field_calc, integrated_green_function)
  type(mesh3d_struct) :: mesh3d
  logical, optional :: direct_field_calc, integrated_green_function
  integer :: idirect, igf
  idirect = 1
  igf = 1
  if (present(direct_field_calc)) then
    if (.not. direct_field_calc) idirect = 0
  endif
  if (present(integrated_green_function)) then
    if (.not. integrated_green_function) igf = 0
  endif
  call osc_freespace_solver(mesh3d%rho, mesh3d%gamma, mesh3d%delta, mesh3d%phi, mesh3d%efield, mesh3d%bfield, &
      mesh3d%nlo, mesh3d%nhi, mesh3d%nlo, mesh3d%nhi, mesh3d%npad, idirect, igf)
end subroutine

! code/open_spacecharge_mod.f90:83-103
subroutine space_charge_cathodeimages(mesh3d, direct_field_calc, integrated_green_function, image_method)
  type(mesh3d_struct) :: mesh3d
  logical, optional :: direct_field_calc, integrated_green_function
  integer, optional :: image_method
  integer :: idirect, igf, imethod
  idirect = 1
  igf = 1
  imethod = 1
  if (present(direct_field_calc)) then
    if (.not. direct_field_calc) idirect = 0
  endif
  if (present(integrated_green_function)) then
    if (.not. integrated_green_function) igf = 0
  endif
  if (present(image_method)) then
    if (image_method == 2) imethod = 2
  endif
  call osc_cathodeimages_solver(mesh3d%rho, mesh3d%gamma, mesh3d%min, mesh3d%delta, mesh3d%phi, mesh3d%efield, &
      mesh3d%bfield, mesh3d%nlo, mesh3d%nhi, mesh3d%nlo, mesh3d%nhi, mesh3d%npad, idirect, igf, imethod)
end subroutine

! code/open_spacecharge_mod.f90:110-127
subroutine space_charge_rectpipe(mesh3d, apipe, bpipe, direct_field_calc, integrated_green_function)
  type(mesh3d_struct) :: mesh3d
  real(dp) :: apipe, bpipe
  logical, optional :: direct_field_calc, integrated_green_function
  integer :: idirect, igf
  idirect = 1
  igf = 1
  if (present(direct_field_calc)) then
    if (.not. direct_field_calc) idirect = 0
  endif
  if (present(integrated_green_function)) then
    if (.not. integrated_green_function) igf = 0
  endif
  call osc_rectpipe_solver(mesh3d%rho, apipe, bpipe, mesh3d%gamma, mesh3d%delta, mesh3d%min, mesh3d%phi, &
      mesh3d%efield, mesh3d%bfield, mesh3d%nlo, mesh3d%nhi, mesh3d%nlo, mesh3d%nhi, idirect, igf)
end subroutine

!-----------------------------------------------------------------------------------------
! code/open_spacecharge_mod.f90:311-390: trilinear gather at one point, cells clamped to
! [1, nhi-1] with a message, weights from the unclamped position (host arithmetic).
subroutine interpolate_field(x, y, z, mesh3d, E, B)
  type(mesh3d_struct) :: mesh3d
  real(dp) :: x, y, z
  real(dp), optional :: E(3), B(3)
  real(dp) :: h(3), p(3), w(3)
  integer :: c(3), d
  p = [x, y, z]
  h = 1.0_dp / mesh3d%delta
  do d = 1, 3
    c(d) = floor((p(d) - mesh3d%min(d)) * h(d) + 1)
    if (c(d) < 1 .or. c(d) > mesh3d%nhi(d) - 1) then
      write(6, *) 'interpolate_field: cell index clamped on axis', d, ':', c(d), (p(d) - mesh3d%min(d)) * h(d)
      c(d) = max(1, min(c(d), mesh3d%nhi(d) - 1))
    endif
    w(d) = ((mesh3d%min(d) - p(d)) + c(d) * mesh3d%delta(d)) * h(d)
  enddo
  if (present(E)) E = gather(mesh3d%efield)
  if (present(B)) B = gather(mesh3d%bfield)
contains
  function gather(f) result(v)
    real(dp), intent(in) :: f(mesh3d%nlo(1):, mesh3d%nlo(2):, mesh3d%nlo(3):, :)
    real(dp) :: v(3)
    integer :: i, j, k
    real(dp) :: wx, wy, wz
    v = 0
    do k = 0, 1
      wz = merge(w(3), 1.0_dp - w(3), k == 0)
      do j = 0, 1
        wy = merge(w(2), 1.0_dp - w(2), j == 0)
        do i = 0, 1
          wx = merge(w(1), 1.0_dp - w(1), i == 0)
          v = v + f(c(1) + i, c(2) + j, c(3) + k, :) * (wx * wy * wz)
        enddo
      enddo
    enddo
  end function
end subroutine

! Many points at once on the GPU: E(:, n) (and B(:, n)) at (x(n), y(n), z(n)).
subroutine interpolate_field_batch(x, y, z, mesh3d, E, B)
  real(dp), intent(in) :: x(:), y(:), z(:)
  type(mesh3d_struct), target :: mesh3d
  real(dp), optional, target :: E(:,:), B(:,:)
  type(c_ptr) :: pe, pb, fe, fb
  integer(c_int64_t) :: ncl
  pe = c_null_ptr
  pb = c_null_ptr
  fe = c_null_ptr
  fb = c_null_ptr
  if (present(E)) then
    pe = c_loc(E)
    fe = c_loc(mesh3d%efield)
  endif
  if (present(B)) then
    pb = c_loc(B)
    fb = c_loc(mesh3d%bfield)
  endif
  call osc_check(c_interpolate_field(osc_context(), to_c(mesh3d), fe, fb, int(size(x), c_int64_t), x, y, z, pe, &
      pb, ncl), 'interpolate_field_batch')
end subroutine

end module open_spacecharge_mod
