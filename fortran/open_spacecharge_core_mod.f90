!-----------------------------------------------------------------------------------------
! open_spacecharge_core_mod (drop-in): the legacy solvers and the rectangular-pipe Green
! function routines of code/open_spacecharge_core_mod.f90, with the same names and dummy
! arguments, forwarded to libopensc_b200.so (include/opensc_gpu.h) through iso_c_binding.
!
! The reference keeps the transformed pipe Green arrays cgrn1..4 in module variables
! (code/open_spacecharge_core_mod.f90:22-23); here they live on the library context, which
! this module creates on first use (device osc_device, default 0).  Solves run in
! osc_precision (default OSC_PREC_FP64; osc_set_precision changes it).
!-----------------------------------------------------------------------------------------
module open_spacecharge_core_mod

use, intrinsic :: iso_c_binding
use, intrinsic :: iso_fortran_env

implicit none

integer, parameter, private :: dp = REAL64

! bind(C) twin of osc_mesh3d (include/opensc_gpu.h)
type, bind(C) :: osc_mesh3d_c
  integer(c_int32_t) :: nlo(3), nhi(3), npad(3)
  real(c_double) :: min(3), max(3), delta(3)
  real(c_double) :: gamma, charge
end type

integer(c_int), parameter :: OSC_PREC_FP32 = 0, OSC_PREC_FP64 = 1, OSC_PREC_FP64_PLAIN = 2
integer(c_int), parameter :: OSC_OK = 0, OSC_E_NOCHARGE = 8

type(c_ptr), save :: osc_ctx = c_null_ptr
integer(c_int), save :: osc_device = 0
integer(c_int), save :: osc_precision = OSC_PREC_FP64

! geometry recorded by osc_alloc_rectpipe_arrays for the later pipe calls
integer, save, private :: pipe_nlo(3) = 1, pipe_nhi(3) = 1, pipe_npad(3) = 1
real(dp), save, private :: pipe_delta(3) = 0, pipe_umin(3) = 0, pipe_gamma = 1

interface
  integer(c_int) function c_ctx_create(device, ctx) bind(C, name="osc_ctx_create")
    import :: c_int, c_ptr
    integer(c_int), value :: device
    type(c_ptr) :: ctx
  end function
  type(c_ptr) function c_last_error(ctx) bind(C, name="osc_last_error")
    import :: c_ptr
    type(c_ptr), value :: ctx
  end function
  integer(c_int) function c_space_charge_freespace(ctx, mesh, rho, direct, igf, prec, phi, efield, bfield) &
      bind(C, name="osc_space_charge_freespace")
    import :: c_ptr, c_int, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    type(osc_mesh3d_c), intent(in) :: mesh
    real(c_double), intent(in) :: rho(*)
    integer(c_int), value :: direct, igf, prec
    real(c_double) :: phi(*), efield(*), bfield(*)
  end function
  integer(c_int) function c_space_charge_cathodeimages(ctx, mesh, rho, direct, igf, method, prec, phi, efield, &
      bfield) bind(C, name="osc_space_charge_cathodeimages")
    import :: c_ptr, c_int, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    type(osc_mesh3d_c), intent(in) :: mesh
    real(c_double) :: rho(*)
    integer(c_int), value :: direct, igf, method, prec
    real(c_double) :: phi(*), efield(*), bfield(*)
  end function
  integer(c_int) function c_rectpipe_green(ctx, mesh, apipe, bpipe, prec) bind(C, name="osc_rectpipe_green")
    import :: c_ptr, c_int, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    type(osc_mesh3d_c), intent(in) :: mesh
    real(c_double), value :: apipe, bpipe
    integer(c_int), value :: prec
  end function
  integer(c_int) function c_space_charge_rectpipe(ctx, mesh, rho, apipe, bpipe, direct, igf, prec, phi, efield, &
      bfield) bind(C, name="osc_space_charge_rectpipe")
    import :: c_ptr, c_int, c_double, osc_mesh3d_c
    type(c_ptr), value :: ctx
    type(osc_mesh3d_c), intent(in) :: mesh
    real(c_double), intent(in) :: rho(*)
    real(c_double), value :: apipe, bpipe
    integer(c_int), value :: direct, igf, prec
    real(c_double) :: phi(*), efield(*), bfield(*)
  end function
  integer(c_int) function c_write_rectpipe_grn(ctx, path, apipe, bpipe, mesh) bind(C, name="osc_write_rectpipe_grn")
    import :: c_ptr, c_int, c_double, c_char, osc_mesh3d_c
    type(c_ptr), value :: ctx
    character(kind=c_char), intent(in) :: path(*)
    real(c_double), value :: apipe, bpipe
    type(osc_mesh3d_c), intent(in) :: mesh
  end function
  integer(c_int) function c_read_rectpipe_grn(ctx, path, mesh, apipe, bpipe) bind(C, name="osc_read_rectpipe_grn")
    import :: c_ptr, c_int, c_double, c_char, osc_mesh3d_c
    type(c_ptr), value :: ctx
    character(kind=c_char), intent(in) :: path(*)
    type(osc_mesh3d_c), intent(in) :: mesh
    real(c_double) :: apipe, bpipe
  end function
end interface

contains

!-----------------------------------------------------------------------------------------
! Library context of this process (created on first use).
function osc_context() result(ctx)
  type(c_ptr) :: ctx
  integer(c_int) :: rc
  if (.not. c_associated(osc_ctx)) then
    rc = c_ctx_create(osc_device, osc_ctx)
    if (rc /= OSC_OK) then
      write(6, *) 'open_spacecharge: no CUDA device for the space-charge library (status ', rc, ')'
      error stop
    endif
  endif
  ctx = osc_ctx
end function

subroutine osc_set_precision(precision)
  integer, intent(in) :: precision
  osc_precision = int(precision, c_int)
end subroutine

! Last error message of the context as a Fortran string.
function osc_error_message() result(msg)
  character(len=:), allocatable :: msg
  type(c_ptr) :: p
  character(kind=c_char), pointer :: s(:)
  integer :: n
  p = c_last_error(osc_ctx)
  msg = ''
  if (.not. c_associated(p)) return
  call c_f_pointer(p, s, [4096])
  n = 0
  do while (n < 4096)
    if (s(n + 1) == c_null_char) exit
    n = n + 1
  enddo
  allocate(character(len=n) :: msg)
  msg = transfer(s(1:n), msg)
end function

! Non-zero statuses print the library's message and stop, as the reference stops on errors.
subroutine osc_check(rc, what)
  integer(c_int), intent(in) :: rc
  character(len=*), intent(in) :: what
  if (rc == OSC_OK) return
  write(6, *) what, ': ', osc_error_message()
  error stop
end subroutine

function osc_mesh(nlo, nhi, npad, umin, delta, gamma) result(m)
  integer, intent(in) :: nlo(3), nhi(3), npad(3)
  real(dp), intent(in) :: umin(3), delta(3), gamma
  type(osc_mesh3d_c) :: m
  m%nlo = int(nlo, c_int32_t)
  m%nhi = int(nhi, c_int32_t)
  m%npad = int(npad, c_int32_t)
  m%min = umin
  m%delta = delta
  m%max = umin + (nhi - nlo) * delta
  m%gamma = gamma
  m%charge = 0
end function

!-----------------------------------------------------------------------------------------
! code/open_spacecharge_core_mod.f90:30 (legacy free space, npad-based wrap)
subroutine osc_freespace_solver(rho,gam0,delta,phi,efield,bfield,nlo,nhi,nlo_gbl,nhi_gbl,npad,idirectfieldcalc,igfflag)
  integer, intent(in) :: igfflag, idirectfieldcalc
  real(dp), intent(in), dimension(3) :: delta
  integer, intent(in), dimension(3) :: nlo, nhi, nlo_gbl, nhi_gbl, npad
  real(dp), intent(in) :: gam0
  real(dp), intent(in), dimension(:,:,:) :: rho
  real(dp), intent(out), dimension(:,:,:) :: phi
  real(dp), intent(out), dimension(:,:,:,:) :: efield, bfield
  type(osc_mesh3d_c) :: m
  real(dp) :: zero3(3) = 0
  m = osc_mesh(nlo, nhi, npad, zero3, delta, gam0)
  call osc_check(c_space_charge_freespace(osc_context(), m, rho, int(idirectfieldcalc, c_int), &
      int(igfflag, c_int), osc_precision, phi, efield, bfield), 'osc_freespace_solver')
end subroutine

! code/open_spacecharge_core_mod.f90:905 (legacy cathode images, methods 1 and 2)
subroutine osc_cathodeimages_solver(rho,gam0,umin,delta,phi,efield,bfield,nlo,nhi,nlo_gbl,nhi_gbl,npad, &
    idirectfieldcalc,igfflag,imethod)
  integer, intent(in) :: igfflag, idirectfieldcalc, imethod
  real(dp), intent(in), dimension(3) :: umin, delta
  integer, intent(in), dimension(3) :: nlo, nhi, nlo_gbl, nhi_gbl, npad
  real(dp), intent(in) :: gam0
  real(dp), dimension(:,:,:) :: rho
  real(dp), intent(out), dimension(:,:,:) :: phi
  real(dp), intent(out), dimension(:,:,:,:) :: efield, bfield
  type(osc_mesh3d_c) :: m
  m = osc_mesh(nlo, nhi, npad, umin, delta, gam0)
  call osc_check(c_space_charge_cathodeimages(osc_context(), m, rho, int(idirectfieldcalc, c_int), &
      int(igfflag, c_int), int(imethod, c_int), osc_precision, phi, efield, bfield), 'osc_cathodeimages_solver')
end subroutine

! code/open_spacecharge_core_mod.f90:876: records the pipe geometry (the arrays themselves
! are allocated by the library when osc_getgrnpipe or osc_read_rectpipe_grn runs).
subroutine osc_alloc_rectpipe_arrays(nlo,nhi,npad)
  integer, intent(in), dimension(3) :: nlo, nhi, npad
  pipe_nlo = nlo
  pipe_nhi = nhi
  pipe_npad = npad
end subroutine

! code/open_spacecharge_core_mod.f90:632
subroutine osc_getgrnpipe(gam,a,b,delta,umin,npad)
  real(dp), dimension(3) :: delta, umin
  integer, dimension(3) :: npad
  real(dp) :: gam, a, b
  type(osc_mesh3d_c) :: m
  pipe_npad = npad
  pipe_delta = delta
  pipe_umin = umin
  pipe_gamma = gam
  m = osc_mesh(pipe_nlo, pipe_nhi, pipe_npad, umin, delta, gam)
  call osc_check(c_rectpipe_green(osc_context(), m, a, b, osc_precision), 'osc_getgrnpipe')
end subroutine

! code/open_spacecharge_core_mod.f90:536
subroutine osc_rectpipe_solver(rho,a,b,gam0,delta,umin,phi,efield,bfield,nlo,nhi,nlo_gbl,nhi_gbl, &
    idirectfieldcalc,igfflag)
  integer, intent(in) :: igfflag, idirectfieldcalc
  real(dp), intent(in) :: a, b, gam0
  real(dp), intent(in), dimension(3) :: delta, umin
  integer, intent(in), dimension(3) :: nlo, nhi, nlo_gbl, nhi_gbl
  real(dp), intent(in), dimension(:,:,:) :: rho
  real(dp), intent(out), dimension(:,:,:) :: phi
  real(dp), intent(out), dimension(:,:,:,:) :: efield, bfield
  type(osc_mesh3d_c) :: m
  m = osc_mesh(nlo, nhi, pipe_npad, umin, delta, gam0)
  call osc_check(c_space_charge_rectpipe(osc_context(), m, rho, a, b, int(idirectfieldcalc, c_int), &
      int(igfflag, c_int), osc_precision, phi, efield, bfield), 'osc_rectpipe_solver')
end subroutine

! code/open_spacecharge_core_mod.f90:851: rectpipegrn.dat in the working directory
subroutine osc_write_rectpipe_grn(apipe,bpipe,delta,umin,umax,nlo,nhi,gamma)
  real(dp) :: apipe, bpipe, gamma
  real(dp), dimension(3) :: delta, umin, umax
  integer, dimension(3) :: nlo, nhi
  type(osc_mesh3d_c) :: m
  m = osc_mesh(nlo, nhi, pipe_npad, umin, delta, gamma)
  m%max = umax
  call osc_check(c_write_rectpipe_grn(osc_context(), 'rectpipegrn.dat'//c_null_char, apipe, bpipe, m), &
      'osc_write_rectpipe_grn')
end subroutine

! code/open_spacecharge_core_mod.f90:825: rectpipegrn.dat from the working directory, for
! the geometry recorded by osc_alloc_rectpipe_arrays
subroutine osc_read_rectpipe_grn
  type(osc_mesh3d_c) :: m
  real(c_double) :: a, b
  m = osc_mesh(pipe_nlo, pipe_nhi, pipe_npad, pipe_umin, pipe_delta, pipe_gamma)
  call osc_check(c_read_rectpipe_grn(osc_context(), 'rectpipegrn.dat'//c_null_char, m, a, b), &
      'osc_read_rectpipe_grn')
  write(6, *) 'Done reading rectpipe transformed Green functions with these parameters:'
  write(6, *) 'apipe,bpipe=', a, b
end subroutine

end module open_spacecharge_core_mod
