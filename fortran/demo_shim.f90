! Drives the drop-in modules the way the reference's test program drives its own
! (code/test_opensc.f90:156-228, free space): particles from a stream file, deposit with
! mesh refit, space_charge_3d with B, then interpolate_field at every particle; E is
! written as a stream file.  Usage: demo_shim <particles.bin> <E.bin>
program demo_shim
use open_spacecharge_mod
implicit none
integer, parameter :: dp = kind(1.d0)
real(dp), allocatable :: x(:), y(:), z(:)
type(mesh3d_struct) :: mesh
integer :: u, i
integer(8) :: np
real(dp) :: E(3)
character(len=512) :: fin, fout

call get_command_argument(1, fin)
call get_command_argument(2, fout)
open(newunit=u, file=trim(fin), access='stream', form='unformatted', status='old')
read(u) np
allocate(x(np), y(np), z(np))
read(u) x, y, z
close(u)

mesh%nhi = [24, 24, 32]
mesh%gamma = 9.784756683727565_dp
call deposit_particles(x, y, z, mesh, total_charge=1.0e-9_dp)
call space_charge_3d(mesh, calc_bfield=.true.)

open(newunit=u, file=trim(fout), access='stream', form='unformatted', status='replace')
do i = 1, int(np)
  call interpolate_field(x(i), y(i), z(i), mesh, E=E)
  write(u) E
enddo
close(u)
end program
