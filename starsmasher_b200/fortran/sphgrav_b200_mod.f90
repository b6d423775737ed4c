! sphgrav_b200_mod.f90 -- iso_c_binding interface to libsphgrav_b200 for the
! StarSmasher Fortran host (parallel_bleeding_edge/src).
!
! The three legacy symbols (firsthalf_grav_forces_, lasthalf_grav_forces_,
! gpu_init_dev_) need no interface: gfortran's implicit external calls in
! grav.f:25, balAV3.f:418 and main.f:270 resolve to them unchanged.  This
! module adds explicit interfaces for the status-returning and
! device-resident entry points, for callers that want error codes instead of
! an abort.  Compiled with the host code (no Fortran compiler was available
! where the library was built; the interface mirrors include/sphgrav_b200.h).
module sphgrav_b200_mod
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: SPHGRAV_OK = 0
  integer(c_int), parameter :: SPHGRAV_FP64 = 0, SPHGRAV_F32SPLIT = 1, SPHGRAV_TREE = 2

  interface
    integer(c_int) function sphgrav_create(ctx, device) bind(C, name="sphgrav_create")
      import :: c_int, c_ptr
      type(c_ptr), intent(out) :: ctx
      integer(c_int), value :: device
    end function

    integer(c_int) function sphgrav_destroy(ctx) bind(C, name="sphgrav_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    ! rows [i_begin, i_begin+ni) with 0-based i_begin
    integer(c_int) function sphgrav_firsthalf(ctx, n, i_begin, ni, x, y, z, mass, range2, &
                                              nkernel, precision) bind(C, name="sphgrav_firsthalf")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n, i_begin, ni, nkernel, precision
      real(c_double), intent(in) :: x(*), y(*), z(*), mass(*), range2(*)
    end function

    integer(c_int) function sphgrav_lasthalf(ctx, ax, ay, az, pot) bind(C, name="sphgrav_lasthalf")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: ax(*), ay(*), az(*), pot(*)
    end function

    ! grav.f:12-26 + balAV3.f:418 in one call: range2 built from hp and u
    integer(c_int) function sphgrav_gravforce(ctx, ntot, ngrav_lower, ngrav_upper, x, y, z, am, &
                                              hp, u, nkernel, precision, gx, gy, gz, grpot) &
                                              bind(C, name="sphgrav_gravforce")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ntot, ngrav_lower, ngrav_upper, nkernel, precision
      real(c_double), intent(in) :: x(*), y(*), z(*), am(*), hp(*), u(*)
      real(c_double), intent(inout) :: gx(*), gy(*), gz(*), grpot(*)
    end function

    ! device-resident form: every array argument is a device pointer (for
    ! example from OpenACC/CUDA Fortran, or c_loc of a managed array)
    integer(c_int) function sphgrav_gravforce_device(ctx, ntot, ngrav_lower, ngrav_upper, x, y, z, &
                                                     am, hp, u, nkernel, precision, gx, gy, gz, &
                                                     grpot) bind(C, name="sphgrav_gravforce_device")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: ntot, ngrav_lower, ngrav_upper, nkernel, precision
      type(c_ptr), value :: x, y, z, am, hp, u, gx, gy, gz, grpot
    end function

    integer(c_int) function sphgrav_batch_forces(ctx, nsets, offsets, x, y, z, mass, range2, &
                                                 nkernel, precision, ax, ay, az, pot, w) &
                                                 bind(C, name="sphgrav_batch_forces")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsets, nkernel, precision
      integer(c_int), intent(in) :: offsets(*)
      real(c_double), intent(in) :: x(*), y(*), z(*), mass(*), range2(*)
      real(c_double), intent(inout) :: ax(*), ay(*), az(*), pot(*), w(*)
    end function

    integer(c_int) function sphgrav_legacy_set_precision(precision) &
                                              bind(C, name="sphgrav_legacy_set_precision")
      import :: c_int
      integer(c_int), value :: precision
    end function

    ! SPHGRAV_TREE: opening angle in [0, 2] (gpu_init_dev_'s theta sets the
    ! legacy calls' angle)
    integer(c_int) function sphgrav_set_theta(ctx, theta) bind(C, name="sphgrav_set_theta")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: theta
    end function

    ! SPHGRAV_TREE: walking groups of the last call, and those handed to the
    ! direct FP64 sum
    integer(c_int) function sphgrav_tree_stats(ctx, groups, heavy) bind(C, name="sphgrav_tree_stats")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: groups, heavy
    end function

    type(c_ptr) function sphgrav_last_error_message() bind(C, name="sphgrav_last_error_message")
      import :: c_ptr
    end function
  end interface
end module sphgrav_b200_mod
