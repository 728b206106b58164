!  Drop-in replacements for bipoly_hydro's potsetup and potential_solver
!  (potsetup.F90:6, potential_solver.F90:6).  Same names, same empty
!  argument lists, same COMMON blocks; the work is done by libbph.so (the
!  B200 solver) through its C ABI (include/bph.h).  Link this file instead
!  of potential_solver.F90, helmadi.F90, realft.F90, tridagr.F90,
!  tridagz.F90, bessel.F90, potsetup.F90, tm.F90, sm.F90, bm.F90, elle.F90,
!  ellf.F90, rd.F90, rf.F90, gammln.F90 and the four swap_* files, and add
!  -L<dir> -lbph to the link line.
!
!  One rank owns the whole (r,z) grid: numr_dd = numr, numz_dd = numz.
!  A non-zero status stops the run, as rf/rd's STOP did.
module bph_c
   use iso_c_binding
   implicit none
   type, bind(c) :: bph_grid_t
      integer(c_int) :: numr, numz, numphi
      real(c_double) :: dr
      integer(c_int) :: isym, mmax
   end type bph_grid_t
   interface
      integer(c_int) function bph_setup(grid, ctx) bind(c, name="bph_setup")
         import :: c_int, c_ptr, bph_grid_t
         type(bph_grid_t), intent(in) :: grid
         type(c_ptr), intent(out) :: ctx
      end function bph_setup
      integer(c_int) function bph_potential_solver(ctx, rho, pot, tstep) &
            bind(c, name="bph_potential_solver")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: rho(*)
         real(c_double), intent(out) :: pot(*)
         integer(c_int), value :: tstep
      end function bph_potential_solver
      integer(c_int) function bph_register_host(a, bytes) bind(c, name="bph_register_host")
         import :: c_int, c_double, c_size_t
         real(c_double), intent(in) :: a(*)
         integer(c_size_t), value :: bytes
      end function bph_register_host
      integer(c_int) function bph_restore_continuation(ctx, path, rho) &
            bind(c, name="bph_restore_continuation")
         import :: c_int, c_ptr, c_char
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
         type(c_ptr), value :: rho
      end function bph_restore_continuation
      type(c_ptr) function bph_last_error() bind(c, name="bph_last_error")
         import :: c_ptr
      end function bph_last_error
   end interface
   type(c_ptr), save :: bph_context = c_null_ptr
end module bph_c

subroutine potsetup
   use bph_c
   implicit none
   include 'runhydro.h'
   include 'pot.h'
   real :: dr, dz, dphi, drinv, dzinv, dphiinv
   common /coord_differentials/ dr, dz, dphi, drinv, dzinv, dphiinv
   integer :: isym
   integer, dimension(3) :: boundary_condition
   common /boundary_conditions/ isym, boundary_condition
   real, dimension(numr_dd,numz_dd,numphi) :: pot, rho
   common /poisson/ pot, rho
   type(bph_grid_t) :: grid
   integer(c_int) :: rc
   integer(c_size_t) :: nbytes
   grid = bph_grid_t(numr, numz, numphi, real(dr, c_double), isym, mmax)
   rc = bph_setup(grid, bph_context)
   if (rc /= 0) then
      write(6,*) 'bph_setup failed with status ', rc
      error stop
   endif
   ! COMMON /poisson/ lives at a fixed address for the whole run: pin it once
   ! so that every potential_solver call copies at pinned-memory speed
   nbytes = int(8, c_size_t) * int(numr_dd, c_size_t) * int(numz_dd, c_size_t) * int(numphi, c_size_t)
   rc = bph_register_host(rho, nbytes)
   if (rc == 0) rc = bph_register_host(pot, nbytes)
   if (rc /= 0) then
      write(6,*) 'bph_register_host failed with status ', rc
      error stop
   endif
end subroutine potsetup

subroutine potential_solver
   use bph_c
   implicit none
   include 'runhydro.h'
   real, dimension(numr_dd,numz_dd,numphi) :: pot, rho
   common /poisson/ pot, rho
   real :: dt, time, dt_visc
   integer :: tstep
   common /timestep/ dt, time, dt_visc, tstep
   integer(c_int) :: rc
   rc = bph_potential_solver(bph_context, rho, pot, int(tstep, c_int))
   if (rc /= 0) then
      write(6,*) 'bph_potential_solver failed with status ', rc
      error stop
   endif
end subroutine potential_solver
