!
! cfd2lcs_inc_sp.f90 -- Fortran include file of libcfd2lcs_b200, single precision build.
! Same names and values as the reference's src/cfd2lcs_inc_single.f90:15-69, so Fortran
! solvers that INCLUDE it and call cfd2lcs_init / cfd2lcs_diagnostic_init / cfd2lcs_update /
! cfd2lcs_set_option / cfd2lcs_set_param / cfd2lcs_diagnostic_destroy / cfd2lcs_finalize
! (external subroutines, gfortran-mangled) link against libcfd2lcs_b200_sp.so unchanged.
!
integer, parameter   :: LCSRP = 4
integer, parameter   :: LCSIP = 4
integer(LCSIP),parameter:: LCS_NAMELEN = 128
integer(LCSIP),parameter:: &
      LCS_INTERNAL = 0, &
      LCS_INFLOW = 1, &
      LCS_OUTFLOW = 2, &
      LCS_WALL = 3, &
      LCS_SLIP = 4, &
      LCS_2D = 5, &
      LCS_MASK = 6
integer(LCSIP),parameter:: &
      FTLE_FWD = 0, &
      FTLE_BKWD = 1, &
      LP_TRACER = 2
integer(LCSIP),parameter:: &
      EULER = 0, &
      TRAPEZOIDAL = 1, &
      RK2 = 2, &
      RK3 = 3, &
      RK4 = 4
integer(LCSIP),parameter:: &
      NEAREST_NBR = 0, &
      LINEAR = 1, &
      QUADRATIC = 2, &
      CUBIC = 3, &
      TSE = 5, &
      TSE_LIMIT = 6
integer(LCSIP),parameter:: &
      LCS_FALSE = 0, &
      LCS_TRUE = 1
