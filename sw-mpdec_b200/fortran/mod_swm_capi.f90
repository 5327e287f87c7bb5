!===============================================================================!
! MOD_SWM_CAPI -- ISO_C_BINDING interface of the sm_100a mPDeC5 time step
! (include/swm.h, libswm.so) for the reference's Fortran driver.
!
! The driver keeps t, dt, the output cadence and I/O.  Three edits in the
! reference make the library a drop-in for its time step:
!   timediscretization.f90:58     dt_min = TimeStep()       -> SWM_TimeStep()
!   timediscretization.f90:71-76  CALL TimeDiscretizationByMPDeC5/2(t)
!                                                           -> CALL SWM_Step(t)
!   timediscretization.f90:86 and main.f90:28, before WriteSolutionToDisk and
!   PostProcessing:              CALL SWM_Pull()  (copies U and V back)
! and one at start-up (after FillInitialConditions, main.f90:25):
!   CALL SWM_Init()              (parameters, state, well-balanced reference)
! Optionally the driver's initial condition, output and post-processing also run
! on the device: SWM_FillInitialConditions, SWM_WriteSolution(t), SWM_WriteMesh,
! SWM_PostProcessing (see the subroutines below).
! No Fortran compiler exists in the image this was written in; the interface
! follows the header's types one to one (c_int, c_double, c_ptr by value).
!===============================================================================!
MODULE MOD_SWM_CAPI
USE ISO_C_BINDING
IMPLICIT NONE
PRIVATE

TYPE, BIND(C), PUBLIC :: swm_params_t
  INTEGER(C_INT)  :: nx, ny
  REAL(C_DOUBLE)  :: x0(2), x1(2)
  REAL(C_DOUBLE)  :: g, cfl
  INTEGER(C_INT)  :: timescheme, bathy_flag
  REAL(C_DOUBLE)  :: bathy_par(5)
  INTEGER(C_INT)  :: well_balanced, precision, solver, jacobi_maxiter
  REAL(C_DOUBLE)  :: jacobi_tol
  INTEGER(C_INT)  :: jacobi_block, mpdec2_compat, use_graph, device
  INTEGER(C_INT)  :: source_table
END TYPE swm_params_t

TYPE, BIND(C), PUBLIC :: swm_stats_t
  INTEGER(C_INT)     :: status, n_solves
  INTEGER(C_INT)     :: jacobi_iters(16)
  INTEGER(C_INT)     :: jacobi_iters_min, jacobi_iters_max
  INTEGER(C_LONG_LONG) :: jacobi_iters_total, steps
  REAL(C_DOUBLE)     :: lambda_max(2)
END TYPE swm_stats_t

INTERFACE
  INTEGER(C_INT) FUNCTION swm_params_default(p, nx, ny, x00, x01, x10, x11) &
      BIND(C, NAME="swm_params_default")
    IMPORT :: C_INT, C_DOUBLE, swm_params_t
    TYPE(swm_params_t), INTENT(OUT) :: p
    INTEGER(C_INT), VALUE :: nx, ny
    REAL(C_DOUBLE), VALUE :: x00, x01, x10, x11
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_create(p, h) BIND(C, NAME="swm_create")
    IMPORT :: C_INT, C_PTR, swm_params_t
    TYPE(swm_params_t), INTENT(IN) :: p
    TYPE(C_PTR), INTENT(OUT) :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_destroy(h) BIND(C, NAME="swm_destroy")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_set_state(h, U) BIND(C, NAME="swm_set_state")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(IN) :: U(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_get_state(h, U, V) BIND(C, NAME="swm_get_state")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: U(*), V(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_set_wb_state(h, Uwb) BIND(C, NAME="swm_set_wb_state")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(IN) :: Uwb(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_timestep(h, dt_min) BIND(C, NAME="swm_timestep")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: dt_min
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_step(h, t, dt) BIND(C, NAME="swm_step")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: t, dt
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_get_stats(h, s) BIND(C, NAME="swm_get_stats")
    IMPORT :: C_INT, C_PTR, swm_stats_t
    TYPE(C_PTR), VALUE :: h
    TYPE(swm_stats_t), INTENT(OUT) :: s
  END FUNCTION
  TYPE(C_PTR) FUNCTION swm_last_error() BIND(C, NAME="swm_last_error")
    IMPORT :: C_PTR
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_fill_ic(h, ic, par, npar) BIND(C, NAME="swm_fill_ic")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: ic, npar
    REAL(C_DOUBLE), INTENT(IN) :: par(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_init_wb_ic(h, ic, par, npar) BIND(C, NAME="swm_init_wb_ic")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: ic, npar
    REAL(C_DOUBLE), INTENT(IN) :: par(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_l1_error(h, ic, par, npar, t, l1) BIND(C, NAME="swm_l1_error")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: ic, npar
    REAL(C_DOUBLE), INTENT(IN) :: par(*)
    REAL(C_DOUBLE), VALUE :: t
    REAL(C_DOUBLE), INTENT(OUT) :: l1(3)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_write_output(h, t, which, ic, par, npar, dir, flags) &
      BIND(C, NAME="swm_write_output")
    IMPORT :: C_INT, C_PTR, C_DOUBLE, C_CHAR
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: t
    INTEGER(C_INT), VALUE :: which, ic, npar, flags
    REAL(C_DOUBLE), INTENT(IN) :: par(*)
    CHARACTER(KIND=C_CHAR), INTENT(IN) :: dir(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION swm_write_mesh(h, dir) BIND(C, NAME="swm_write_mesh")
    IMPORT :: C_INT, C_PTR, C_CHAR
    TYPE(C_PTR), VALUE :: h
    CHARACTER(KIND=C_CHAR), INTENT(IN) :: dir(*)
  END FUNCTION
END INTERFACE

TYPE(C_PTR), SAVE :: handle = C_NULL_PTR

PUBLIC :: SWM_Init, SWM_TimeStep, SWM_Step, SWM_Pull, SWM_Finalize
PUBLIC :: SWM_FillInitialConditions, SWM_WriteSolution, SWM_WriteMesh, SWM_PostProcessing

CONTAINS

! Error convention (include/swm.h): >0 warning (printed, as jacobi_iteration.f90:83-85),
! <0 error (printed, then STOP as parameters.f90:123-126 does).
SUBROUTINE SWM_Check(rc, where)
  INTEGER(C_INT), INTENT(IN) :: rc
  CHARACTER(LEN=*), INTENT(IN) :: where
  CHARACTER(KIND=C_CHAR), POINTER :: msg(:)
  CHARACTER(LEN=256) :: text
  INTEGER :: k
  IF (rc == 0) RETURN
  CALL C_F_POINTER(swm_last_error(), msg, [256])
  text = ' '
  DO k = 1, 256
    IF (msg(k) == C_NULL_CHAR) EXIT
    text(k:k) = msg(k)
  END DO
  IF (rc > 0) THEN
    PRINT*, where, ": ", TRIM(text)
  ELSE
    PRINT*, where, " failed: ", TRIM(text)
    STOP
  END IF
END SUBROUTINE SWM_Check

! Parameters from the reference module globals (parameters.f90:62-147).
SUBROUTINE SWM_Init()
  USE MOD_FiniteVolume2D_vars
  TYPE(swm_params_t) :: p
  CALL SWM_Check(swm_params_default(p, INT(nElemsX, C_INT), INT(nElemsY, C_INT), &
                 MESH_X0(1), MESH_X0(2), MESH_X1(1), MESH_X1(2)), "swm_params_default")
  p%g = Gravity
  p%cfl = CFL
  p%timescheme = timescheme
  p%bathy_flag = BathymetryFlag
#ifdef WELLBALANCED
  p%well_balanced = 1
#endif
  CALL SWM_Check(swm_create(p, handle), "swm_create")
#ifdef WELLBALANCED
  ! UWB cell averages must be in U here (InitializeWBVariables, finitevolume.f90:373-385)
#endif
  CALL SWM_Check(swm_set_state(handle, U), "swm_set_state")
END SUBROUTINE SWM_Init

REAL FUNCTION SWM_TimeStep()
  REAL(C_DOUBLE) :: dt_min
  CALL SWM_Check(swm_timestep(handle, dt_min), "swm_timestep")
  SWM_TimeStep = dt_min
END FUNCTION SWM_TimeStep

SUBROUTINE SWM_Step(t)
  USE MOD_FiniteVolume2D_vars, ONLY: dt
  REAL, INTENT(IN) :: t
  CALL SWM_Check(swm_step(handle, REAL(t, C_DOUBLE), REAL(dt, C_DOUBLE)), "swm_step")
END SUBROUTINE SWM_Step

SUBROUTINE SWM_Pull()
  USE MOD_FiniteVolume2D_vars, ONLY: U, V
  CALL SWM_Check(swm_get_state(handle, U, V), "swm_get_state")
END SUBROUTINE SWM_Pull

! Optional device-side replacements of the driver's initialisation and output
! (reference cases 1..6 of ExactFunction; no parameters).
! CALL FillInitialConditions() (main.f90:23) -> CALL SWM_FillInitialConditions()
SUBROUTINE SWM_FillInitialConditions()
  USE MOD_FiniteVolume2D_vars, ONLY: InitialCondition
  REAL(C_DOUBLE) :: par(1)
  par = 0.0_C_DOUBLE
  CALL SWM_Check(swm_fill_ic(handle, INT(InitialCondition, C_INT), par, 0_C_INT), &
                 "swm_fill_ic")
END SUBROUTINE SWM_FillInitialConditions

! CALL WriteSolutionToDisk(t) (timediscretization.f90:52,87) -> CALL SWM_WriteSolution(t)
SUBROUTINE SWM_WriteSolution(t)
  USE MOD_FiniteVolume2D_vars, ONLY: InitialCondition, WhichOutput
  REAL, INTENT(IN) :: t
  REAL(C_DOUBLE) :: par(1)
  par = 0.0_C_DOUBLE
  IF (WhichOutput < 1 .OR. WhichOutput > 3) RETURN
  CALL SWM_Check(swm_write_output(handle, REAL(t, C_DOUBLE), INT(WhichOutput, C_INT), &
                 INT(InitialCondition, C_INT), par, 0_C_INT, "."//C_NULL_CHAR, 0_C_INT), &
                 "swm_write_output")
END SUBROUTINE SWM_WriteSolution

! CALL WriteMeshToDisk() (timediscretization.f90:50) -> CALL SWM_WriteMesh()
SUBROUTINE SWM_WriteMesh()
  CALL SWM_Check(swm_write_mesh(handle, "."//C_NULL_CHAR), "swm_write_mesh")
END SUBROUTINE SWM_WriteMesh

! CALL PostProcessing() (main.f90:28): the L1 error at tEnd, written as
! ErrorL1_XXXX_XXXX.dat (postprocessing.f90:52-58)
SUBROUTINE SWM_PostProcessing()
  USE MOD_FiniteVolume2D_vars, ONLY: InitialCondition, tEnd, nElemsX, nElemsY
  REAL(C_DOUBLE) :: par(1), l1(3)
  CHARACTER(LEN=255) :: FNAME
  par = 0.0_C_DOUBLE
  CALL SWM_Check(swm_l1_error(handle, INT(InitialCondition, C_INT), par, 0_C_INT, &
                 REAL(tEnd, C_DOUBLE), l1), "swm_l1_error")
  FNAME = 'ErrorL1_XXXX_XXXX.dat'
  WRITE(FNAME(9:12),FMT="(I4.4)") nElemsX
  WRITE(FNAME(14:17),FMT="(I4.4)") nElemsY
  OPEN(666,FILE=TRIM(FNAME))
  WRITE(666,*) l1(1:3)
  CLOSE(666)
END SUBROUTINE SWM_PostProcessing

SUBROUTINE SWM_Finalize()
  INTEGER(C_INT) :: rc
  rc = swm_destroy(handle)
  handle = C_NULL_PTR
END SUBROUTINE SWM_Finalize

END MODULE MOD_SWM_CAPI
