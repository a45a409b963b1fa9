!-------------------------------------------------------------------------------
! hecmw_solver_gpu33.f90 -- Fortran binding of the B200 3x3-block CG solver
! (include/hecmw33_gpu.h) for FrontISTR's hecmw1.
!
! It replaces, for NDOF=3 and METHOD=1 (CG), the call
!     call hecmw_solve_iterative(hecMESH, hecMAT)
! inside hecmw_solve (hecmw1/src/solver/main/hecmw_solver.f90:39-42) with
!     call hecmw_solve_gpu33(hecMESH, hecMAT)
! keeping hecmw_solve's signature and the hecmwST_matrix layout: the arrays are
! passed by reference, unchanged.  The C side runs the zero-RHS and zero-diagonal
! checks, the preconditioner recycle policy (flags 96/97/98), the preconditioner
! setup, CG, the true residual and the converged/diverged flags, as
! hecmw_solve + hecmw_solve_iterative do.
!
! One GPU domain only: hecMAT%N must equal hecMAT%NP (no halo exchange).
! This file is not compiled in this repository (no Fortran compiler on the
! build image); the same entry points are exercised from C and Python.
!-------------------------------------------------------------------------------
module hecmw_solver_gpu33
  use iso_c_binding
  use hecmw_util
  use hecmw_matrix_dump
  use m_hecmw_solve_error
  implicit none
  private
  public :: hecmw_solve_gpu33
  public :: hecmw_solve_gpu33_finalize

  integer(c_int), save :: gpu_handle = 0

  interface
    subroutine hecmw33_gpu_create(handle, ierr) bind(C, name="hecmw33_gpu_create")
      import :: c_int
      integer(c_int), intent(out) :: handle, ierr
    end subroutine hecmw33_gpu_create

    subroutine hecmw33_gpu_destroy(handle, ierr) bind(C, name="hecmw33_gpu_destroy")
      import :: c_int
      integer(c_int), intent(in) :: handle
      integer(c_int), intent(out) :: ierr
    end subroutine hecmw33_gpu_destroy

    subroutine hecmw33_gpu_solve(handle, N, NP, NPL, NPU, indexL, itemL, indexU, itemU, &
        D, AL, AU, B, X, Iarray, Rarray, iter, resid, times, ierr) bind(C, name="hecmw33_gpu_solve")
      import :: c_int, c_double
      integer(c_int), intent(in) :: handle, N, NP, NPL, NPU
      integer(c_int), intent(in) :: indexL(*), itemL(*), indexU(*), itemU(*)
      real(c_double), intent(in) :: D(*), AL(*), AU(*), B(*)
      real(c_double), intent(inout) :: X(*)
      integer(c_int), intent(inout) :: Iarray(100)
      real(c_double), intent(inout) :: Rarray(100)
      integer(c_int), intent(out) :: iter, ierr
      real(c_double), intent(out) :: resid, times(3)
    end subroutine hecmw33_gpu_solve
  end interface

contains

  subroutine hecmw_solve_gpu33(hecMESH, hecMAT)
    type(hecmwST_local_mesh) :: hecMESH
    type(hecmwST_matrix), target :: hecMAT
    integer(c_int) :: ierr, iter
    real(c_double) :: resid, times(3)

    if (hecMAT%NDOF /= 3 .or. hecMAT%N /= hecMAT%NP) then
      ierr = HECMW_SOLVER_ERROR_INCONS_PC
      call hecmw_solve_error(hecMESH, ierr)
      return
    endif
    if (gpu_handle == 0) then
      call hecmw33_gpu_create(gpu_handle, ierr)
      if (ierr /= 0) call hecmw_abort(hecmw_comm_get_comm())
    endif
    ! hecmw_solve_iterative dumps the matrix and right-hand side before the solve
    ! (hecmw_solver_Iterative.f90:90, DUMPTYPE of !SOLVER) and the solution after it
    ! (:160); both return at once when no dump is requested
    call hecmw_mat_dump(hecMAT, hecMESH)
    call hecmw33_gpu_solve(gpu_handle, hecMAT%N, hecMAT%NP, hecMAT%indexL(hecMAT%N), &
      hecMAT%indexU(hecMAT%N), hecMAT%indexL, hecMAT%itemL, hecMAT%indexU, hecMAT%itemU, &
      hecMAT%D, hecMAT%AL, hecMAT%AU, hecMAT%B, hecMAT%X, hecMAT%Iarray, hecMAT%Rarray, &
      iter, resid, times, ierr)
    call hecmw_mat_dump_solution(hecMAT)
    if (hecmw_mat_get_timelog(hecMAT) >= 1 .and. hecMESH%my_rank == 0) then
      write (*,'(/a)')          '### summary of linear solver (GPU)'
      write (*,'(i10,a, 1pe16.6)')      iter, ' iterations  ', resid
      write (*,'(a, 1pe16.6 )') '    set-up time      : ', times(1)
      write (*,'(a, 1pe16.6 )') '    solver time      : ', times(2)
    endif
    ! 1001/2001 abort, 2002/3001 warn, 3002-3004 are reported through the diverged flag
    if (ierr /= 0 .and. ierr < 9000) call hecmw_solve_error(hecMESH, ierr)
    if (ierr >= 9000) call hecmw_abort(hecmw_comm_get_comm())
  end subroutine hecmw_solve_gpu33

  subroutine hecmw_solve_gpu33_finalize()
    integer(c_int) :: ierr
    if (gpu_handle /= 0) call hecmw33_gpu_destroy(gpu_handle, ierr)
    gpu_handle = 0
  end subroutine hecmw_solve_gpu33_finalize

end module hecmw_solver_gpu33
