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
! A domain of a distributed run (hecMAT%N < hecMAT%NP) registers its communication
! table (hecMESH%n_neighbor_pe, neighbor_pe, import_*/export_*) with
! hecmw33_gpu_set_domain; the C side calls back gpu33_exchange (hecmw_update_R
! through the mesh's own hecmw_solve_send_recv) and gpu33_allreduce
! (hecmw_allreduce_R1) at the points where hecmw_solve_CG communicates.
! This file is not compiled in this repository (no Fortran compiler on the
! build image); the same entry points are exercised from C and Python.
!-------------------------------------------------------------------------------
module hecmw_solver_gpu33
  use iso_c_binding
  use hecmw_util
  use hecmw_matrix_dump
  use m_hecmw_solve_error
  use m_hecmw_comm_f
  implicit none
  private
  public :: hecmw_solve_gpu33
  public :: hecmw_solve_gpu33_finalize

  integer(c_int), save :: gpu_handle = 0
  ! the mesh of the solve in progress, for the communication callbacks
  type(hecmwST_local_mesh), pointer, save :: cb_mesh => null()
  integer(kind=kint), save :: cb_np = 0

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

    subroutine hecmw33_gpu_set_matrix(handle, N, NP, NPL, NPU, indexL, itemL, indexU, itemU, &
        D, AL, AU, Iarray, ierr) bind(C, name="hecmw33_gpu_set_matrix")
      import :: c_int, c_double
      integer(c_int), intent(in) :: handle, N, NP, NPL, NPU
      integer(c_int), intent(in) :: indexL(*), itemL(*), indexU(*), itemU(*), Iarray(100)
      real(c_double), intent(in) :: D(*), AL(*), AU(*)
      integer(c_int), intent(out) :: ierr
    end subroutine hecmw33_gpu_set_matrix

    subroutine hecmw33_gpu_set_domain(handle, n_neighbor_pe, neighbor_pe, import_index, import_item, &
        export_index, export_item, exchange, allreduce, ctx, ierr) bind(C, name="hecmw33_gpu_set_domain")
      import :: c_int, c_funptr, c_ptr
      integer(c_int), intent(in) :: handle, n_neighbor_pe
      integer(c_int), intent(in) :: neighbor_pe(*), import_index(*), import_item(*)
      integer(c_int), intent(in) :: export_index(*), export_item(*)
      type(c_funptr), value :: exchange, allreduce
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: ierr
    end subroutine hecmw33_gpu_set_domain

    subroutine hecmw33_gpu_set_mpc(handle, n_mpc, mpc_index, mpc_item, mpc_dof, mpc_val, mpc_const, ierr) &
        bind(C, name="hecmw33_gpu_set_mpc")
      import :: c_int, c_double
      integer(c_int), intent(in) :: handle, n_mpc
      integer(c_int), intent(in) :: mpc_index(*), mpc_item(*), mpc_dof(*)
      real(c_double), intent(in) :: mpc_val(*), mpc_const(*)
      integer(c_int), intent(out) :: ierr
    end subroutine hecmw33_gpu_set_mpc

    subroutine hecmw33_gpu_solve_resident(handle, B, X, Iarray, Rarray, iter, resid, times, ierr) &
        bind(C, name="hecmw33_gpu_solve_resident")
      import :: c_int, c_double
      integer(c_int), intent(in) :: handle
      real(c_double), intent(in) :: B(*)
      real(c_double), intent(inout) :: X(*)
      integer(c_int), intent(inout) :: Iarray(100)
      real(c_double), intent(inout) :: Rarray(100)
      integer(c_int), intent(out) :: iter, ierr
      real(c_double), intent(out) :: resid, times(3)
    end subroutine hecmw33_gpu_solve_resident
  end interface

contains

  subroutine hecmw_solve_gpu33(hecMESH, hecMAT)
    type(hecmwST_local_mesh) :: hecMESH
    type(hecmwST_matrix), target :: hecMAT
    integer(c_int) :: ierr, iter
    real(c_double) :: resid, times(3)

    if (hecMAT%NDOF /= 3) then
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
    if (hecMAT%N == hecMAT%NP .and. hecMESH%mpc%n_mpc > 0) then
      ! the mesh's MPCs: MPC-CG when MPC_METHOD = 2 (hecmw_solver_Iterative.f90:79-84)
      call hecmw33_gpu_set_matrix(gpu_handle, hecMAT%N, hecMAT%NP, hecMAT%indexL(hecMAT%NP), &
        hecMAT%indexU(hecMAT%NP), hecMAT%indexL, hecMAT%itemL, hecMAT%indexU, hecMAT%itemU, &
        hecMAT%D, hecMAT%AL, hecMAT%AU, hecMAT%Iarray, ierr)
      if (ierr == 0) call hecmw33_gpu_set_mpc(gpu_handle, hecMESH%mpc%n_mpc, hecMESH%mpc%mpc_index, &
        hecMESH%mpc%mpc_item, hecMESH%mpc%mpc_dof, hecMESH%mpc%mpc_val, hecMESH%mpc%mpc_const, ierr)
      if (ierr == 0) call hecmw33_gpu_solve_resident(gpu_handle, hecMAT%B, hecMAT%X, hecMAT%Iarray, &
        hecMAT%Rarray, iter, resid, times, ierr)
    else if (hecMAT%N == hecMAT%NP) then
      call hecmw33_gpu_solve(gpu_handle, hecMAT%N, hecMAT%NP, hecMAT%indexL(hecMAT%NP), &
        hecMAT%indexU(hecMAT%NP), hecMAT%indexL, hecMAT%itemL, hecMAT%indexU, hecMAT%itemU, &
        hecMAT%D, hecMAT%AL, hecMAT%AU, hecMAT%B, hecMAT%X, hecMAT%Iarray, hecMAT%Rarray, &
        iter, resid, times, ierr)
    else
      ! one domain of a distributed run
      cb_mesh => hecMESH
      cb_np = hecMAT%NP
      call hecmw33_gpu_set_matrix(gpu_handle, hecMAT%N, hecMAT%NP, hecMAT%indexL(hecMAT%NP), &
        hecMAT%indexU(hecMAT%NP), hecMAT%indexL, hecMAT%itemL, hecMAT%indexU, hecMAT%itemU, &
        hecMAT%D, hecMAT%AL, hecMAT%AU, hecMAT%Iarray, ierr)
      if (ierr == 0) call hecmw33_gpu_set_domain(gpu_handle, hecMESH%n_neighbor_pe, hecMESH%neighbor_pe, &
        hecMESH%import_index, hecMESH%import_item, hecMESH%export_index, hecMESH%export_item, &
        c_funloc(gpu33_exchange), c_funloc(gpu33_allreduce), c_null_ptr, ierr)
      if (ierr == 0) call hecmw33_gpu_solve_resident(gpu_handle, hecMAT%B, hecMAT%X, hecMAT%Iarray, &
        hecMAT%Rarray, iter, resid, times, ierr)
      nullify(cb_mesh)
    endif
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

  ! hecmw33_exchange_fn: hecmw_update_R of the mesh on a scratch vector that holds
  ! the send values at the export items; the received values are read back at the
  ! import items (hecmw_solver_SR.F90:97-161 does the transfer).
  subroutine gpu33_exchange(ctx, send, recv) bind(C)
    type(c_ptr), value :: ctx
    real(c_double), intent(in) :: send(*)
    real(c_double), intent(out) :: recv(*)
    real(kind=kreal), allocatable :: w(:)
    integer(kind=kint) :: k, j, n
    allocate(w(3 * cb_np))
    w = 0.d0
    n = cb_mesh%n_neighbor_pe
    do k = 1, cb_mesh%export_index(n)
      j = cb_mesh%export_item(k)
      w(3*j-2:3*j) = send(3*k-2:3*k)
    enddo
    call hecmw_update_R(cb_mesh, w, cb_np, 3)
    do k = 1, cb_mesh%import_index(n)
      j = cb_mesh%import_item(k)
      recv(3*k-2:3*k) = w(3*j-2:3*j)
    enddo
    deallocate(w)
  end subroutine gpu33_exchange

  ! hecmw33_allreduce_fn: hecmw_allreduce_R1 with hecmw_sum
  function gpu33_allreduce(ctx, v) bind(C) result(s)
    type(c_ptr), value :: ctx
    real(c_double), value :: v
    real(c_double) :: s
    real(kind=kreal) :: t
    t = v
    call hecmw_allreduce_R1(cb_mesh, t, hecmw_sum)
    s = t
  end function gpu33_allreduce

  subroutine hecmw_solve_gpu33_finalize()
    integer(c_int) :: ierr
    if (gpu_handle /= 0) call hecmw33_gpu_destroy(gpu_handle, ierr)
    gpu_handle = 0
  end subroutine hecmw_solve_gpu33_finalize

end module hecmw_solver_gpu33
