! mld_d_gpu_prec_mod.f90 -- MLD2P4's preconditioner with its apply on the B200.
!
! An extension of mld_dprec_type (mlprec/mld_d_prec_type.f90:84-116) that
! keeps the reference's whole host set-up -- init / set / hierarchy_build /
! smoothers_build, so the aggregates, prolongators, Galerkin products and
! ILU(0) factors are the reference's own -- and then:
!   * gpu_build uploads every level once through the C ABI (mldg_cbind):
!     the level matrix, the maps P = map_Y2X and R = map_X2Y stored at the
!     coarser level, and the smoother data (ILU(0) factors L, U and the
!     inverse pivots d; the Jacobi off-diagonal part ND and the inverse
!     diagonal; the GS strict triangles and the diagonal), then finalizes;
!   * psb_d_apply2_vect, the method psb_krylov calls on every iteration
!     (mld_d_prec_type.f90:112, 575-604), runs the V-cycle on the GPU with
!     the same arguments, trans values and info codes.
! A solver or storage the GPU path does not take (a non-CSR level matrix, an
! AS smoother, a direct coarse solver) leaves gpu_build with an error code
! and the caller keeps the reference's own apply.
!
! Needs PSBLAS >= 3.5 (psb_base_mod) and MLD2P4 2.1 (mld_prec_mod) at compile
! time, and libmldgpu.so at link time.
module mld_d_gpu_prec_mod
  use iso_c_binding
  use psb_base_mod
  use mld_prec_mod
  use mld_d_jac_smoother, only: mld_d_jac_smoother_type
  use mld_d_ilu_solver, only: mld_d_ilu_solver_type
  use mld_d_diag_solver, only: mld_d_diag_solver_type
  use mld_d_gs_solver, only: mld_d_gs_solver_type, mld_d_bwgs_solver_type
  use mldg_cbind
  implicit none

  type, extends(mld_dprec_type) :: mld_d_gpu_prec_type
    type(c_ptr)    :: h = c_null_ptr
    integer(c_int) :: precision = MLDG_PREC_FP64
    ! strict lower triangle and diagonal of GS levels, kept until finalize
    integer(psb_ipk_), allocatable :: gs_irp(:,:), gs_ja(:,:)
    real(psb_dpk_), allocatable    :: gs_val(:,:), gs_d(:,:)
  contains
    procedure, pass(prec) :: gpu_build => mld_d_gpu_build
    procedure, pass(prec) :: gpu_free  => mld_d_gpu_free
    procedure, pass(prec) :: psb_d_apply2_vect => mld_d_gpu_apply2_vect
    procedure, pass(prec) :: apply_device => mld_d_gpu_apply_device
  end type mld_d_gpu_prec_type

contains

  ! a view of a host CSR matrix (PSBLAS psb_d_csr_sparse_mat, 1-based)
  subroutine csr_view(m, c, info)
    type(psb_dspmat_type), intent(in), target :: m
    type(mldg_csr), intent(out) :: c
    integer(psb_ipk_), intent(out) :: info
    info = 0
    select type (aa => m%a)
    type is (psb_d_csr_sparse_mat)
      c%nrows = int(aa%get_nrows(), c_int32_t)
      c%ncols = int(aa%get_ncols(), c_int32_t)
      c%irp = c_loc(aa%irp)
      c%ja = c_loc(aa%ja)
      c%val = c_loc(aa%val)
    class default
      info = MLDG_ERR_ARG   ! convert with m%cscnv(info, type='CSR') first
    end select
  end subroutine csr_view

  subroutine mld_d_gpu_build(prec, info, precision, device)
    class(mld_d_gpu_prec_type), intent(inout), target :: prec
    integer(psb_ipk_), intent(out) :: info
    integer(c_int), intent(in), optional :: precision, device
    type(mldg_opts) :: opts
    type(mldg_level_desc) :: desc
    integer(psb_ipk_) :: il, nlev
    integer(c_int) :: rc

    info = 0
    if (.not. allocated(prec%precv)) then
      info = MLDG_ERR_NOT_BUILT
      return
    end if
    nlev = size(prec%precv)
    call prec%gpu_free()
    opts = mldg_opts()
    opts%index_base = 1
    if (present(device)) opts%device = device
    if (present(precision)) prec%precision = precision
    rc = mldg_create(prec%h, opts)
    if (rc /= 0) then
      info = rc
      return
    end if
    do il = 1, nlev
      desc = mldg_level_desc()
      if (.not. associated(prec%precv(il)%base_a)) then
        info = MLDG_ERR_NOT_BUILT
        return
      end if
      call csr_view(prec%precv(il)%base_a, desc%a, info)
      if (info /= 0) return
      if (il > 1) then
        call csr_view(prec%precv(il)%map%map_Y2X, desc%p, info)   ! n_{il-1} x n_il
        if (info /= 0) return
        call csr_view(prec%precv(il)%map%map_X2Y, desc%r, info)   ! n_il x n_{il-1}
        if (info /= 0) return
      end if
      desc%sweeps_pre = prec%precv(il)%parms%sweeps_pre
      desc%sweeps_post = prec%precv(il)%parms%sweeps_post
      desc%damping = 1.0_c_double
      call level_smoother(prec, il, desc, info)
      if (info /= 0) return
      rc = mldg_upload_level(prec%h, int(il - 1, c_int), desc)
      if (rc /= 0) then
        info = rc
        return
      end if
    end do
    rc = mldg_finalize(prec%h, int(nlev, c_int), prec%precision)
    if (rc /= 0) info = rc
    if (allocated(prec%gs_irp)) deallocate(prec%gs_irp, prec%gs_ja, prec%gs_val, prec%gs_d)
  end subroutine mld_d_gpu_build

  ! smoother data of level il (mld_d_jac_smoother_type with an ILU, diag or
  ! GS solver; mld_d_jac_smoother.f90:56-62, mld_d_ilu_solver.f90:63-68,
  ! mld_d_diag_solver.f90:53-55, mld_d_gs_solver.f90:57-60)
  subroutine level_smoother(prec, il, desc, info)
    class(mld_d_gpu_prec_type), intent(inout), target :: prec
    integer(psb_ipk_), intent(in) :: il
    type(mldg_level_desc), intent(inout) :: desc
    integer(psb_ipk_), intent(out) :: info
    info = 0
    if (.not. allocated(prec%precv(il)%sm)) then
      info = MLDG_ERR_NO_SOLVER
      return
    end if
    select type (sm => prec%precv(il)%sm)
    type is (mld_d_jac_smoother_type)
      if (.not. allocated(sm%sv)) then
        info = MLDG_ERR_NO_SOLVER
        return
      end if
      select type (sv => sm%sv)
      type is (mld_d_ilu_solver_type)
        ! one rank: the off-block part is empty and a sweep is one ILU solve
        call csr_view(sv%l, desc%l, info)
        if (info == 0) call csr_view(sv%u, desc%u, info)
        if (.not. allocated(sv%d)) info = MLDG_ERR_NO_DIAG
        if (info == 0) desc%d = c_loc(sv%d)
        desc%smoother_kind = MLDG_SMOOTHER_BJAC
      type is (mld_d_diag_solver_type)
        if (sm%nd%get_nzeros() > 0) call csr_view(sm%nd, desc%nd, info)
        if (.not. allocated(sv%d)) info = MLDG_ERR_NO_DIAG
        if (info == 0) desc%d = c_loc(sv%d)
        desc%smoother_kind = MLDG_SMOOTHER_JACOBI
      type is (mld_d_gs_solver_type)
        ! sv%l holds tril(A) with the diagonal (mld_d_gs_solver_bld.f90:79):
        ! split it into the strict triangle and the diagonal the C ABI takes
        call split_gs(prec, il, sv%l, desc, info)
        if (info == 0) call csr_view(sv%u, desc%u, info)
        desc%smoother_kind = MLDG_SMOOTHER_FBGS
      class default
        info = MLDG_ERR_NO_SOLVER
      end select
    class default
      info = MLDG_ERR_NO_SOLVER
    end select
  end subroutine level_smoother

  subroutine split_gs(prec, il, lw, desc, info)
    class(mld_d_gpu_prec_type), intent(inout), target :: prec
    integer(psb_ipk_), intent(in) :: il
    type(psb_dspmat_type), intent(in), target :: lw
    type(mldg_level_desc), intent(inout) :: desc
    integer(psb_ipk_), intent(out) :: info
    integer(psb_ipk_) :: n, nz, i, k, q, nlev
    info = 0
    nlev = size(prec%precv)
    select type (aa => lw%a)
    type is (psb_d_csr_sparse_mat)
      n = aa%get_nrows()
      nz = aa%irp(n + 1) - 1
      if (.not. allocated(prec%gs_irp)) then
        allocate(prec%gs_irp(n + 1, nlev), prec%gs_ja(nz, nlev), prec%gs_val(nz, nlev), prec%gs_d(n, nlev))
      end if
      if (size(prec%gs_irp, 1) < n + 1 .or. size(prec%gs_ja, 1) < nz) then
        deallocate(prec%gs_irp, prec%gs_ja, prec%gs_val, prec%gs_d)
        allocate(prec%gs_irp(n + 1, nlev), prec%gs_ja(nz, nlev), prec%gs_val(nz, nlev), prec%gs_d(n, nlev))
      end if
      q = 1
      prec%gs_irp(1, il) = 1
      do i = 1, n
        prec%gs_d(i, il) = 0.0_psb_dpk_
        do k = aa%irp(i), aa%irp(i + 1) - 1
          if (aa%ja(k) < i) then
            prec%gs_ja(q, il) = aa%ja(k)
            prec%gs_val(q, il) = aa%val(k)
            q = q + 1
          else if (aa%ja(k) == i) then
            prec%gs_d(i, il) = aa%val(k)
          end if
        end do
        prec%gs_irp(i + 1, il) = q
      end do
      desc%l%nrows = int(n, c_int32_t)
      desc%l%ncols = int(n, c_int32_t)
      desc%l%irp = c_loc(prec%gs_irp(1, il))
      desc%l%ja = c_loc(prec%gs_ja(1, il))
      desc%l%val = c_loc(prec%gs_val(1, il))
      desc%d = c_loc(prec%gs_d(1, il))
    class default
      info = MLDG_ERR_ARG
    end select
  end subroutine split_gs

  ! prec%apply as psb_krylov calls it: y = M^{-1} x or M^{-T} x on the GPU
  ! (replaces mld_d_apply2_vect -> mld_dprecaply2_vect, mld_dprecaply.f90:305-443)
  subroutine mld_d_gpu_apply2_vect(prec, x, y, desc_data, info, trans, work)
    type(psb_desc_type), intent(in) :: desc_data
    class(mld_d_gpu_prec_type), intent(inout) :: prec
    type(psb_d_vect_type), intent(inout), target :: x, y
    integer(psb_ipk_), intent(out) :: info
    character(len=1), optional :: trans
    real(psb_dpk_), intent(inout), optional, target :: work(:)
    character(kind=c_char) :: trans_
    character(len=20) :: name = 'mld_d_gpu_apply'
    integer(c_int) :: rc, n

    info = psb_success_
    if (.not. c_associated(prec%h)) then
      info = MLDG_ERR_NOT_BUILT                ! 3112: apply before build
      call psb_errpush(info, name)
      return
    end if
    trans_ = 'N'
    if (present(trans)) trans_ = psb_toupper(trans)
    n = int(desc_data%get_local_rows(), c_int)
    if (x%get_nrows() < n .or. y%get_nrows() < n) then
      info = MLDG_ERR_SIZE                     ! 36: vector too short
      call psb_errpush(info, name)
      return
    end if
    rc = mldg_apply(prec%h, c_loc(x%v%v), c_loc(y%v%v), trans_, 1_c_int, n, MLDG_MEM_HOST)
    if (rc /= 0) then
      info = rc
      call psb_errpush(info, name, a_err=mldg_error_string(prec%h))
    end if
  end subroutine mld_d_gpu_apply2_vect

  ! The same apply on vectors that already live on the GPU (the device
  ! addresses of a CUDA-resident PSBLAS vector, e.g. one built with a device
  ! vmold, mld_dprecbld.f90:72-74): nothing is copied between host and device.
  ! xdev, ydev: device addresses of n doubles.
  subroutine mld_d_gpu_apply_device(prec, xdev, ydev, n, info, trans)
    class(mld_d_gpu_prec_type), intent(inout) :: prec
    type(c_ptr), intent(in) :: xdev, ydev
    integer(psb_ipk_), intent(in) :: n
    integer(psb_ipk_), intent(out) :: info
    character(len=1), optional :: trans
    character(kind=c_char) :: trans_
    character(len=20) :: name = 'mld_d_gpu_apply_dev'
    integer(c_int) :: rc
    info = psb_success_
    if (.not. c_associated(prec%h)) then
      info = MLDG_ERR_NOT_BUILT
      call psb_errpush(info, name)
      return
    end if
    trans_ = 'N'
    if (present(trans)) trans_ = psb_toupper(trans)
    rc = mldg_apply(prec%h, xdev, ydev, trans_, 1_c_int, int(n, c_int), MLDG_MEM_DEVICE)
    if (rc /= 0) then
      info = rc
      call psb_errpush(info, name, a_err=mldg_error_string(prec%h))
    end if
  end subroutine mld_d_gpu_apply_device

  subroutine mld_d_gpu_free(prec)
    class(mld_d_gpu_prec_type), intent(inout) :: prec
    if (c_associated(prec%h)) call mldg_destroy(prec%h)
    prec%h = c_null_ptr
  end subroutine mld_d_gpu_free

end module mld_d_gpu_prec_mod
