! mldg_cbind.f90 -- Fortran 2003 ISO_C_BINDING interface to libmldgpu.so.
!
! One module, standard Fortran 2003 with ISO_C_BINDING only (no PSBLAS or
! MLD2P4 modules needed): the constants, the bind(c) structures and the
! interfaces of every entry point of include/mldg.h, the C ABI of the B200
! multilevel preconditioner application.  The reference's own host code
! (mld_dprec_type, psb_krylov) reaches the GPU V-cycle through it; see
! mld_d_gpu_prec_mod.f90 for the extension of mld_dprec_type that overrides
! prec%apply (mlprec/mld_d_prec_type.f90:575-604).
!
! Conventions (as in mldg.h): int32 indices, real(c_double) values, CSR with
! ascending columns per row, index_base 1 for PSBLAS's 1-based CSR storage;
! levels numbered from 0 (finest).  Every function returns MLDG_SUCCESS (0)
! or an error code whose message mldg_last_error returns (a C string).
module mldg_cbind
  use iso_c_binding
  implicit none

  ! error codes (values follow the reference's info codes)
  integer(c_int), parameter :: MLDG_SUCCESS = 0
  integer(c_int), parameter :: MLDG_ERR_ARG = 30
  integer(c_int), parameter :: MLDG_ERR_SIZE = 36
  integer(c_int), parameter :: MLDG_ERR_NOT_BUILT = 3112
  integer(c_int), parameter :: MLDG_ERR_NO_SOLVER = 1121
  integer(c_int), parameter :: MLDG_ERR_NO_DIAG = 1124
  integer(c_int), parameter :: MLDG_ERR_TRANS = 40
  integer(c_int), parameter :: MLDG_ERR_CUDA = 4000
  integer(c_int), parameter :: MLDG_ERR_ALLOC = 4010
  integer(c_int), parameter :: MLDG_ERR_TIMEOUT = 4020
  integer(c_int), parameter :: MLDG_ERR_NOT_CONVERGED = 4030
  integer(c_int), parameter :: MLDG_ERR_INTERNAL = 4999
  ! smoother / solver kinds
  integer(c_int), parameter :: MLDG_SMOOTHER_JACOBI = 1
  integer(c_int), parameter :: MLDG_SMOOTHER_BJAC = 2
  integer(c_int), parameter :: MLDG_SMOOTHER_FBGS = 3
  ! precision forms
  integer(c_int), parameter :: MLDG_PREC_FP64 = 0
  integer(c_int), parameter :: MLDG_PREC_FP32 = 1
  integer(c_int), parameter :: MLDG_PREC_FP32_P16 = 2
  integer(c_int), parameter :: MLDG_PREC_FP32_H16 = 3
  ! memory kinds of vector arguments
  integer(c_int), parameter :: MLDG_MEM_HOST = 0
  integer(c_int), parameter :: MLDG_MEM_DEVICE = 1
  ! multilevel cycles
  integer(c_int), parameter :: MLDG_CYCLE_V = 0
  integer(c_int), parameter :: MLDG_CYCLE_W = 1
  integer(c_int), parameter :: MLDG_CYCLE_K = 2
  integer(c_int), parameter :: MLDG_CYCLE_KSYM = 3
  integer(c_int), parameter :: MLDG_CYCLE_ADD = 4
  ! Krylov methods
  integer(c_int), parameter :: MLDG_METHOD_CG = 0
  integer(c_int), parameter :: MLDG_METHOD_FCG = 1
  ! kernel classes of the timing diagnostics
  integer(c_int), parameter :: MLDG_KERNEL_TRSV = 1
  integer(c_int), parameter :: MLDG_KERNEL_SPMV = 2
  integer(c_int), parameter :: MLDG_KERNEL_JACOBI = 3
  integer(c_int), parameter :: MLDG_KERNEL_VEC = 4
  integer(c_int), parameter :: MLDG_NOALLOC_MAX_N = 524288

  type, bind(c) :: mldg_csr
    integer(c_int32_t) :: nrows = 0, ncols = 0
    type(c_ptr)        :: irp = c_null_ptr   ! int32(nrows + 1)
    type(c_ptr)        :: ja = c_null_ptr    ! int32(nnz)
    type(c_ptr)        :: val = c_null_ptr   ! real(c_double)(nnz)
  end type mldg_csr

  type, bind(c) :: mldg_opts
    integer(c_int) :: device = 0, index_base = 1, use_graphs = 1, autotune = 1
  end type mldg_opts

  type, bind(c) :: mldg_level_desc
    type(mldg_csr) :: a, p, r, nd, l, u
    type(c_ptr)    :: d = c_null_ptr
    integer(c_int) :: smoother_kind = 0, sweeps_pre = 1, sweeps_post = 1
    real(c_double) :: damping = 1.0_c_double
  end type mldg_level_desc

  type, bind(c) :: mldg_kernel_stat
    integer(c_int)     :: kind, level
    integer(c_int64_t) :: bytes
    real(c_double)     :: ms
  end type mldg_kernel_stat

  interface
    integer(c_int) function mldg_create(h, opts) bind(c, name='mldg_create')
      import :: c_ptr, c_int, mldg_opts
      type(c_ptr), intent(out) :: h
      type(mldg_opts), intent(in) :: opts
    end function mldg_create

    integer(c_int) function mldg_upload_level(h, lev, desc) bind(c, name='mldg_upload_level')
      import :: c_ptr, c_int, mldg_level_desc
      type(c_ptr), value :: h
      integer(c_int), value :: lev
      type(mldg_level_desc), intent(in) :: desc
    end function mldg_upload_level

    integer(c_int) function mldg_finalize(h, nlev, precision) bind(c, name='mldg_finalize')
      import :: c_ptr, c_int
      type(c_ptr), value :: h
      integer(c_int), value :: nlev, precision
    end function mldg_finalize

    integer(c_int) function mldg_set_cycle(h, cycle) bind(c, name='mldg_set_cycle')
      import :: c_ptr, c_int
      type(c_ptr), value :: h
      integer(c_int), value :: cycle
    end function mldg_set_cycle

    ! x, y: host arrays (MLDG_MEM_HOST) or device addresses passed by value
    ! through c_loc / a device pointer (MLDG_MEM_DEVICE)
    integer(c_int) function mldg_apply(h, x, y, trans, nrhs, ld, mem_kind) bind(c, name='mldg_apply')
      import :: c_ptr, c_int, c_char
      type(c_ptr), value :: h, x, y
      character(kind=c_char), value :: trans
      integer(c_int), value :: nrhs, ld, mem_kind
    end function mldg_apply

    ! a = c_null_ptr: the finest uploaded level matrix
    integer(c_int) function mldg_krylov(h, method, a, b, x, tol, itmax, iters, relres, mem_kind) &
         bind(c, name='mldg_krylov')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h, a, b, x
      integer(c_int), value :: method, itmax, mem_kind
      real(c_double), value :: tol
      integer(c_int), intent(out) :: iters
      real(c_double), intent(out) :: relres
    end function mldg_krylov

    integer(c_int) function mldg_krylov_multi(h, method, a, nrhs, b, ldb, x, ldx, tol, itmax, iters, relres, &
         mem_kind) bind(c, name='mldg_krylov_multi')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h, a, b, x
      integer(c_int), value :: method, nrhs, ldb, ldx, itmax, mem_kind
      real(c_double), value :: tol
      integer(c_int), intent(out) :: iters(*)
      real(c_double), intent(out) :: relres(*)
    end function mldg_krylov_multi

    ! h, b, x: arrays of nsys C pointers
    integer(c_int) function mldg_krylov_batch(nsys, h, method, b, x, tol, itmax, iters, relres, mem_kind, ms) &
         bind(c, name='mldg_krylov_batch')
      import :: c_ptr, c_int, c_double
      integer(c_int), value :: nsys, method, itmax, mem_kind
      type(c_ptr), intent(in) :: h(*), b(*), x(*)
      real(c_double), value :: tol
      integer(c_int), intent(out) :: iters(*)
      real(c_double), intent(out) :: relres(*)
      real(c_double), intent(out) :: ms
    end function mldg_krylov_batch

    integer(c_int) function mldg_adjoint(h, g, lambda, tol, itmax, iters, relres, mem_kind) &
         bind(c, name='mldg_adjoint')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h, g, lambda
      real(c_double), value :: tol
      integer(c_int), value :: itmax, mem_kind
      integer(c_int), intent(out) :: iters
      real(c_double), intent(out) :: relres
    end function mldg_adjoint

    integer(c_int) function mldg_kappa_grad(h, idim, kappa, x, lambda, grad, mem_kind) &
         bind(c, name='mldg_kappa_grad')
      import :: c_ptr, c_int
      type(c_ptr), value :: h, kappa, x, lambda, grad
      integer(c_int), value :: idim, mem_kind
    end function mldg_kappa_grad

    integer(c_int) function mldg_level_info(h, lev, info) bind(c, name='mldg_level_info')
      import :: c_ptr, c_int, c_int64_t
      type(c_ptr), value :: h
      integer(c_int), value :: lev
      integer(c_int64_t), intent(out) :: info(5)
    end function mldg_level_info

    integer(c_int) function mldg_last_timing(h, ms, launches) bind(c, name='mldg_last_timing')
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: h
      real(c_double), intent(out) :: ms
      integer(c_int64_t), intent(out) :: launches
    end function mldg_last_timing

    integer(c_int) function mldg_apply_bytes(h, bytes) bind(c, name='mldg_apply_bytes')
      import :: c_ptr, c_int, c_int64_t
      type(c_ptr), value :: h
      integer(c_int64_t), intent(out) :: bytes
    end function mldg_apply_bytes

    integer(c_int) function mldg_apply_impl_bytes(h, bytes) bind(c, name='mldg_apply_impl_bytes')
      import :: c_ptr, c_int, c_int64_t
      type(c_ptr), value :: h
      integer(c_int64_t), intent(out) :: bytes
    end function mldg_apply_impl_bytes

    integer(c_int) function mldg_probe_set(h, kind, lev, index) bind(c, name='mldg_probe_set')
      import :: c_ptr, c_int
      type(c_ptr), value :: h
      integer(c_int), value :: kind, lev, index
    end function mldg_probe_set

    integer(c_int) function mldg_probe_read(h, total_ms, count, bytes) bind(c, name='mldg_probe_read')
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: h
      real(c_double), intent(out) :: total_ms
      integer(c_int64_t), intent(out) :: count, bytes
    end function mldg_probe_read

    integer(c_int) function mldg_profile(h, trans, max, stats, n) bind(c, name='mldg_profile')
      import :: c_ptr, c_int, c_char, mldg_kernel_stat
      type(c_ptr), value :: h
      character(kind=c_char), value :: trans
      integer(c_int), value :: max
      type(mldg_kernel_stat), intent(out) :: stats(*)
      integer(c_int), intent(out) :: n
    end function mldg_profile

    integer(c_int) function mldg_profile_multi(h, trans, nrhs, max, stats, n) bind(c, name='mldg_profile_multi')
      import :: c_ptr, c_int, c_char, mldg_kernel_stat
      type(c_ptr), value :: h
      character(kind=c_char), value :: trans
      integer(c_int), value :: nrhs, max
      type(mldg_kernel_stat), intent(out) :: stats(*)
      integer(c_int), intent(out) :: n
    end function mldg_profile_multi

    ! a, x, b: device data (see mldg.h)
    integer(c_int) function mldg_relres_noalloc(h, a, x, b, relres) bind(c, name='mldg_relres_noalloc')
      import :: c_ptr, c_int, c_double, mldg_csr
      type(c_ptr), value :: h, x, b
      type(mldg_csr), intent(in) :: a
      real(c_double), intent(out) :: relres
    end function mldg_relres_noalloc

    type(c_ptr) function mldg_last_error(h) bind(c, name='mldg_last_error')
      import :: c_ptr
      type(c_ptr), value :: h
    end function mldg_last_error

    subroutine mldg_destroy(h) bind(c, name='mldg_destroy')
      import :: c_ptr
      type(c_ptr), value :: h
    end subroutine mldg_destroy
  end interface

contains

  ! the message of the last error on h as a Fortran string
  function mldg_error_string(h) result(msg)
    type(c_ptr), intent(in) :: h
    character(len=:), allocatable :: msg
    character(kind=c_char), pointer :: s(:)
    type(c_ptr) :: p
    integer :: k
    interface
      integer(c_size_t) function c_strlen(str) bind(c, name='strlen')
        import :: c_ptr, c_size_t
        type(c_ptr), value :: str
      end function c_strlen
    end interface
    p = mldg_last_error(h)
    if (.not. c_associated(p)) then
      msg = ''
      return
    end if
    call c_f_pointer(p, s, [int(c_strlen(p))])
    allocate(character(len=size(s)) :: msg)
    do k = 1, size(s)
      msg(k:k) = s(k)
    end do
  end function mldg_error_string

end module mldg_cbind
