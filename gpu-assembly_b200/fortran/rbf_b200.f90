! rbf_b200.f90 -- Fortran interface to the B200 assembly library (C ABI of
! include/rbf_b200.h) through bind(c).
!
! The reference's Fortran side is the CUDA Fortran module rbf_cuda
! (src/rbf_cuda.f90) and the demo src/main.f90, which binds the C kernel
! symbol solve_dp with an interface block. This module gives a Fortran
! caller the same reach into the sm_100a library: the context, the k-NN
! stencils, the assembly of fixed-width and CSR stencils, fill_matrices
! (fill_kernel), store_to_csr and solve_dp. All array arguments are device
! addresses (type(c_ptr), e.g. c_loc of a device array, or c_devloc in CUDA
! Fortran); indices are 0-based int32 as in the reference.
!
! Not compiled in this repository's build: the image carries no Fortran
! compiler. The interfaces mirror include/rbf_b200.h line for line.
module rbf_b200
  use, intrinsic :: iso_c_binding
  implicit none
  private

  integer(c_int), parameter, public :: RBFB_OK = 0, RBFB_EINVAL = -1, RBFB_ECUDA = -2, &
      RBFB_ENOMEM = -3, RBFB_EUNSUPPORTED = -4, RBFB_ETIMEOUT = -5, RBFB_EBUDGET = -6, &
      RBFB_ENOTFOUND = -7, RBFB_EBUSY = -8, RBFB_ETOOBIG = -9
  integer(c_int), parameter, public :: RBFB_OP_INTERP = 1, RBFB_OP_LAPLACE = 2, &
      RBFB_OP_DX = 4, RBFB_OP_DY = 8, RBFB_OP_DXX = 16, RBFB_OP_DYY = 32, RBFB_OP_DXY = 64
  integer(c_int), parameter, public :: RBFB_FP64 = 0, RBFB_FP32_IR = 1

  ! rbfb_desc
  type, bind(c), public :: rbfb_desc
    integer(c_int) :: degree = 2
    integer(c_int) :: phs = 0
    integer(c_int) :: ops = 14          ! Laplacian, d/dx, d/dy
    integer(c_int) :: precision = 0
    integer(c_int) :: scale = 1
    integer(c_int) :: max_sweeps = 0
    real(c_double) :: ir_tol = 0.0_c_double
    real(c_double) :: period(2) = 0.0_c_double
    integer(c_int) :: nc = 0
    type(c_ptr) :: xc = c_null_ptr
    type(c_ptr) :: yc = c_null_ptr
  end type

  ! rbfb_stats
  type, bind(c), public :: rbfb_stats
    integer(c_long_long) :: stencils, singular, fallback, sweeps
    integer(c_int) :: max_sweeps_used, buckets
    real(c_float) :: ms
  end type

  public :: rbfb_create, rbfb_destroy, rbfb_knn_stencils, rbfb_assemble, rbfb_assemble_csr
  public :: rbfb_fill_matrices, rbfb_store_to_csr, rbfb_solve_dp, rbfb_spmv
  public :: rbfb_solve_bicgstab

  interface
    integer(c_int) function rbfb_create(ctx, device) bind(c, name="rbfb_create")
      import :: c_int, c_ptr
      type(c_ptr), intent(out) :: ctx
      integer(c_int), value :: device
    end function

    integer(c_int) function rbfb_destroy(ctx) bind(c, name="rbfb_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    ! NodeSet::stencils(k) / KdTree::knn_stencils(k): ja(k, n), period = c_null_ptr
    ! for the open plane or c_loc of a host real(c_double) :: period(2)
    integer(c_int) function rbfb_knn_stencils(ctx, n, x, y, k, period_h, ja, stream) &
        bind(c, name="rbfb_knn_stencils")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, x, y, period_h, ja, stream
      integer(c_int), value :: n, k
    end function

    ! assemble_interp_weights<Config> / the Laplacian assembly: values_h is a
    ! host array of nrhs device addresses (type(c_ptr) :: values(nrhs))
    integer(c_int) function rbfb_assemble(ctx, desc, nstencils, x, y, k, ja, values_h, info, &
        stats, stream) bind(c, name="rbfb_assemble")
      import :: c_int, c_ptr, rbfb_desc
      type(c_ptr), value :: ctx, x, y, ja, values_h, info, stats, stream
      type(rbfb_desc), intent(in) :: desc
      integer(c_int), value :: nstencils, k
    end function

    ! CSR stencils (ia/ja as the reference's fill_kernel takes them)
    integer(c_int) function rbfb_assemble_csr(ctx, desc, nstencils, x, y, ia, ja, degree, &
        values_h, info, stats, stream) bind(c, name="rbfb_assemble_csr")
      import :: c_int, c_ptr, rbfb_desc
      type(c_ptr), value :: ctx, x, y, ia, ja, degree, values_h, info, stats, stream
      type(rbfb_desc), intent(in) :: desc
      integer(c_int), value :: nstencils
    end function

    ! fill_kernel(nstencils, x, y, ia, ja, M, ldm) of src/rbf_cuda.f90, every stencil
    integer(c_int) function rbfb_fill_matrices(ctx, desc, nstencils, x, y, ia, ja, m, ldm, &
        stream) bind(c, name="rbfb_fill_matrices")
      import :: c_int, c_ptr, rbfb_desc
      type(c_ptr), value :: ctx, x, y, ia, ja, m, stream
      type(rbfb_desc), intent(in) :: desc
      integer(c_int), value :: nstencils, ldm
    end function

    ! store_to_csr of src/rbf_cuda.f90: va = wxx + wyy over the CSR rows
    integer(c_int) function rbfb_store_to_csr(nstencils, ia, wxx, wyy, va, stream) &
        bind(c, name="rbfb_store_to_csr")
      import :: c_int, c_ptr
      integer(c_int), value :: nstencils
      type(c_ptr), value :: ia, wxx, wyy, va, stream
    end function

    ! solve_dp<<<1,32>>>(A, ipiv, B, info) of src/rbf_operators.cpp:7-11
    integer(c_int) function rbfb_solve_dp(a, ipiv, b, info, stream) bind(c, name="rbfb_solve_dp")
      import :: c_int, c_ptr
      type(c_ptr), value :: a, ipiv, b, info, stream
    end function

    ! out = A u, out(bnd) = u(bnd): the operator application src/main.cpp:57-66 sketches
    integer(c_int) function rbfb_spmv(n, k, ja, values, u, out, bnd, nbnd, stream) &
        bind(c, name="rbfb_spmv")
      import :: c_int, c_ptr
      integer(c_int), value :: n, k, nbnd
      type(c_ptr), value :: ja, values, u, out, bnd, stream
    end function

    ! BiCGSTAB for A u = f with that operator: the solve src/main.cpp:68 leaves
    ! empty. ia = c_null_ptr selects fixed-width rows of k.
    integer(c_int) function rbfb_solve_bicgstab(ctx, n, k, ia, ja, values, bnd, nbnd, f, u, &
        tol, maxit, iters, relres, stream) bind(c, name="rbfb_solve_bicgstab")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, ia, ja, values, bnd, f, u, stream
      integer(c_int), value :: n, k, nbnd, maxit
      real(c_double), value :: tol
      integer(c_int), intent(out) :: iters
      real(c_double), intent(out) :: relres
    end function
  end interface
end module rbf_b200
