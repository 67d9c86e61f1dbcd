! rbf_cuda.f90 -- drop-in for the reference's CUDA Fortran module rbf_cuda
! (src/rbf_cuda.f90), over the C ABI of include/rbf_b200.h.
!
! Same module name, same public names and the same argument lists as the
! reference: dp, NMAX, fill_kernel(nstencils,x,y,ia,ja,M,ldm),
! fill_rhs(n,x,y,nc,xc,yc,B,ldb), store_to_csr(nstencils,ia,va,W,ldw,idx) and
! print_matrix. Arrays are CUDA Fortran device arrays, as there; indices in
! ia/ja are 0-based, as there. The work runs in the sm_100a library:
!
!   fill_kernel   -> rbfb_fill_kernel: degree-2, r^3 saddle-point matrix from
!                    the absolute coordinates (the reference's arithmetic);
!                    stencil s goes to the ldm x ldm slab at M(1, s*ldm + 1),
!                    so nstencils = 1 fills M itself, as the reference does
!   fill_rhs      -> rbfb_fill_rhs: interpolation right-hand sides
!   store_to_csr  -> rbfb_store_to_csr_stencil: va(ia(idx)+k-1) = W(k,1) + W(k,2)
!
! What changes for a caller: the reference's fill_kernel and fill_rhs are
! kernels launched with chevrons (call fill_kernel<<<grid, block>>>(...)) and
! store_to_csr is a device subroutine called from a kernel; here all three
! are host subroutines with the same arguments (call fill_kernel(...)), which
! launch the library's kernels on the default stream and stop with an error
! message on a nonzero status. Weights for whole node sets come from
! rbfb_assemble / rbfb_assemble_csr (module rbf_b200).
!
! Build (CUDA Fortran): nvfortran -cuda -c rbf_cuda.f90, link with
! -L<repo>/gpu-assembly_b200/lib -lrbf_b200. Not compiled in this
! repository's build: the image carries no Fortran compiler.
module rbf_cuda
    use, intrinsic :: iso_c_binding
    use cudafor
    implicit none
    private

    public :: dp, NMAX, fill_kernel, fill_rhs, store_to_csr, print_matrix

    integer, parameter :: dp = kind(1.0d0)  ! the double-precision kind
    integer, parameter :: NMAX = 64         ! largest stencil the reference stages

    interface
        integer(c_int) function c_fill_kernel(nstencils, x, y, ia, ja, m, ldm, stream) &
            bind(c, name="rbfb_fill_kernel")
            import :: c_int, c_double, c_ptr
            integer(c_int), value :: nstencils, ldm
            real(c_double), device, intent(in) :: x(*), y(*)
            integer(c_int), device, intent(in) :: ia(*), ja(*)
            real(c_double), device :: m(*)
            type(c_ptr), value :: stream
        end function

        integer(c_int) function c_fill_rhs(n, x, y, nc, xc, yc, b, ldb, stream) &
            bind(c, name="rbfb_fill_rhs")
            import :: c_int, c_double, c_ptr
            integer(c_int), value :: n, nc, ldb
            real(c_double), device, intent(in) :: x(*), y(*), xc(*), yc(*)
            real(c_double), device :: b(*)
            type(c_ptr), value :: stream
        end function

        integer(c_int) function c_store_to_csr_stencil(nstencils, ia, va, w, ldw, idx, stream) &
            bind(c, name="rbfb_store_to_csr_stencil")
            import :: c_int, c_double, c_ptr
            integer(c_int), value :: nstencils, ldw, idx
            integer(c_int), device, intent(in) :: ia(*)
            real(c_double), device :: va(*)
            real(c_double), device, intent(in) :: w(*)
            type(c_ptr), value :: stream
        end function
    end interface

contains

subroutine check(status, what)
    integer(c_int), intent(in) :: status
    character(*), intent(in) :: what
    if (status /= 0) then
        print '(a,a,a,i0)', 'rbf_cuda: ', what, ' failed with status ', status
        error stop 1
    end if
end subroutine

! [A P; P^T 0] with phi = r^3 and the six degree-2 monomials, for each stencil
! s of the graph (row s: ja(ia(s)) .. ja(ia(s+1)-1)), from node coordinates
! x, y as given.
subroutine fill_kernel(nstencils, x, y, ia, ja, M, ldm)
    integer, value :: nstencils, ldm
    real(dp), intent(in), device :: x(0:nstencils-1), y(0:nstencils-1)
    integer, intent(in), device :: ia(0:nstencils), ja(0:*)
    real(dp), intent(out), device :: M(ldm,*)
    call check(c_fill_kernel(nstencils, x, y, ia, ja, M, ldm, c_null_ptr), 'fill_kernel')
end subroutine

! Column j of B (j = 1..nc) holds phi(|p - x_k|), k = 1..n, then the six
! monomials, at the evaluation point p = (xc(j), yc(j)).
subroutine fill_rhs(n, x, y, nc, xc, yc, B, ldb)
    integer, value :: n, nc, ldb
    real(dp), intent(in), device :: x(n), y(n), xc(nc), yc(nc)
    real(dp), intent(out), device :: B(ldb,*)
    call check(c_fill_rhs(n, x, y, nc, xc, yc, B, ldb, c_null_ptr), 'fill_rhs')
end subroutine

! Stencil idx's Laplacian weights into its CSR row: the sum of the two
! columns of W (d2/dx2 and d2/dy2 weights).
subroutine store_to_csr(nstencils, ia, va, W, ldw, idx)
    integer, value :: nstencils, ldw, idx
    integer, intent(in), device :: ia(0:nstencils)
    real(dp), intent(inout), device :: va(0:*)
    real(dp), intent(in), device :: W(ldw,2)
    call check(c_store_to_csr_stencil(nstencils, ia, va, W, ldw, idx, c_null_ptr), &
               'store_to_csr')
end subroutine

! The leading nrows x ncols block of M (leading dimension ld), one matrix row
! per output line in f10.4 fields, after the label when one is given.
subroutine print_matrix(nrows, ncols, M, ld, label)
    integer, intent(in) :: nrows, ncols, ld
    real(dp), intent(in) :: M(ld, ncols)
    character(*), intent(in), optional :: label
    integer :: r, c
    if (present(label)) write (*, '(a)') label
    do r = 1, nrows
        write (*, '(*(f10.4))') (M(r, c), c = 1, ncols)
    end do
    write (*, *)
end subroutine

end module rbf_cuda
