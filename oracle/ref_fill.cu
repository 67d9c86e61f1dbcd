// ref_fill.cu -- host entry point over the reference's own fill templates:
// PHS<Q>, PolyBasis<P>, fill_matrix<N,P,Q> and fill_rhs<N,P,NRHS,Q>
// (src/rbf_operators.h:39-185).
//
// TEST INFRASTRUCTURE. Compiled by oracle/Makefile from the reference header
// where it lies (nothing of it is copied here), against the declarations-only
// oracle/stub/cusolverdx.hpp, into oracle/_ref/libref_fill.so. Only tests/
// load it: it pins the oracle's saddle-point matrix and interpolation
// right-hand sides to the reference's own arithmetic, bit for bit.
#include "rbf_operators.h"

namespace {

template <int N, int P, int Q>
int fill(const double* xs, const double* ys, int nc, const double* xc, const double* yc, double* M,
         double* B) {
    constexpr int nt = N + rbf_operators::npoly(P);
    // one "thread" covering every row: the whole system on the host
    rbf_operators::fill_matrix<N, P, Q>(M, xs, ys, 0, 1);
    for (int j = 0; j < nc; ++j)
        rbf_operators::fill_rhs<N, P, 1, Q>(B + j * nt, xs, ys, xc + j, yc + j, 0, 1);
    return nt;
}

}  // namespace

extern "C" {

// M (nt x nt, column-major, ldm = nt) and B (nt x nc, column-major, ldb = nt)
// of one stencil of k nodes at local coordinates xs, ys, for the compiled
// (k, P, Q) combinations; returns nt, or -1 for a combination not compiled.
int ref_fill(int k, int P, int Q, const double* xs, const double* ys, int nc, const double* xc,
             const double* yc, double* M, double* B) {
#define RBFB_REF_CASE(N_, P_, Q_) \
    if (k == N_ && P == P_ && Q == Q_) return fill<N_, P_, Q_>(xs, ys, nc, xc, yc, M, B);
    RBFB_REF_CASE(21, 2, 3)
    RBFB_REF_CASE(28, 3, 5)
    RBFB_REF_CASE(35, 3, 5)
    RBFB_REF_CASE(48, 4, 7)
    RBFB_REF_CASE(64, 4, 7)
#undef RBFB_REF_CASE
    return -1;
}

}  // extern "C"
