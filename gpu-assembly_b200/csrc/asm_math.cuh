// asm_math.cuh -- pinned FP64 arithmetic of the RBF-FD system: PHS, monomials
// and the operator right-hand sides, evaluated in the same operation order as
// the CPU oracle so that the FP64 kernel reproduces it bit for bit.
//
// Reference: PHS<Q> src/rbf_operators.h:39-76, PolyBasis<P> :78-114,
// fill_matrix :116-154, fill_rhs :156-185.
#pragma once

#include <cstdint>

namespace rbfb {

constexpr int kOpInterp = 1, kOpLaplace = 2, kOpDx = 4, kOpDy = 8, kOpDxx = 16, kOpDyy = 32,
              kOpDxy = 64;

__host__ __device__ constexpr int npoly(int P) { return P < 0 ? 0 : (P + 1) * (P + 2) / 2; }

// Order of the derivative an operator takes (the power of the radius scale
// its weights carry).
__host__ __device__ inline int op_order(int op) {
    return op == kOpInterp ? 0 : ((op == kOpDx || op == kOpDy) ? 1 : 2);
}

// ---- FP64 with every rounding explicit (no contraction by the compiler) ----
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// squared distance, dx*dx + dy*dy rounded per operation
__device__ __forceinline__ double dist2(double dx, double dy) {
    return dadd(dmul(dx, dx), dmul(dy, dy));
}

// phi(r) = r^Q from r^2 in the reference's product order.
template <int Q>
__device__ __forceinline__ double phs64(double r2) {
    static_assert(Q >= 1 && Q % 2 == 1, "odd PHS exponent");
    if constexpr (Q == 1) {
        return dsqrt(r2);
    } else if constexpr (Q == 3) {
        return dmul(r2, dsqrt(r2));
    } else if constexpr (Q == 5) {
        return dmul(dmul(r2, r2), dsqrt(r2));
    } else if constexpr (Q == 7) {
        const double r4 = dmul(r2, r2);
        return dmul(dmul(r4, r2), dsqrt(r2));
    } else {
        double p = dsqrt(r2);
#pragma unroll
        for (int i = 0; i < (Q - 1) / 2; ++i) p = dmul(p, r2);
        return p;
    }
}

// x^a * y^b with the powers built by repeated multiplication, the
// reference's PolyBasis arithmetic (X[i] = X[i-1]*x). a, b <= P.
template <int P>
__device__ __forceinline__ double mono_ab(double x, double y, int a, int b) {
    double X = 1.0, Y = 1.0;
#pragma unroll
    for (int i = 1; i <= P; ++i) {
        X = (i <= a) ? dmul(X, x) : X;
        Y = (i <= b) ? dmul(Y, y) : Y;
    }
    return dmul(X, Y);
}

// Exponents (a, b) of monomial number m: m = d(d+1)/2 + j, a = d - j, b = j.
__host__ __device__ inline void mono_exps(int m, int& a, int& b) {
    int d = 0;
    while ((d + 1) * (d + 2) / 2 <= m) ++d;
    const int j = m - d * (d + 1) / 2;
    a = d - j;
    b = j;
}

// All monomials of (x, y) in the reference's order.
template <int P>
__device__ __forceinline__ void monomials(double x, double y, double* b) {
    double X[P + 1], Y[P + 1];
    X[0] = Y[0] = 1.0;
#pragma unroll
    for (int i = 1; i <= P; ++i) {
        X[i] = dmul(X[i - 1], x);
        Y[i] = dmul(Y[i - 1], y);
    }
    int k = 0;
#pragma unroll
    for (int d = 0; d <= P; ++d)
#pragma unroll
        for (int j = 0; j <= d; ++j) b[k++] = dmul(X[d - j], Y[j]);
}

// Operator applied to monomial m at the origin.
__device__ __forceinline__ double poly_op_origin(int op, int m) {
    switch (op) {
        case kOpLaplace: return (m == 3 || m == 5) ? 2.0 : 0.0;
        case kOpDx: return m == 1 ? 1.0 : 0.0;
        case kOpDy: return m == 2 ? 1.0 : 0.0;
        case kOpDxx: return m == 3 ? 2.0 : 0.0;
        case kOpDyy: return m == 5 ? 2.0 : 0.0;
        case kOpDxy: return m == 4 ? 1.0 : 0.0;
        default: return 0.0;
    }
}

// Operator applied in the evaluation point to phi(|x_e - x_k|), at x_e = 0,
// for a node at (xk, yk) in the stencil-local frame.
template <int Q>
__device__ __forceinline__ double phs_op_origin(int op, double xk, double yk) {
    const double r2 = dist2(xk, yk);
    const double rq2 = phs64<Q - 2>(r2);
    const double q = static_cast<double>(Q);
    switch (op) {
        case kOpLaplace: return dmul(q * q, rq2);
        case kOpDx: return -dmul(dmul(q, rq2), xk);
        case kOpDy: return -dmul(dmul(q, rq2), yk);
        case kOpDxx:
        case kOpDyy:
        case kOpDxy: {
            if (r2 == 0.0) return 0.0;
            const double a = dmul(q, rq2);
            const double b = dmul(q * (q - 2.0), rq2);
            if (op == kOpDxx) return dadd(a, dmul(b, ddiv(dmul(xk, xk), r2)));
            if (op == kOpDyy) return dadd(a, dmul(b, ddiv(dmul(yk, yk), r2)));
            return dmul(b, ddiv(dmul(xk, yk), r2));
        }
        default: return 0.0;
    }
}

// PeriodicBox::minimum_image (src/rbf_spatial.h:74-76), rounded per operation.
__device__ __forceinline__ double min_image(double d, double L) {
    return L > 0.0 ? dsub(d, dmul(L, rint(ddiv(d, L)))) : d;
}

}  // namespace rbfb
