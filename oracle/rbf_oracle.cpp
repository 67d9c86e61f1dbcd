// rbf_oracle.cpp -- CPU restatement of the RBF-FD assembly path of
// ivan-pi/gpu-assembly, in FP64.
//
// TEST INFRASTRUCTURE. This file is the checker, never the product: only
// tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
// bench.py load it. The CUDA library never links or calls it.
//
// What it restates (reference paths are relative to the reference repo):
//   phs()            PHS<Q>                         src/rbf_operators.h:39-76
//   monomials()      PolyBasis<P>, npoly            src/rbf_operators.h:78-114
//   fill_system()    fill_matrix<N,P,Q>             src/rbf_operators.h:116-154
//   interp rhs       fill_rhs<N,P,NRHS,Q>           src/rbf_operators.h:156-185
//   gather/shift     assemble_interp_weights        src/rbf_operators.h:350-358
//   scatter          assemble_interp_weights        src/rbf_operators.h:368-375
//   minimum image    PeriodicBox::minimum_image     src/rbf_spatial.h:74-76
//   brute k-NN       test_spatial brute_knn + metric  test/test_spatial.cpp:59-82
//                    nanoflann L2_Simple_Adaptor    third_party/nanoflann/nanoflann.hpp:690-699
//                    ckdtree wrap_distance          third_party/ckdtree/src/distance.h:262-272
//   curve keys       zidx / hidx                    src/rbf_ordering.F90:82-218
//   curve order      morton_order / hilbert_order   src/rbf_reorder.h:180-185,210-230
//   boundary last    boundary_last_by_flag          src/rbf_reorder.h:232-244
//   renumbering      renumber_stencils / _csr       src/rbf_reorder.h:256-303
//
// What it adds, because the reference has it only as intent:
//   * derivative right-hand sides at the stencil centre (Laplacian, d/dx,
//     d/dy, d2/dx2, d2/dy2, d2/dxdy); the Fortran store_to_csr forms the
//     Laplacian from two second-derivative columns (src/rbf_cuda.f90:139-157)
//     and src/main.cpp:15-16 names a Laplacian assembly that does not exist.
//   * radius scaling by a power of two (exact in binary floating point).
//   * the solver. The reference calls cuSolverDx gesv_partial_pivot, a
//     closed library, so the solve here is the textbook Gaussian
//     elimination with partial pivoting (Golub & Van Loan, Matrix
//     Computations, alg. 3.4.1) in its row-implicit form: rows are never
//     swapped; at step c the pivot is the unused row with the largest
//     |a(r,c)| compared by the high 32 bits of its binary64 representation
//     without their 7 lowest bits (sign, exponent and the 13 leading
//     mantissa bits), ties going to the lowest row index; multipliers are
//     a(r,c) * (1 / pivot); updates are fma(-l, u, a); back substitution
//     is column oriented, x_c = y_c * (1 / pivot_c). The CUDA FP64 kernel
//     performs the same operations in the same order.
//
// Arithmetic is pinned: compiled with -ffp-contract=off, every fused
// multiply-add is an explicit std::fma, everything else rounds per operation.
//
// Pinning. The k-NN part is pinned against the reference itself: its golden
// periodic graphs (data/poisson_32_*.graph) and its own nanoflann / ckdtree
// searches compiled from its sources (ref_knn.cpp). The WEIGHTS are parity
// unpinned: no reference test or fixture holds an assembled weight, and the
// reference's solver (cuSolverDx gesv_partial_pivot, MathDx 26.06) is closed
// and absent. The restatement is checked instead by properties the exact
// weights have -- polynomial reproduction to degree P, scale covariance,
// agreement with LAPACK's LU and with an x87 long-double run of the same
// algorithm -- and its own output is frozen in tests/golden/weights_*.npz.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kMaxSys = 160;  // largest system (stencil size + polynomial terms)
constexpr int kMaxRhs = 16;   // largest number of right-hand sides

// Operator bits, the same values as include/rbf_b200.h.
enum : int {
    OP_INTERP = 1,
    OP_LAPLACE = 2,
    OP_DX = 4,
    OP_DY = 8,
    OP_DXX = 16,
    OP_DYY = 32,
    OP_DXY = 64,
};

inline int npoly(int P) { return P < 0 ? 0 : (P + 1) * (P + 2) / 2; }

// phi(r) = r^Q from r^2, src/rbf_operators.h:39-76: the Q = 3, 5, 7
// specialisations, else the generic loop.
inline double phs(int Q, double r2) {
    switch (Q) {
        case 3:
            return r2 * std::sqrt(r2);
        case 5:
            return r2 * r2 * std::sqrt(r2);
        case 7: {
            const double r4 = r2 * r2;
            return r4 * r2 * std::sqrt(r2);
        }
        default: {
            const double r = std::sqrt(r2);
            double p = r;
            for (int i = 0; i < (Q - 1) / 2; ++i) p *= r2;
            return p;
        }
    }
}

// r^m for odd m >= 1, the same product order as phs().
inline double rpow_odd(int m, double r2) { return m == 1 ? std::sqrt(r2) : phs(m, r2); }

// 2-D monomials of total degree <= P, ordered by degree d, then by the
// power j of y: x^(d-j) y^j. src/rbf_operators.h:81-99.
inline void monomials(int P, double x, double y, double* b, int inc) {
    double X[8], Y[8];
    X[0] = Y[0] = 1.0;
    for (int i = 1; i <= P; ++i) {
        X[i] = X[i - 1] * x;
        Y[i] = Y[i - 1] * y;
    }
    int k = 0;
    for (int d = 0; d <= P; ++d)
        for (int j = 0; j <= d; ++j) b[(k++) * inc] = X[d - j] * Y[j];
}

// Value of the differential operator `op` applied to monomial number i at
// the origin: only the monomials 1, x, y, x^2, xy, y^2 (i = 0..5) can be
// nonzero there.
inline double poly_op_at_origin(int op, int i) {
    switch (op) {
        case OP_LAPLACE: return (i == 3 || i == 5) ? 2.0 : 0.0;
        case OP_DX: return i == 1 ? 1.0 : 0.0;
        case OP_DY: return i == 2 ? 1.0 : 0.0;
        case OP_DXX: return i == 3 ? 2.0 : 0.0;
        case OP_DYY: return i == 5 ? 2.0 : 0.0;
        case OP_DXY: return i == 4 ? 1.0 : 0.0;
        default: return 0.0;
    }
}

// Operator applied in the evaluation point x_e to phi(|x_e - x_k|), at
// x_e = 0, for a node at (xk, yk) with r2 = xk^2 + yk^2:
//   d/dx  : -Q r^(Q-2) xk                d/dy : -Q r^(Q-2) yk
//   Lap   :  Q^2 r^(Q-2)
//   d2/dx2:  Q r^(Q-2) + Q(Q-2) r^(Q-2) xk^2 / r^2   (0 at r = 0)
//   d2/dy2:  likewise with yk;  d2/dxdy: Q(Q-2) r^(Q-2) xk yk / r^2
inline double phs_op_at_origin(int op, int Q, double xk, double yk, double r2) {
    const double rq2 = rpow_odd(Q - 2, r2);
    const double q = static_cast<double>(Q);
    switch (op) {
        case OP_LAPLACE: return (q * q) * rq2;
        case OP_DX: return -((q * rq2) * xk);
        case OP_DY: return -((q * rq2) * yk);
        case OP_DXX:
        case OP_DYY:
        case OP_DXY: {
            if (r2 == 0.0) return 0.0;
            const double a = q * rq2;
            const double b = (q * (q - 2.0)) * rq2;
            if (op == OP_DXX) return a + b * ((xk * xk) / r2);
            if (op == OP_DYY) return a + b * ((yk * yk) / r2);
            return b * ((xk * yk) / r2);
        }
        default: return 0.0;
    }
}

// Order of the derivative an operator takes: the power of the radius
// scale its weights carry.
inline int op_order(int op) {
    switch (op) {
        case OP_INTERP: return 0;
        case OP_DX:
        case OP_DY: return 1;
        default: return 2;
    }
}

// Right-hand-side columns in output order: nc interpolation points first
// (when OP_INTERP is set), then the derivative operators in bit order.
int rhs_columns(int ops, int nc, int* col_op) {
    int m = 0;
    if (ops & OP_INTERP)
        for (int j = 0; j < nc; ++j) col_op[m++] = OP_INTERP;
    for (int bit = OP_LAPLACE; bit <= OP_DXY; bit <<= 1)
        if (ops & bit) col_op[m++] = bit;
    return m;
}

// Power-of-two radius scale: returns e with 2^(e-1) <= max|d| < 2^e, so
// scaled coordinates ldexp(d, -e) lie in (-1, 1). e = 0 when all
// displacements are zero.
inline int scale_exponent(const double* xs, const double* ys, int k) {
    double m = 0.0;
    for (int j = 0; j < k; ++j) m = std::max(m, std::max(std::fabs(xs[j]), std::fabs(ys[j])));
    if (m == 0.0) return 0;
    int e;
    std::frexp(m, &e);
    return e;
}

// PeriodicBox::minimum_image, src/rbf_spatial.h:74-76.
inline double minimum_image(double d, double L) {
    if (L <= 0.0) return d;
    return d - L * std::rint(d / L);
}

struct Desc {
    int ops;
    int nc;
    const double* xc;  // interpolation points, stencil-local frame
    const double* yc;
    int scale;         // 1: power-of-two radius scaling
    double Lx, Ly;     // periods, <= 0 for an open axis
};

// The augmented system of one stencil, row-major a[r][c], r < n, c < W =
// n + nrhs, from the shifted (and scaled) coordinates xs, ys and the scale
// exponent e. The reference's saddle-point matrix [A P; P^T 0] (fill_matrix,
// src/rbf_operators.h:123-154) is formed with its polynomial block first:
// equations [P^T rows (np); node rows (k)], unknowns [lambda (np); w (k)].
// This relabelling of equations and unknowns fixes the elimination order the
// CUDA kernel uses; the solution is the reference system's. Right-hand-side
// column q is column n + q: fill_rhs (src/rbf_operators.h:158-185) for
// interpolation points, the operator at the centre otherwise.
void fill_system(const Desc& D, int P, int Q, int k, const double* xs, const double* ys, int e,
                 const int* col_op, int nrhs, double* a) {
    const int np = npoly(P);
    const int n = k + np;
    const int W = n + nrhs;
    std::fill(a, a + static_cast<size_t>(n) * W, 0.0);
    for (int i = 0; i < k; ++i) {
        double* row = a + static_cast<size_t>(np + i) * W;
        for (int j = 0; j < k; ++j) {
            const double dx = xs[j] - xs[i];
            const double dy = ys[j] - ys[i];
            row[np + j] = phs(Q, dx * dx + dy * dy);
        }
        double b[64];
        monomials(P, xs[i], ys[i], b, 1);
        for (int m = 0; m < np; ++m) {
            row[m] = b[m];                 // P block (node row i, monomial m)
            a[m * W + np + i] = b[m];      // P^T block (monomial row m, node i)
        }
    }
    int ic = 0;
    for (int q = 0; q < nrhs; ++q) {
        const int op = col_op[q];
        if (op == OP_INTERP) {
            // src/rbf_operators.h:158-185
            const double xe = std::ldexp(D.xc[ic], -e), ye = std::ldexp(D.yc[ic], -e);
            ++ic;
            for (int i = 0; i < k; ++i) {
                const double dx = xe - xs[i], dy = ye - ys[i];
                a[(np + i) * W + n + q] = phs(Q, dx * dx + dy * dy);
            }
            double b[64];
            monomials(P, xe, ye, b, 1);
            for (int m = 0; m < np; ++m) a[m * W + n + q] = b[m];
        } else {
            for (int i = 0; i < k; ++i) {
                const double r2 = xs[i] * xs[i] + ys[i] * ys[i];
                a[(np + i) * W + n + q] = phs_op_at_origin(op, Q, xs[i], ys[i], r2);
            }
            for (int m = 0; m < np; ++m) a[m * W + n + q] = poly_op_at_origin(op, m);
        }
    }
}

// Gather + FP64 shift to the stencil centre (src/rbf_operators.h:354-358),
// minimum image in a periodic box, and the power-of-two radius scale.
// Returns the scale exponent e (0 without scaling).
int stencil_coords(const Desc& D, int s, int k, const int* idx, const double* x, const double* y,
                   double* xs, double* ys) {
    const double x0 = x[s], y0 = y[s];
    for (int j = 0; j < k; ++j) {
        xs[j] = minimum_image(x[idx[j]] - x0, D.Lx);
        ys[j] = minimum_image(y[idx[j]] - y0, D.Ly);
    }
    const int e = D.scale ? scale_exponent(xs, ys, k) : 0;
    if (e != 0)
        for (int j = 0; j < k; ++j) {
            xs[j] = std::ldexp(xs[j], -e);
            ys[j] = std::ldexp(ys[j], -e);
        }
    return e;
}

// Assemble one stencil. idx[0..k) are the node indices (idx[0] the
// centre by convention, but the centre is node s whatever idx holds).
// Writes w[col][j] = weight of node idx[j] for right-hand side col into
// out[col] + j. Returns info: 0, or c + 1 for the first zero pivot.
int assemble_one(const Desc& D, int P, int Q, int s, int k, const int* idx, const double* x,
                 const double* y, double* const* out, long long out_off,
                 double* sol_out /* optional n*nrhs, row-major, solution incl. polynomial part */) {
    const int np = npoly(P);
    const int n = k + np;
    int col_op[kMaxRhs + 64];
    const int nrhs = rhs_columns(D.ops, D.nc, col_op);
    const int W = n + nrhs;

    double xs[kMaxSys], ys[kMaxSys];
    const int e = stencil_coords(D, s, k, idx, x, y, xs, ys);

    static thread_local std::vector<double> abuf;
    abuf.resize(static_cast<size_t>(n) * W);
    double* a = abuf.data();
    fill_system(D, P, Q, k, xs, ys, e, col_op, nrhs, a);

    // Gaussian elimination with row-implicit partial pivoting
    bool used[kMaxSys];
    int pstep_row[kMaxSys];  // row pivoted at step c
    double pinv[kMaxSys];    // 1 / pivot at step c
    std::fill(used, used + n, false);
    int info = 0;
    for (int c = 0; c < n; ++c) {
        // pivot: the unused row of largest |a(r,c)| compared by the high 32
        // bits of its binary64 representation without their 7 lowest bits
        // (the GPU reduces this as one 32-bit key with the row index in the
        // freed bits), ties to the lowest row
        int p = -1;
        uint64_t best = 0;
        for (int r = 0; r < n; ++r) {
            if (used[r]) continue;
            const double v = std::fabs(a[r * W + c]);
            uint64_t bits;
            std::memcpy(&bits, &v, sizeof bits);
            const uint64_t key = ((bits >> 32) >> 7) + 1;  // +1: an unused zero still counts
            if (key > best) {
                best = key;
                p = r;
            }
        }
        if (best <= 1) {  // zero pivot column
            info = c + 1;
            break;
        }
        used[p] = true;
        pstep_row[c] = p;
        const double inv = 1.0 / a[p * W + c];
        pinv[c] = inv;
        const double* u = a + static_cast<size_t>(p) * W;
        for (int r = 0; r < n; ++r) {
            if (used[r]) continue;
            double* ar = a + static_cast<size_t>(r) * W;
            const double l = ar[c] * inv;
            ar[c] = l;
            for (int j = c + 1; j < W; ++j) ar[j] = std::fma(-l, u[j], ar[j]);
        }
    }

    double* xsol = sol_out;
    std::vector<double> xtmp;
    if (!xsol) {
        xtmp.resize(static_cast<size_t>(n) * nrhs);
        xsol = xtmp.data();
    }
    if (info == 0) {
        // column-oriented back substitution on the transformed right-hand sides
        for (int c = n - 1; c >= 0; --c) {
            const int p = pstep_row[c];
            for (int q = 0; q < nrhs; ++q) xsol[c * nrhs + q] = a[p * W + n + q] * pinv[c];
            for (int t = 0; t < c; ++t) {
                const int r = pstep_row[t];
                const double urc = a[r * W + c];
                for (int q = 0; q < nrhs; ++q)
                    a[r * W + n + q] = std::fma(-urc, xsol[c * nrhs + q], a[r * W + n + q]);
            }
        }
    } else {
        const double nan = std::numeric_limits<double>::quiet_NaN();
        for (int i = 0; i < n * nrhs; ++i) xsol[i] = nan;
    }
    // scatter the k node weights (unknowns np..np+k-1), rescaled,
    // src/rbf_operators.h:368-375; the polynomial coefficients are dropped
    for (int q = 0; q < nrhs; ++q) {
        const int m = op_order(col_op[q]);
        double* dst = out[q] + out_off;
        for (int j = 0; j < k; ++j) dst[j] = std::ldexp(xsol[(np + j) * nrhs + q], -m * e);
    }
    return info;
}

int check_desc(const Desc& D, int P, int Q, int kmax) {
    if (P < -1 || P > 6) return -1;
    if (Q < 1 || Q % 2 == 0) return -1;
    if (kmax < 1 || kmax + npoly(P) > kMaxSys) return -1;
    int col_op[kMaxRhs + 64];
    if ((D.ops & OP_INTERP) && (D.nc < 1 || !D.xc || !D.yc)) return -1;
    if (D.nc > kMaxRhs) return -1;
    const int nrhs = rhs_columns(D.ops, D.nc, col_op);
    if (nrhs < 1 || nrhs > kMaxRhs) return -1;
    return nrhs;
}

}  // namespace

extern "C" {

// Threads used by the OpenMP loops below (0 = leave the runtime default).
void orc_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_npoly(int P) { return npoly(P); }

double orc_phs(int Q, double r2) { return phs(Q, r2); }

// Number of right-hand-side columns for an operator mask.
int orc_num_rhs(int ops, int nc) {
    int col_op[kMaxRhs + 64];
    return rhs_columns(ops, nc, col_op);
}

// Fixed-width stencils: ja has nstencils*k entries, row s at ja[s*k]
// (src/rbf_operators.h:307-313). out[q] has nstencils*k entries for each
// of the orc_num_rhs(ops, nc) columns. Returns the number of singular
// stencils (info != 0), or -1 on bad arguments.
long long orc_assemble_fixed(int nstencils, const double* x, const double* y, int k,
                             const int* ja, int P, int Q, int ops, int nc, const double* xc,
                             const double* yc, int scale, double Lx, double Ly,
                             double* const* out, int* info) {
    Desc D{ops, nc, xc, yc, scale, Lx, Ly};
    if (check_desc(D, P, Q, k) < 0 || nstencils < 0) return -1;
    long long bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : bad)
    for (int s = 0; s < nstencils; ++s) {
        const int st = assemble_one(D, P, Q, s, k, ja + static_cast<size_t>(s) * k, x, y, out,
                                    static_cast<long long>(s) * k, nullptr);
        if (info) info[s] = st;
        bad += (st != 0);
    }
    return bad;
}

// Ragged stencils in CSR form: row s holds ja[ia[s] .. ia[s+1]). degree
// is per stencil (P_s) or NULL for the uniform P; phs_q <= 0 selects
// Q_s = 2 P_s - 1 per stencil. out[q] has ia[nstencils] entries.
long long orc_assemble_csr(int nstencils, const double* x, const double* y, const int* ia,
                           const int* ja, const signed char* degree, int P, int Q, int ops,
                           int nc, const double* xc, const double* yc, int scale, double Lx,
                           double Ly, double* const* out, int* info) {
    Desc D{ops, nc, xc, yc, scale, Lx, Ly};
    long long bad = 0;
    int err = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : bad, err)
    for (int s = 0; s < nstencils; ++s) {
        const int ks = ia[s + 1] - ia[s];
        const int Ps = degree ? degree[s] : P;
        const int Qs = Q > 0 ? Q : 2 * Ps - 1;
        if (check_desc(D, Ps, Qs, ks) < 0) {
            err += 1;
            continue;
        }
        const int st = assemble_one(D, Ps, Qs, s, ks, ja + ia[s], x, y, out, ia[s], nullptr);
        if (info) info[s] = st;
        bad += (st != 0);
    }
    return err ? -1 : bad;
}

// One stencil's shifted (and scaled) coordinates xs, ys (k each) and its
// augmented system as the elimination receives it: row-major n x (n + nrhs),
// polynomial block first, right-hand sides as the last nrhs columns (see
// fill_system). Returns the scale exponent, or -1000 on bad arguments. For
// tests: pins the system against the reference's own fill_matrix/fill_rhs.
int orc_system(int s, const double* x, const double* y, int k, const int* idx, int P, int Q,
               int ops, int nc, const double* xc, const double* yc, int scale, double Lx,
               double Ly, double* xs, double* ys, double* a) {
    Desc D{ops, nc, xc, yc, scale, Lx, Ly};
    const int nrhs = check_desc(D, P, Q, k);
    if (nrhs < 0) return -1000;
    int col_op[kMaxRhs + 64];
    rhs_columns(D.ops, D.nc, col_op);
    const int e = stencil_coords(D, s, k, idx, x, y, xs, ys);
    fill_system(D, P, Q, k, xs, ys, e, col_op, nrhs, a);
    return e;
}

// One stencil's full solution, row-major n x nrhs in the scaled frame:
// polynomial coefficients (np rows) first, then the k weights. For tests.
int orc_solve_stencil(int s, const double* x, const double* y, int k, const int* idx, int P,
                      int Q, int ops, int nc, const double* xc, const double* yc, int scale,
                      double Lx, double Ly, double* sol, double* const* out) {
    Desc D{ops, nc, xc, yc, scale, Lx, Ly};
    if (check_desc(D, P, Q, k) < 0) return -1;
    return assemble_one(D, P, Q, s, k, idx, x, y, out, 0, sol);
}

// The saddle-point matrix of one stencil, column-major n x n with leading
// dimension ldm (fill_matrix's layout, src/rbf_operators.h:116-122), in the
// shifted frame and, with scale = 1, the scaled one; with shift = 0 from the
// absolute coordinates, as the Fortran fill_kernel (src/rbf_cuda.f90:56-70).
// Returns the scale exponent e.
int orc_fill_matrix(int s, const double* x, const double* y, int k, const int* idx, int P,
                    int Q, int scale, double Lx, double Ly, double* M, int ldm, int shift) {
    const int np = npoly(P);
    double xs[kMaxSys], ys[kMaxSys];
    const double x0 = shift ? x[s] : 0.0, y0 = shift ? y[s] : 0.0;
    for (int j = 0; j < k; ++j) {
        xs[j] = minimum_image(x[idx[j]] - x0, Lx);
        ys[j] = minimum_image(y[idx[j]] - y0, Ly);
    }
    const int e = scale ? scale_exponent(xs, ys, k) : 0;
    for (int j = 0; j < k; ++j) {
        xs[j] = std::ldexp(xs[j], -e);
        ys[j] = std::ldexp(ys[j], -e);
    }
    const int n = k + np;
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) M[r + c * ldm] = 0.0;
    for (int c = 0; c < k; ++c)
        for (int r = 0; r < k; ++r) {
            const double dx = xs[c] - xs[r];
            const double dy = ys[c] - ys[r];
            M[r + c * ldm] = phs(Q, dx * dx + dy * dy);
        }
    for (int r = 0; r < k; ++r) {
        monomials(P, xs[r], ys[r], &M[r + k * ldm], ldm);
        monomials(P, xs[r], ys[r], &M[k + r * ldm], 1);
    }
    return e;
}

// Brute-force k nearest neighbours of nq query points among n points,
// ordered by (squared distance, index). The squared distance is formed as
// the reference's searches form it: dx*dx + dy*dy of the plain differences
// (nanoflann, open plane), or of ckdtree's wrapped differences in a
// periodic box (Lx, Ly > 0). O(n) per query: small clouds only.
int orc_knn_brute(int n, const double* x, const double* y, int nq, const double* xq,
                  const double* yq, int k, double Lx, double Ly, int* ja, double* d2out) {
    if (k < 1 || k > n) return -1;
#pragma omp parallel
    {
        std::vector<std::pair<double, int>> cand(n);
#pragma omp for schedule(dynamic, 16)
        for (int q = 0; q < nq; ++q) {
            for (int j = 0; j < n; ++j) {
                double dx = xq[q] - x[j];
                double dy = yq[q] - y[j];
                if (Lx > 0) {  // ckdtree wrap_distance
                    const double hb = 0.5 * Lx;
                    if (dx < -hb) dx = Lx + dx;
                    else if (dx > hb) dx = dx - Lx;
                }
                if (Ly > 0) {
                    const double hb = 0.5 * Ly;
                    if (dy < -hb) dy = Ly + dy;
                    else if (dy > hb) dy = dy - Ly;
                }
                cand[j] = {dx * dx + dy * dy, j};
            }
            std::partial_sort(cand.begin(), cand.begin() + k, cand.end());
            for (int t = 0; t < k; ++t) {
                ja[static_cast<size_t>(q) * k + t] = cand[t].second;
                if (d2out) d2out[static_cast<size_t>(q) * k + t] = cand[t].first;
            }
        }
    }
    return 0;
}

// Squared distances of a stencil table, in the same arithmetic as
// orc_knn_brute; used to compare stencils up to tie order.
void orc_stencil_d2(int n, const double* x, const double* y, int k, const int* ja, double Lx,
                    double Ly, double* d2) {
#pragma omp parallel for schedule(static)
    for (int s = 0; s < n; ++s)
        for (int t = 0; t < k; ++t) {
            const int j = ja[static_cast<size_t>(s) * k + t];
            double dx = x[s] - x[j];
            double dy = y[s] - y[j];
            if (Lx > 0) {
                const double hb = 0.5 * Lx;
                if (dx < -hb) dx = Lx + dx;
                else if (dx > hb) dx = dx - Lx;
            }
            if (Ly > 0) {
                const double hb = 0.5 * Ly;
                if (dy < -hb) dy = Ly + dy;
                else if (dy > hb) dy = dy - Ly;
            }
            d2[static_cast<size_t>(s) * k + t] = dx * dx + dy * dy;
        }
}

}  // extern "C"

// ---- extended precision (x87 long double, 64-bit significand) -----------------
// The same system and elimination in long double, from the same FP64 node
// coordinates. Used only to measure how far FP64 (and the FP32-refined
// result) are from a more accurate solution on ill-conditioned stencils.
namespace {

inline long double phs_ld(int Q, long double r2) {
    const long double r = sqrtl(r2);
    long double p = r;
    for (int i = 0; i < (Q - 1) / 2; ++i) p *= r2;
    return p;
}

int assemble_one_ld(const Desc& D, int P, int Q, int s, int k, const int* idx, const double* x,
                    const double* y, double* const* out, long long out_off) {
    const int np = npoly(P);
    const int n = k + np;
    int col_op[kMaxRhs + 64];
    const int nrhs = rhs_columns(D.ops, D.nc, col_op);
    const int W = n + nrhs;
    std::vector<long double> xs(k), ys(k);
    double xd[kMaxSys], yd[kMaxSys];
    for (int j = 0; j < k; ++j) {
        xd[j] = minimum_image(x[idx[j]] - x[s], D.Lx);
        yd[j] = minimum_image(y[idx[j]] - y[s], D.Ly);
    }
    const int e = D.scale ? scale_exponent(xd, yd, k) : 0;
    for (int j = 0; j < k; ++j) {
        xs[j] = ldexpl((long double)xd[j], -e);
        ys[j] = ldexpl((long double)yd[j], -e);
    }
    std::vector<long double> a(static_cast<size_t>(n) * W, 0.0L);
    auto mono = [&](long double xx, long double yy, long double* b) {
        long double X[8], Y[8];
        X[0] = Y[0] = 1.0L;
        for (int i = 1; i <= P; ++i) { X[i] = X[i - 1] * xx; Y[i] = Y[i - 1] * yy; }
        int m = 0;
        for (int d = 0; d <= P; ++d)
            for (int j = 0; j <= d; ++j) b[m++] = X[d - j] * Y[j];
    };
    for (int i = 0; i < k; ++i) {
        long double* row = &a[static_cast<size_t>(np + i) * W];
        for (int j = 0; j < k; ++j) {
            const long double dx = xs[j] - xs[i], dy = ys[j] - ys[i];
            row[np + j] = phs_ld(Q, dx * dx + dy * dy);
        }
        long double b[64];
        mono(xs[i], ys[i], b);
        for (int m = 0; m < np; ++m) { row[m] = b[m]; a[m * W + np + i] = b[m]; }
    }
    for (int q = 0; q < nrhs; ++q) {
        const int op = col_op[q];
        for (int i = 0; i < k; ++i) {
            const long double xk = xs[i], yk = ys[i];
            const long double r2 = xk * xk + yk * yk;
            const long double rq2 = (Q - 2 == 1) ? sqrtl(r2) : phs_ld(Q - 2, r2);
            const long double qq = Q;
            long double v = 0.0L;
            switch (op) {
                case OP_LAPLACE: v = qq * qq * rq2; break;
                case OP_DX: v = -qq * rq2 * xk; break;
                case OP_DY: v = -qq * rq2 * yk; break;
                default: v = 0.0L; break;
            }
            a[(np + i) * W + n + q] = v;
        }
        for (int m = 0; m < np; ++m) a[m * W + n + q] = poly_op_at_origin(op, m);
    }
    std::vector<char> used(n, 0);
    std::vector<int> prow(n);
    for (int c = 0; c < n; ++c) {
        int p = -1;
        long double best = -1.0L;
        for (int r = 0; r < n; ++r)
            if (!used[r] && fabsl(a[r * W + c]) > best) { best = fabsl(a[r * W + c]); p = r; }
        if (!(best > 0.0L)) return c + 1;
        used[p] = 1;
        prow[c] = p;
        for (int r = 0; r < n; ++r) {
            if (used[r]) continue;
            const long double l = a[r * W + c] / a[p * W + c];
            a[r * W + c] = l;
            for (int j = c + 1; j < W; ++j) a[r * W + j] -= l * a[p * W + j];
        }
    }
    std::vector<long double> xsol(static_cast<size_t>(n) * nrhs);
    for (int c = n - 1; c >= 0; --c) {
        const int p = prow[c];
        for (int q = 0; q < nrhs; ++q) xsol[c * nrhs + q] = a[p * W + n + q] / a[p * W + c];
        for (int t = 0; t < c; ++t) {
            const int r = prow[t];
            for (int q = 0; q < nrhs; ++q) a[r * W + n + q] -= a[r * W + c] * xsol[c * nrhs + q];
        }
    }
    for (int q = 0; q < nrhs; ++q) {
        const int m = op_order(col_op[q]);
        for (int j = 0; j < k; ++j)
            out[q][out_off + j] = (double)ldexpl(xsol[(np + j) * nrhs + q], -m * e);
    }
    return 0;
}

}  // namespace

extern "C" long long orc_assemble_fixed_ld(int nstencils, const double* x, const double* y, int k,
                                           const int* ja, int P, int Q, int ops, int scale,
                                           double Lx, double Ly, double* const* out, int* info) {
    Desc D{ops, 0, nullptr, nullptr, scale, Lx, Ly};
    if ((ops & OP_INTERP) || check_desc(D, P, Q, k) < 0 || nstencils < 0) return -1;
    long long bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : bad)
    for (int s = 0; s < nstencils; ++s) {
        const int st = assemble_one_ld(D, P, Q, s, k, ja + static_cast<size_t>(s) * k, x, y, out,
                                       static_cast<long long>(s) * k);
        if (info) info[s] = st;
        bad += (st != 0);
    }
    return bad;
}

// Operator application with the boundary fix, in the order the CUDA kernel
// sums: acc = fma(values[s*k+j], u[ja[s*k+j]], acc) for j = 0..k-1 from zero;
// then out[bnd[b]] = u[bnd[b]].
extern "C" void orc_spmv(int n, int k, const int* ja, const double* values, const double* u,
                         double* out, const int* bnd, int nbnd) {
#pragma omp parallel for schedule(static)
    for (int s = 0; s < n; ++s) {
        double acc = 0.0;
        for (int j = 0; j < k; ++j)
            acc = std::fma(values[static_cast<size_t>(s) * k + j], u[ja[static_cast<size_t>(s) * k + j]], acc);
        out[s] = acc;
    }
    for (int b = 0; b < nbnd; ++b) out[bnd[b]] = u[bnd[b]];
}

// ---- node renumbering ------------------------------------------------------------
// Curve keys as zidx / hidx compute them (src/rbf_ordering.F90:82-218): at
// each of ndiv levels the key shifts by two bits, the quadrant q of the
// point against the box midpoint cx = x0 + 0.5 * (x1 - x0) (each operation
// rounded) is added (Morton) or mapped through the Hilbert state tables
// (table(q, rot), tr(q, rot)), and the box shrinks to that quadrant. bbox is
// {xmin, ymin, xmax, ymax}, NULL for the points' own (compute_bbox,
// src/rbf_reorder.h:60-66). curve 0 = Morton, 1 = Hilbert.
extern "C" int orc_curve_keys(int n, const double* x, const double* y, const double* bbox, int ndiv,
                              int curve, long long* keys) {
    if (n < 0 || ndiv < 1 || ndiv > 31 || (curve != 0 && curve != 1)) return -1;
    if (n == 0) return 0;
    double bb[4];
    if (bbox) {
        for (int i = 0; i < 4; ++i) bb[i] = bbox[i];
    } else {
        bb[0] = *std::min_element(x, x + n);
        bb[1] = *std::min_element(y, y + n);
        bb[2] = *std::max_element(x, x + n);
        bb[3] = *std::max_element(y, y + n);
    }
    // hidx's table(q, rot) and tr(q, rot), as [rot][q]
    static const int hdigit[4][4] = {{0, 3, 1, 2}, {2, 3, 1, 0}, {2, 1, 3, 0}, {0, 1, 3, 2}};
    static const int hnext[4][4] = {{3, 1, 0, 0}, {1, 0, 1, 2}, {2, 2, 3, 1}, {0, 3, 2, 3}};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double x0 = bb[0], y0 = bb[1], x1 = bb[2], y1 = bb[3];
        long long z = 0;
        int rot = 0;
        for (int l = 0; l < ndiv; ++l) {
            z <<= 2;
            const double cx = x0 + 0.5 * (x1 - x0);
            const double cy = y0 + 0.5 * (y1 - y0);
            const int q = (x[i] > cx ? 1 : 0) + (y[i] > cy ? 2 : 0);
            if (curve == 0) {
                z += q;
            } else {
                z += hdigit[rot][q];
                rot = hnext[rot][q];
            }
            if (x[i] > cx) x0 = cx; else x1 = cx;
            if (y[i] > cy) y0 = cy; else y1 = cy;
        }
        keys[i] = z;
    }
    return 0;
}

// morton_order / hilbert_order: indices stably sorted by key (order_by_keys,
// src/rbf_reorder.h:180-185). perm[i] = old index at new position i.
extern "C" int orc_curve_order(int n, const double* x, const double* y, const double* bbox,
                               int ndiv, int curve, int* perm) {
    std::vector<long long> keys(static_cast<size_t>(std::max(n, 0)));
    if (orc_curve_keys(n, x, y, bbox, ndiv, curve, keys.data()) < 0) return -1;
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::stable_sort(perm, perm + n, [&keys](int a, int b) { return keys[a] < keys[b]; });
    return 0;
}

// boundary_last_by_flag (src/rbf_reorder.h:232-244): stable partition,
// nonzero flag last.
extern "C" void orc_boundary_last(int n, const int* flag, int* perm) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::stable_partition(perm, perm + n, [flag](int i) { return flag[i] == 0; });
}

// renumber_stencils (src/rbf_reorder.h:272-281), out of place:
// out[s*k+j] = inv[ja[perm[s]*k+j]].
extern "C" void orc_renumber_stencils(int n, int k, const int* ja, const int* perm, int* out) {
    std::vector<int> inv(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) inv[perm[i]] = i;
    for (int s = 0; s < n; ++s)
        for (int j = 0; j < k; ++j)
            out[static_cast<size_t>(s) * k + j] = inv[ja[static_cast<size_t>(perm[s]) * k + j]];
}

// renumber_csr (src/rbf_reorder.h:286-303), out of place.
extern "C" void orc_renumber_csr(int n, const int* ia, const int* ja, const int* perm, int* ia_out,
                                 int* ja_out) {
    std::vector<int> inv(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) inv[perm[i]] = i;
    ia_out[0] = 0;
    for (int i = 0; i < n; ++i) {
        const int a = ia[perm[i]], b = ia[perm[i] + 1];
        for (int t = a; t < b; ++t) ja_out[ia_out[i] + (t - a)] = inv[ja[t]];
        ia_out[i + 1] = ia_out[i] + (b - a);
    }
}

// ---- iterative solve ---------------------------------------------------------------
// BiCGSTAB (van der Vorst, 1992) on the operator orc_spmv applies: stencil
// rows (fixed width k, or CSR rows when ia is given) with identity rows at
// the boundary list; the solve the reference leaves after building that
// operator (src/main.cpp:57-68). Every sum is taken in the order the CUDA
// solver takes it, so results agree bit for bit: rows in fused
// multiply-adds from zero; thread T = b * 256 + t of a grid of `grid` blocks
// owns rows T, T + 256 * grid, ... in ascending order; a warp sums by an
// xor butterfly over rounds 16, 8, 4, 2, 1; a block by the butterfly over
// its 8 warp sums (lanes 8..31 zero); the grid by thread t adding the
// partials of blocks t, t + 256, ... and the block butterfly of those.
// Returns 0 (converged), -10 (maxit reached), -11 (breakdown) or -1 (bad
// argument), as rbfb_solve_bicgstab.
namespace {

double butterfly32(double* v) {
    double t[32];
    for (int o = 16; o; o >>= 1) {
        for (int l = 0; l < 32; ++l) t[l] = v[l] + v[l ^ o];
        for (int l = 0; l < 32; ++l) v[l] = t[l];
    }
    return v[0];
}

double block_butterfly(const double* th) {  // 256 thread values
    double lanes[32], ws[8];
    for (int w = 0; w < 8; ++w) {
        for (int l = 0; l < 32; ++l) lanes[l] = th[w * 32 + l];
        ws[w] = butterfly32(lanes);
    }
    for (int l = 0; l < 32; ++l) lanes[l] = l < 8 ? ws[l] : 0.0;
    return butterfly32(lanes);
}

struct SolveSums {
    int n, grid;
    std::vector<double> th, part, g;
    SolveSums(int n_, int grid_)
        : n(n_), grid(grid_), th(static_cast<size_t>(grid_) * 256), part(grid_), g(256) {}
    double dot(const double* x, const double* y) {
        std::fill(th.begin(), th.end(), 0.0);
        const size_t nt = th.size();
        for (size_t s = 0; s < static_cast<size_t>(n); ++s) th[s % nt] = std::fma(x[s], y[s], th[s % nt]);
        for (int b = 0; b < grid; ++b) part[b] = block_butterfly(&th[static_cast<size_t>(b) * 256]);
        for (int t = 0; t < 256; ++t) {
            double a = 0.0;
            for (int b = t; b < grid; b += 256) a += part[b];
            g[t] = a;
        }
        return block_butterfly(g.data());
    }
};

template <class W>
double apply_row(int s, int k, const int* ia, const int* ja, const double* values,
                 const std::vector<unsigned char>& bflag, W w) {
    if (bflag[s]) return w(s);
    const long long b = ia ? ia[s] : static_cast<long long>(s) * k;
    const long long e = ia ? ia[s + 1] : b + k;
    double acc = 0.0;
    for (long long q = b; q < e; ++q) acc = std::fma(values[q], w(ja[q]), acc);
    return acc;
}

}  // namespace

extern "C" int orc_solve_grid(int n, int sms) {
    const long long want = (static_cast<long long>(n) + 255) / 256;
    return static_cast<int>(std::max(1LL, std::min(want, 6LL * sms)));
}

extern "C" int orc_bicgstab(int n, int k, const int* ia, const int* ja, const double* values,
                            const int* bnd, int nbnd, const double* f, double* u, double tol,
                            int maxit, int grid, int* iters, double* relres) {
    *iters = 0;
    *relres = 0.0;
    if (n < 0 || nbnd < 0 || maxit < 0 || !(tol >= 0.0) || !std::isfinite(tol) || (!ia && k < 1) ||
        grid < 1)
        return -1;
    if (n == 0) return 0;
    std::vector<unsigned char> bflag(n, 0);
    for (int b = 0; b < nbnd; ++b) {
        if (bnd[b] < 0 || bnd[b] >= n) return -1;
        bflag[bnd[b]] = 1;
    }
    const size_t N = n;
    std::vector<double> r(N), rh(N), p(N, 0.0), v(N, 0.0), s(N), t(N);
    SolveSums sums(n, grid);
    for (int i = 0; i < n; ++i) {
        r[i] = f[i] - apply_row(i, k, ia, ja, values, bflag, [u](int j) { return u[j]; });
        rh[i] = r[i];
    }
    double rr = sums.dot(r.data(), r.data());
    const double ff = sums.dot(f, f);
    const double thresh2 = tol * tol * ff;
    auto finish = [&](int code) {
        *relres = ff > 0.0 ? std::sqrt(rr / ff) : 0.0;
        return code;
    };
    if (!std::isfinite(rr) || !std::isfinite(ff)) return finish(-11);
    if (rr <= thresh2) return finish(0);
    if (ff == 0.0) {
        std::fill(u, u + n, 0.0);
        return 0;
    }
    if (maxit <= 0) return finish(-10);
    double rho = rr, alpha = 1.0, omega = 1.0, beta = 0.0;
    int iter = 0;
    for (;;) {
        for (int i = 0; i < n; ++i) p[i] = std::fma(beta, std::fma(-omega, v[i], p[i]), r[i]);
        for (int i = 0; i < n; ++i)
            v[i] = apply_row(i, k, ia, ja, values, bflag, [&p](int j) { return p[j]; });
        const double sigma = sums.dot(rh.data(), v.data());
        if (sigma == 0.0 || !std::isfinite(sigma)) return finish(-11);
        alpha = rho / sigma;
        for (int i = 0; i < n; ++i) s[i] = std::fma(-alpha, v[i], r[i]);
        for (int i = 0; i < n; ++i)
            t[i] = apply_row(i, k, ia, ja, values, bflag, [&s](int j) { return s[j]; });
        const double ts = sums.dot(t.data(), s.data());
        const double tt = sums.dot(t.data(), t.data());
        const double ss = sums.dot(s.data(), s.data());
        bool pending = false;
        if (ss <= thresh2) {
            omega = 0.0;
        } else if (tt == 0.0 || !std::isfinite(tt) || !std::isfinite(ts)) {
            omega = 0.0;
            pending = true;
        } else {
            omega = ts / tt;
        }
        for (int i = 0; i < n; ++i) {
            u[i] = std::fma(omega, s[i], std::fma(alpha, p[i], u[i]));
            r[i] = std::fma(-omega, t[i], s[i]);
        }
        const double rho_new = sums.dot(rh.data(), r.data());
        rr = sums.dot(r.data(), r.data());
        *iters = ++iter;
        if (!std::isfinite(rr)) return finish(-11);
        if (rr <= thresh2) return finish(0);
        if (pending || omega == 0.0) return finish(-11);
        if (iter >= maxit) return finish(-10);
        if (rho_new == 0.0 || !std::isfinite(rho_new)) return finish(-11);
        beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
    }
}

// ---- D2Q9 lattice Boltzmann -------------------------------------------------
//
// Restates feq_kernel, macros_kernel and bgk_kernel_split of the reference
// (src/lbm/d2q9_kernels.cu:13-150; lattice constants src/lbm/d2q9_kernels.h:
// 16-31) for float and double: every product, sum and quotient in the
// source's order, each rounded once (this file is compiled with
// -ffp-contract=off). Planar storage, direction a of node i at pdf[i + n*a].
// The streaming step (which the reference does not ship) sums the
// interpolation weights times the gathered populations in the order the CUDA
// kernel does: in entry order, w_0 * f_0 rounded, then one fused
// multiply-add per entry j = 1 .. k-1.
namespace lbm {

template <typename T>
struct Lat {
    static constexpr T w0 = T(4) / T(9);
    static constexpr T ws = T(1) / T(9);
    static constexpr T wd = T(1) / T(36);
    static constexpr T three_w0 = T(3) * w0;
    static constexpr T three_ws = T(3) * ws;
    static constexpr T three_wd = T(3) * wd;
    static constexpr T one_third = T(1) / T(3);
    static constexpr T one_half = T(1) / T(2);
    static constexpr T three_halves = T(3) / T(2);
};

template <typename T>
void moments(const T* f, T& rho, T& ux, T& uy) {
    rho = (((f[5] + f[7]) + (f[6] + f[8])) + ((f[1] + f[3]) + (f[2] + f[4]))) + f[0];
    const T invrho = T(1) / rho;
    ux = invrho * (((f[5] - f[7]) + (f[8] - f[6])) + (f[1] - f[3]));
    uy = invrho * (((f[5] - f[7]) + (f[6] - f[8])) + (f[2] - f[4]));
}

// out[a] = s_a * rho * term_a + omegabar * f[a] (omegabar * f absent when
// f == nullptr: the equilibrium itself, feq_kernel's form)
template <typename T>
void relax(const T* f, T omegabar, T s0, T ss, T sd, T rho, T ux, T uy, T* out, T* indp_out) {
    using L = Lat<T>;
    const T uxsq = ux * ux;
    const T uysq = uy * uy;
    const T indp = L::one_third - L::one_half * (uxsq + uysq);
    if (indp_out) *indp_out = indp;
    T term[9];
    term[0] = indp;
    const T v13 = indp + L::three_halves * uxsq;
    term[1] = v13 + ux;
    term[3] = v13 - ux;
    const T v24 = indp + L::three_halves * uysq;
    term[2] = v24 + uy;
    term[4] = v24 - uy;
    const T xpy = ux + uy;
    const T v57 = indp + L::three_halves * xpy * xpy;
    term[5] = v57 + xpy;
    term[7] = v57 - xpy;
    const T xmy = ux - uy;
    const T v68 = indp + L::three_halves * xmy * xmy;
    term[6] = v68 - xmy;
    term[8] = v68 + xmy;
    const T sc[9] = {s0, ss, ss, ss, ss, sd, sd, sd, sd};
    for (int a = 0; a < 9; ++a) {
        const T e = sc[a] * rho * term[a];
        out[a] = f ? omegabar * f[a] + e : e;
    }
}

template <typename T>
void feq(int n, const T* rho, const T* ux, const T* uy, T* pdf) {
    using L = Lat<T>;
    const size_t N = static_cast<size_t>(n);
    for (int i = 0; i < n; ++i) {
        T out[9];
        relax<T>(nullptr, T(0), L::three_w0, L::three_ws, L::three_wd, rho[i], ux[i], uy[i], out,
                 nullptr);
        for (int a = 0; a < 9; ++a) pdf[i + N * a] = out[a];
    }
}

template <typename T>
void collide(const T* f, T omega, T* out, T* rho, T* ux, T* uy, T* indp) {
    using L = Lat<T>;
    const T omegabar = T(1) - omega;
    moments(f, *rho, *ux, *uy);
    relax<T>(f, omegabar, omega * L::three_w0, omega * L::three_ws, omega * L::three_wd, *rho,
             *ux, *uy, out, indp);
}

template <typename T>
void bgk(int n, T omega, T* pdf, T* rho, T* ux, T* uy, T* indp) {
    const size_t N = static_cast<size_t>(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        T f[9], o[9], d;
        for (int a = 0; a < 9; ++a) f[a] = pdf[i + N * a];
        collide(f, omega, o, rho + i, ux + i, uy + i, &d);
        if (indp) indp[i] = d;
        for (int a = 0; a < 9; ++a) pdf[i + N * a] = o[a];
    }
}

template <typename T>
void macros(int n, const T* pdf, T* rho, T* ux, T* uy) {
    const size_t N = static_cast<size_t>(n);
    for (int i = 0; i < n; ++i) {
        T f[9];
        for (int a = 0; a < 9; ++a) f[a] = pdf[i + N * a];
        moments(f, rho[i], ux[i], uy[i]);
    }
}

template <typename T>
T fma_t(T a, T b, T c) {
    return std::fma(a, b, c);
}

template <typename T>
void stream_collide(int n, int k, const int* ja, const double* W, T omega, const T* pin, T* pout,
                    T* rho, T* ux, T* uy) {
    const size_t N = static_cast<size_t>(n);
    const size_t nnz = N * static_cast<size_t>(k);
#pragma omp parallel for schedule(static)
    for (int s = 0; s < n; ++s) {
        const size_t row = static_cast<size_t>(s) * k;
        T f[9];
        f[0] = pin[s];
        for (int a = 1; a < 9; ++a) {
            const double* Wa = W + static_cast<size_t>(a - 1) * nnz + row;
            const T* pa = pin + N * a;
            T v = static_cast<T>(Wa[0]) * pa[ja[row]];
            for (int j = 1; j < k; ++j) v = fma_t(static_cast<T>(Wa[j]), pa[ja[row + j]], v);
            f[a] = v;
        }
        T o[9], r, u, w, d;
        collide(f, omega, o, &r, &u, &w, &d);
        for (int a = 0; a < 9; ++a) pout[s + N * a] = o[a];
        if (rho) rho[s] = r;
        if (ux) ux[s] = u;
        if (uy) uy[s] = w;
    }
}

}  // namespace lbm

extern "C" {

// precision 0: double arrays, 1: float arrays (RBFB_LBM_FP64 / RBFB_LBM_FP32)
void orc_lbm_feq(int n, int precision, const void* rho, const void* ux, const void* uy, void* pdf) {
    if (precision == 0)
        lbm::feq<double>(n, static_cast<const double*>(rho), static_cast<const double*>(ux),
                         static_cast<const double*>(uy), static_cast<double*>(pdf));
    else
        lbm::feq<float>(n, static_cast<const float*>(rho), static_cast<const float*>(ux),
                        static_cast<const float*>(uy), static_cast<float*>(pdf));
}

void orc_lbm_macros(int n, int precision, const void* pdf, void* rho, void* ux, void* uy) {
    if (precision == 0)
        lbm::macros<double>(n, static_cast<const double*>(pdf), static_cast<double*>(rho),
                            static_cast<double*>(ux), static_cast<double*>(uy));
    else
        lbm::macros<float>(n, static_cast<const float*>(pdf), static_cast<float*>(rho),
                           static_cast<float*>(ux), static_cast<float*>(uy));
}

void orc_lbm_bgk(int n, int precision, double omega, void* pdf, void* rho, void* ux, void* uy,
                 void* indp) {
    if (precision == 0)
        lbm::bgk<double>(n, omega, static_cast<double*>(pdf), static_cast<double*>(rho),
                         static_cast<double*>(ux), static_cast<double*>(uy),
                         static_cast<double*>(indp));
    else
        lbm::bgk<float>(n, static_cast<float>(omega), static_cast<float*>(pdf),
                        static_cast<float*>(rho), static_cast<float*>(ux), static_cast<float*>(uy),
                        static_cast<float*>(indp));
}

void orc_lbm_stream_collide(int n, int precision, int k, const int* ja, const double* W,
                            double omega, const void* pin, void* pout, void* rho, void* ux,
                            void* uy) {
    if (precision == 0)
        lbm::stream_collide<double>(n, k, ja, W, omega, static_cast<const double*>(pin),
                                    static_cast<double*>(pout), static_cast<double*>(rho),
                                    static_cast<double*>(ux), static_cast<double*>(uy));
    else
        lbm::stream_collide<float>(n, k, ja, W, static_cast<float>(omega),
                                   static_cast<const float*>(pin), static_cast<float*>(pout),
                                   static_cast<float*>(rho), static_cast<float*>(ux),
                                   static_cast<float*>(uy));
}

}  // extern "C"
