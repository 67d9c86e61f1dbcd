// compat.cu -- counterparts of the reference's smaller GPU entry points:
//
//   solve_dp              extern "C" __global__ kernel with the reference's
//                         signature (src/rbf_operators.cpp:7-11): one 15x15
//                         system, 9 right-hand sides, FP64, <<<1, 32>>>;
//   rbfb_fill_matrices    fill_matrix (src/rbf_operators.h:116-154) in the
//                         shifted (and scaled) frame of the assembly;
//   rbfb_fill_kernel      the Fortran fill_kernel (src/rbf_cuda.f90:36-99):
//                         degree 2, r^3, absolute coordinates;
//   rbfb_fill_rhs         the Fortran fill_rhs (src/rbf_cuda.f90:101-136);
//   rbfb_store_to_csr     the Fortran store_to_csr (src/rbf_cuda.f90:139-157)
//                         over every stencil, rbfb_store_to_csr_stencil for
//                         one stencil with its arguments.
#include <cuda_runtime.h>

#include <algorithm>

#include "asm_math.cuh"
#include "runtime.h"

namespace rbfb {

// ---- solve_dp --------------------------------------------------------------------
// Gaussian elimination with partial pivoting and row interchanges, LAPACK
// getrf/getrs conventions: ipiv[j] (1-based) is the row swapped with row j
// at step j; the pivot is the first row of largest |a| (idamax); info = j+1
// at the first exactly zero pivot, in which case B is left unsolved.
constexpr int kDpN = 15, kDpRhs = 9;

}  // namespace rbfb

extern "C" __global__ void __launch_bounds__(32) solve_dp(double* A, int* ipiv, double* B,
                                                          int* info) {
    using namespace rbfb;
    __shared__ double a[kDpN][kDpN + 1];  // a[col][row]
    __shared__ double b[kDpRhs][kDpN + 1];
    __shared__ int piv[kDpN];
    const int lane = threadIdx.x;
    for (int i = lane; i < kDpN * kDpN; i += 32) a[i / kDpN][i % kDpN] = A[i];
    for (int i = lane; i < kDpN * kDpRhs; i += 32) b[i / kDpN][i % kDpN] = B[i];
    __syncwarp();
    int inf = 0;
    for (int j = 0; j < kDpN; ++j) {
        // pivot: first index of the largest |a(r, j)|, r >= j
        double v = (lane >= j && lane < kDpN) ? fabs(a[j][lane]) : -1.0;
        int r = lane;
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_down_sync(0xffffffffu, v, o);
            const int r2 = __shfl_down_sync(0xffffffffu, r, o);
            if (v2 > v || (v2 == v && r2 < r)) {
                v = v2;
                r = r2;
            }
        }
        r = __shfl_sync(0xffffffffu, r, 0);
        v = __shfl_sync(0xffffffffu, v, 0);
        if (lane == 0) piv[j] = r;
        if (v == 0.0 && inf == 0) inf = j + 1;
        // swap rows j and r in A (all columns) and B
        if (r != j) {
            for (int c = lane; c < kDpN + kDpRhs; c += 32) {
                double* col = c < kDpN ? a[c] : b[c - kDpN];
                const double t = col[j];
                col[j] = col[r];
                col[r] = t;
            }
        }
        __syncwarp();
        if (v != 0.0) {
            const double inv = 1.0 / a[j][j];
            if (lane > j && lane < kDpN) a[j][lane] *= inv;
            __syncwarp();
            // trailing update, one column per lane (A and B)
            for (int c = j + 1 + lane; c < kDpN + kDpRhs; c += 32) {
                double* col = c < kDpN ? a[c] : b[c - kDpN];
                const double u = col[j];
                for (int rr = j + 1; rr < kDpN; ++rr) col[rr] = fma(-a[j][rr], u, col[rr]);
            }
        }
        __syncwarp();
    }
    if (inf == 0) {
        // back substitution, one right-hand side per lane
        if (lane < kDpRhs) {
            double* x = b[lane];
            for (int i = kDpN - 1; i >= 0; --i) {
                double s = x[i];
                for (int c = i + 1; c < kDpN; ++c) s = fma(-a[c][i], x[c], s);
                x[i] = s / a[i][i];
            }
        }
    }
    __syncwarp();
    for (int i = lane; i < kDpN * kDpN; i += 32) A[i] = a[i / kDpN][i % kDpN];
    if (inf == 0)
        for (int i = lane; i < kDpN * kDpRhs; i += 32) B[i] = b[i / kDpN][i % kDpN];
    if (lane < kDpN) ipiv[lane] = piv[lane] + 1;
    if (lane == 0) *info = inf;
}

namespace rbfb {

// ---- fill_matrix ------------------------------------------------------------------
// One warp per stencil; M + s*ldm*ldm is the column-major saddle-point matrix
// [A P; P^T 0] of stencil s in the reference's layout and arithmetic order.
// shift = 0 fills from the absolute coordinates, as the Fortran fill_kernel
// does (subtracting a zero centre is exact).
template <int P>
__global__ void fill_kernel(int nstencils, const double* x, const double* y, const int* ia,
                            const int* ja, int Q, int scale, double Lx, double Ly, double* M,
                            int ldm, int shift) {
    const int lane = threadIdx.x & 31;
    const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    constexpr int NP = npoly(P);
    for (int s = wg; s < nstencils; s += nw) {
        const int off = ia[s], k = ia[s + 1] - ia[s];
        if (k < 1 || k + NP > ldm) continue;  // does not fit its slab: left untouched
        double* Ms = M + static_cast<size_t>(s) * ldm * ldm;
        const double x0 = shift ? x[s] : 0.0, y0 = shift ? y[s] : 0.0;
        int emax = -100000;
        for (int j = lane; j < k; j += 32) {
            const int nb = ja[off + j];
            const double dx = min_image(dsub(x[nb], x0), Lx);
            const double dy = min_image(dsub(y[nb], y0), Ly);
            if (dx != 0.0) emax = max(emax, ilogb(fabs(dx)) + 1);
            if (dy != 0.0) emax = max(emax, ilogb(fabs(dy)) + 1);
        }
        int e = __reduce_max_sync(0xffffffffu, emax);
        e = (scale && e > -100000) ? e : 0;
        const int n = k + NP;
        for (int col = 0; col < n; ++col)
            for (int r = lane; r < n; r += 32) {
                double v = 0.0;
                if (col < k && r < k) {
                    const int a = ja[off + col], b = ja[off + r];
                    const double xc = scalbn(min_image(dsub(x[a], x0), Lx), -e);
                    const double yc = scalbn(min_image(dsub(y[a], y0), Ly), -e);
                    const double xr = scalbn(min_image(dsub(x[b], x0), Lx), -e);
                    const double yr = scalbn(min_image(dsub(y[b], y0), Ly), -e);
                    const double r2 = dist2(dsub(xc, xr), dsub(yc, yr));
                    switch (Q) {
                        case 1: v = phs64<1>(r2); break;
                        case 3: v = phs64<3>(r2); break;
                        case 5: v = phs64<5>(r2); break;
                        case 7: v = phs64<7>(r2); break;
                        default: v = phs64<9>(r2); break;
                    }
                } else if (col >= k && r < k) {
                    const int b = ja[off + r];
                    double mon[NP];
                    monomials<P>(scalbn(min_image(dsub(x[b], x0), Lx), -e),
                                 scalbn(min_image(dsub(y[b], y0), Ly), -e), mon);
#pragma unroll
                    for (int m = 0; m < NP; ++m)
                        if (m == col - k) v = mon[m];
                } else if (col < k && r >= k) {
                    const int b = ja[off + col];
                    double mon[NP];
                    monomials<P>(scalbn(min_image(dsub(x[b], x0), Lx), -e),
                                 scalbn(min_image(dsub(y[b], y0), Ly), -e), mon);
#pragma unroll
                    for (int m = 0; m < NP; ++m)
                        if (m == r - k) v = mon[m];
                }
                Ms[r + static_cast<size_t>(col) * ldm] = v;
            }
    }
}

// The Fortran fill_rhs: B(k, j) = |(xc_j, yc_j) - (x_k, y_k)|^3 for the n
// stencil nodes, B(n + i, j) = monomial i (degree 2) at (xc_j, yc_j);
// column-major with leading dimension ldb. One warp per column.
__global__ void fill_rhs_kernel(int n, const double* x, const double* y, int nc, const double* xc,
                                const double* yc, double* B, int ldb) {
    const int lane = threadIdx.x & 31;
    const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = wg; j < nc; j += nw) {
        double* Bj = B + static_cast<size_t>(j) * ldb;
        const double xe = xc[j], ye = yc[j];
        for (int k = lane; k < n; k += 32) Bj[k] = phs64<3>(dist2(dsub(xe, x[k]), dsub(ye, y[k])));
        if (lane == 0) {
            double mon[6];
            monomials<2>(xe, ye, mon);
            for (int m = 0; m < 6; ++m) Bj[n + m] = mon[m];
        }
    }
}

// The Fortran store_to_csr for stencil idx: va[ia[idx] + k] = W(k,1) + W(k,2)
// for the stencil's nodes, W column-major with leading dimension ldw.
__global__ void store_to_csr_one_kernel(const int* ia, double* va, const double* W, int ldw,
                                        int idx) {
    const int a = ia[idx], n = ia[idx + 1] - a;
    for (int k = threadIdx.x; k < n; k += blockDim.x) va[a + k] = W[k] + W[k + ldw];
}

__global__ void store_to_csr_kernel(int nstencils, const int* ia, const double* wxx,
                                     const double* wyy, double* va) {
    const int nnz = ia[nstencils] - ia[0];
    const int base = ia[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x)
        va[base + i] = wxx[base + i] + wyy[base + i];
}

}  // namespace rbfb

using namespace rbfb;

extern "C" {

int rbfb_solve_dp(double* A, int* ipiv, double* B, int* info, void* stream) {
    if (!A || !ipiv || !B || !info) return RBFB_EINVAL;
    solve_dp<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(A, ipiv, B, info);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_fill_matrices(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                       const double* y, const int* ia, const int* ja, double* M, int ldm,
                       void* stream) {
    if (!ctx || !desc || !x || !y || !ia || !ja || !M) return fail(ctx, RBFB_EINVAL, "null argument");
    if (nstencils < 0 || ldm < 1) return fail(ctx, RBFB_EINVAL, "bad sizes");
    const int P = desc->degree;
    const int Q = desc->phs ? desc->phs : 2 * P - 1;
    if (P < 0 || P > 4 || Q < 1 || Q > 9 || Q % 2 == 0)
        return fail(ctx, RBFB_EUNSUPPORTED, "fill supports P 0..4, odd Q 1..9");
    if (nstencils == 0) return RBFB_OK;
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = std::max(1, std::min((nstencils + 3) / 4, ctx->sms * 8));
    const double Lx = desc->period[0], Ly = desc->period[1];
    switch (P) {
        case 0: fill_kernel<0><<<blocks, 128, 0, st>>>(nstencils, x, y, ia, ja, Q, desc->scale, Lx, Ly, M, ldm, 1); break;
        case 1: fill_kernel<1><<<blocks, 128, 0, st>>>(nstencils, x, y, ia, ja, Q, desc->scale, Lx, Ly, M, ldm, 1); break;
        case 2: fill_kernel<2><<<blocks, 128, 0, st>>>(nstencils, x, y, ia, ja, Q, desc->scale, Lx, Ly, M, ldm, 1); break;
        case 3: fill_kernel<3><<<blocks, 128, 0, st>>>(nstencils, x, y, ia, ja, Q, desc->scale, Lx, Ly, M, ldm, 1); break;
        default: fill_kernel<4><<<blocks, 128, 0, st>>>(nstencils, x, y, ia, ja, Q, desc->scale, Lx, Ly, M, ldm, 1); break;
    }
    ctx->launches += 1;
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

int rbfb_fill_kernel(int nstencils, const double* x, const double* y, const int* ia,
                     const int* ja, double* M, int ldm, void* stream) {
    if (!x || !y || !ia || !ja || !M) return RBFB_EINVAL;
    if (nstencils < 0 || ldm < 1) return RBFB_EINVAL;
    if (nstencils == 0) return RBFB_OK;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return RBFB_ECUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = std::max(1, std::min((nstencils + 3) / 4, std::max(sms, 1) * 8));
    fill_kernel<2><<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        nstencils, x, y, ia, ja, 3, 0, 0.0, 0.0, M, ldm, 0);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_fill_rhs(int n, const double* x, const double* y, int nc, const double* xc,
                  const double* yc, double* B, int ldb, void* stream) {
    if (n < 0 || nc < 0 || ldb < n + 6) return RBFB_EINVAL;
    if (nc == 0) return RBFB_OK;
    if (!x || !y || !xc || !yc || !B) return RBFB_EINVAL;
    const int blocks = std::max(1, std::min((nc + 3) / 4, 1024));
    fill_rhs_kernel<<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(n, x, y, nc, xc, yc, B,
                                                                           ldb);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_store_to_csr_stencil(int nstencils, const int* ia, double* va, const double* W, int ldw,
                              int idx, void* stream) {
    if (!ia || !va || !W || idx < 0 || idx >= nstencils || ldw < 1) return RBFB_EINVAL;
    store_to_csr_one_kernel<<<1, 128, 0, static_cast<cudaStream_t>(stream)>>>(ia, va, W, ldw, idx);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_store_to_csr(int nstencils, const int* ia, const double* wxx, const double* wyy,
                      double* va, void* stream) {
    if (nstencils < 0 || !ia || !wxx || !wyy || !va) return RBFB_EINVAL;
    if (nstencils == 0) return RBFB_OK;
    store_to_csr_kernel<<<256, 256, 0, static_cast<cudaStream_t>(stream)>>>(nstencils, ia, wxx, wyy, va);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

}  // extern "C"
