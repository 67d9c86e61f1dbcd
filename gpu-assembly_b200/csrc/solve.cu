// solve.cu -- BiCGSTAB on an assembled operator: A u = f, where A is the
// stencil operator with identity rows at the listed boundary nodes (the
// mv_op the reference builds after its assembly and leaves unsolved,
// src/main.cpp:57-68).
//
// The method is van der Vorst's BiCGSTAB (1992) without a preconditioner:
//
//   r = f - A u, rh = r, rho = (rh, r), p = v = 0, beta = 0
//   repeat: p = r + beta (p - omega v)
//           v = A p;            alpha = rho / (rh, v)
//           s = r - alpha v;    t = A s;   omega = (t, s) / (t, t)
//           u = u + alpha p + omega s;     r = s - omega t
//           stop when (r, r) <= tol^2 (f, f); beta = ((rh, r) / rho) (alpha / omega)
//
// The iteration streams memory, so HBM bandwidth is its roofline: each step
// reads the operator (12 B per stored weight, twice) and a handful of
// vectors. What holds the operator passes below it is the latency of their
// gathers (one per stored weight), which each thread hides by summing its
// own row in row order with eight gathers in flight (row_sum.cuh). It is
// laid out as five kernels per iteration, each one pass over the rows:
//   p_kernel       p = r + beta (p - omega v)
//   spmv_v_kernel  v = A p, with the partial sums of (rh, v)
//   s_kernel       s = r - alpha v
//   spmv_t_kernel  t = A s, with the partial sums of (t, s), (t, t), (s, s)
//   update_kernel  u += alpha p + omega s, r = s - omega t, with (rh, r), (r, r)
// s gets a pass of its own so that A s gathers one vector per stored weight
// rather than forming s from two gathered ones (r and v).
// The scalars live in device memory: the block that finishes a kernel last
// (an atomic arrival count, no waiting) adds the blocks' partial sums in
// block order and computes the next coefficients and the stop flag, which
// every later kernel reads at entry. The host only looks at the flag once
// per chunk of kChunk iterations, which run as one CUDA graph on a
// non-default stream.
//
// Every sum has a fixed order, so results are reproducible and the CPU
// oracle follows them exactly: rows in fused multiply-adds from zero; a
// thread's rows (grid stride) in ascending order; a warp by an xor
// butterfly (16, 8, 4, 2, 1); a block by the butterfly over its warps'
// sums; the grid by thread t summing the partials of blocks t, t + 256, ...
// then the block butterfly. The grid is min(ceil(n / 256), 6 * SMs) blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "row_sum.cuh"
#include "runtime.h"
#include "stream_copy.cuh"

namespace rbfb {
namespace solve {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kChunk = 8;  // iterations between two looks at the stop flag
// Blocks per SM that stay resident together (at most 40 registers a
// thread); the grid is that many per SM, so none waits for a second wave.
constexpr int kBlocksPerSm = 6;
// The operator passes stage each warp's 32 rows (its entries in one piece,
// up to kStageEntries) in shared memory: 96 KB a block, two blocks per SM;
// the same grid then runs in three waves.
constexpr int kStageEntries = 1024;
constexpr int kStagedBlocksPerSm = 2;
constexpr size_t kStageBytes = static_cast<size_t>(kWarps) * kStageEntries * (sizeof(double) + sizeof(int));

enum : int { RUNNING = 0, CONVERGED = 1, MAXIT = 2, BREAKDOWN = 3, ZERO_RHS = 4, BAD_INPUT = 5 };

struct State {
    double rho, alpha, omega, beta;
    double ff, thresh2, rr;
    int iter, maxit, done, pending_breakdown;
    unsigned int arrive;  // blocks of the running kernel that have finished
    int bad_bnd;          // boundary indices outside [0, n)
};

struct Args {
    int n, k;
    bool vec;  // ja and values 16-byte aligned: vector loads in row_sum
    const int* ia;
    const int* ja;
    const double* values;
    const unsigned char* bflag;
    const double* f;
    double* u;
    double *r, *rh, *p, *v, *s, *t;
    double* part;  // 3 x gridDim.x partial sums
    State* st;
};

struct Workspace {
    size_t cap = 0;    // rows the vectors hold
    int grid_cap = 0;  // blocks the partial sums hold
    double* vec = nullptr;
    unsigned char* bflag = nullptr;
    double* part = nullptr;
    State* st = nullptr;
    State* st_h = nullptr;  // pinned copy of the state
    cudaGraphExec_t graph = nullptr;
    std::vector<unsigned char> key;
    long long graph_launches = 0;
};

// (A w)_s: row s of the operator applied to the vector w(j), j < n, summed
// in row order (row_sum); a boundary row is the identity.
template <class W>
__device__ __forceinline__ double apply_row(const Args& a, long long s, W w) {
    if (a.bflag[s]) return w(static_cast<int>(s));
    long long q, e;
    if (a.ia) {
        q = __ldg(a.ia + s);
        e = __ldg(a.ia + s + 1);
    } else {
        q = s * a.k;
        e = q + a.k;
    }
    return row_sum(a.ja, a.values, q, e, a.vec, w);
}

// Row sum over staged entries lo .. hi-1 of the warp's slab, in row order
// (the sums of row_sum), eight gathers of w in flight (sixteen measured
// slower).
template <class W>
__device__ __forceinline__ double row_sum_staged(const double* sval, const int* sja, int lo,
                                                 int hi, W w) {
    double acc = 0.0;
    int q = lo;
    for (; q + 8 <= hi; q += 8) {
        double v[8], x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = w(sja[q + i]);
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = sval[q + i];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc = fma(v[i], x[i], acc);
    }
    for (; q < hi; ++q) acc = fma(sval[q], w(sja[q]), acc);
    return acc;
}

// This thread's rows in ascending order (the grid-stride rows of apply_row's
// callers), each as f(s, (A w)_s). A warp takes its 32 consecutive rows at
// once: their entries (one contiguous piece of ja and values, from a 4-entry
// boundary) are copied into the warp's shared-memory slab with 16-byte
// copies under an L2 evict-first policy, and each lane sums its own row from
// there. A piece above kStageEntries (or unaligned arrays) is walked from
// global memory by row_sum. Same rows, same order, same sums as apply_row.
template <class W, class F>
__device__ __forceinline__ void walk_rows(const Args& a, unsigned char* smem, W w, F f) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* sval = reinterpret_cast<double*>(smem) + static_cast<size_t>(wid) * kStageEntries;
    int* sja = reinterpret_cast<int*>(reinterpret_cast<double*>(smem) +
                                      static_cast<size_t>(kWarps) * kStageEntries) +
               static_cast<size_t>(wid) * kStageEntries;
    const unsigned long long pol = evict_first_policy();
    const long long stride = static_cast<long long>(gridDim.x) * kThreads;
    for (long long t0 = static_cast<long long>(blockIdx.x) * kThreads + wid * 32; t0 < a.n;
         t0 += stride) {
        const long long s = t0 + lane;
        const long long s1 = min(t0 + 32, static_cast<long long>(a.n));
        long long q0, q1;
        if (a.ia) {
            q0 = __ldg(a.ia + t0);
            q1 = __ldg(a.ia + s1);
        } else {
            q0 = t0 * a.k;
            q1 = s1 * a.k;
        }
        const long long qa = q0 & ~3LL;
        const bool staged = a.vec && q1 - qa <= kStageEntries;
        if (staged) {
            const int m = static_cast<int>(q1 - qa);
            const double* gv = a.values + qa;
            const int* gj = a.ja + qa;
            for (int c = lane; c < m / 2; c += 32) cp_async_stream<16>(sval + 2 * c, gv + 2 * c, pol);
            if ((m & 1) && lane == 0) cp_async_stream<8>(sval + m - 1, gv + m - 1, pol);
            for (int c = lane; c < m / 4; c += 32) cp_async_stream<16>(sja + 4 * c, gj + 4 * c, pol);
            for (int e = (m & ~3) + lane; e < m; e += 32) cp_async_stream<4>(sja + e, gj + e, pol);
            cp_async_commit();
            cp_async_wait<0>();
            __syncwarp();
        }
        if (s < a.n) {
            double v;
            if (a.bflag[s]) {
                v = w(static_cast<int>(s));
            } else {
                long long q, e;
                if (a.ia) {
                    q = __ldg(a.ia + s);
                    e = __ldg(a.ia + s + 1);
                } else {
                    q = s * a.k;
                    e = q + a.k;
                }
                v = staged ? row_sum_staged(sval, sja, static_cast<int>(q - qa),
                                            static_cast<int>(e - qa), w)
                           : row_sum(a.ja, a.values, q, e, a.vec, w);
            }
            f(s, v);
        }
        __syncwarp();  // the slab is refilled for the next rows
    }
}

// Sums NV values over the block; the totals end up in every lane of warp 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sh)[NV]) {
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
        for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
#pragma unroll
        for (int i = 0; i < NV; ++i) sh[w][i] = v[i];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            v[i] = l < kWarps ? sh[l][i] : 0.0;
#pragma unroll
            for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
        }
    }
}

// Stores the block's partial sums and counts the block in. Returns true in
// every thread of the block that finished last; tot then holds the grid
// totals in thread 0 (all of warp 0). The other blocks return false.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], const Args& a, double (&tot)[NV]) {
    __shared__ double sh[kWarps][NV];
    __shared__ int last;
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) a.part[i * gridDim.x + blockIdx.x] = v[i];
        __threadfence();
        last = atomicAdd(&a.st->arrive, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double g[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) g[i] = 0.0;
    for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += kThreads)
#pragma unroll
        for (int i = 0; i < NV; ++i) g[i] += __ldcg(a.part + i * gridDim.x + b);
    block_sum<NV>(g, sh);
#pragma unroll
    for (int i = 0; i < NV; ++i) tot[i] = g[i];
    return true;
}

__device__ __forceinline__ bool is_fin(double x) { return isfinite(x); }

__global__ void flag_kernel(int n, int nb, const int* __restrict__ bnd, unsigned char* bflag,
                            State* st) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int i = bnd[b];
        if (i >= 0 && i < n)
            bflag[i] = 1;
        else
            atomicAdd(&st->bad_bnd, 1);
    }
}

// r = f - A u, rh = r, p = v = 0; rho = (r, r), ff = (f, f).
__global__ void __launch_bounds__(kThreads, kBlocksPerSm) init_kernel(Args a, double tol, int maxit) {
    double acc[2] = {0.0, 0.0};
    const long long stride = static_cast<long long>(gridDim.x) * kThreads;
    const double* u = a.u;
    for (long long s = static_cast<long long>(blockIdx.x) * kThreads + threadIdx.x; s < a.n;
         s += stride) {
        const double au = apply_row(a, s, [u](int j) { return u[j]; });
        const double fs = a.f[s];
        const double r = fs - au;
        a.r[s] = r;
        a.rh[s] = r;
        a.p[s] = 0.0;
        a.v[s] = 0.0;
        acc[0] = fma(r, r, acc[0]);
        acc[1] = fma(fs, fs, acc[1]);
    }
    double tot[2];
    if (!grid_sum<2>(acc, a, tot) || threadIdx.x != 0) return;
    State* st = a.st;
    st->rr = tot[0];
    st->ff = tot[1];
    st->rho = tot[0];
    st->alpha = 1.0;
    st->omega = 1.0;
    st->beta = 0.0;
    st->thresh2 = tol * tol * tot[1];
    st->iter = 0;
    st->maxit = maxit;
    st->pending_breakdown = 0;
    int done = RUNNING;
    if (st->bad_bnd)
        done = BAD_INPUT;  // nothing below may run on an out-of-range boundary list
    else if (!is_fin(tot[0]) || !is_fin(tot[1]))
        done = BREAKDOWN;
    else if (tot[0] <= st->thresh2)
        done = CONVERGED;
    else if (tot[1] == 0.0)
        done = ZERO_RHS;
    else if (maxit <= 0)
        done = MAXIT;
    st->done = done;
    st->arrive = 0;
}

__global__ void __launch_bounds__(kThreads, kBlocksPerSm) p_kernel(Args a) {
    const State* st = a.st;
    if (st->done) return;
    const double beta = st->beta, omega = st->omega;
    const long long stride = static_cast<long long>(gridDim.x) * kThreads;
    for (long long s = static_cast<long long>(blockIdx.x) * kThreads + threadIdx.x; s < a.n;
         s += stride)
        a.p[s] = fma(beta, fma(-omega, a.v[s], a.p[s]), a.r[s]);
}

__global__ void __launch_bounds__(kThreads, kStagedBlocksPerSm) spmv_v_kernel(Args a) {
    State* st = a.st;
    if (st->done) return;
    extern __shared__ __align__(16) unsigned char stage_smem[];
    double acc[1] = {0.0};
    const double* p = a.p;
    walk_rows(a, stage_smem, [p](int j) { return __ldg(p + j); }, [&](long long s, double v) {
        a.v[s] = v;
        acc[0] = fma(a.rh[s], v, acc[0]);
    });
    double tot[1];
    if (!grid_sum<1>(acc, a, tot) || threadIdx.x != 0) return;
    const double sigma = tot[0];
    if (sigma == 0.0 || !is_fin(sigma))
        st->done = BREAKDOWN;
    else
        st->alpha = st->rho / sigma;
    st->arrive = 0;
}

__global__ void __launch_bounds__(kThreads, kBlocksPerSm) s_kernel(Args a) {
    const State* st = a.st;
    if (st->done) return;
    const double alpha = st->alpha;
    const long long stride = static_cast<long long>(gridDim.x) * kThreads;
    for (long long i = static_cast<long long>(blockIdx.x) * kThreads + threadIdx.x; i < a.n;
         i += stride)
        a.s[i] = fma(-alpha, a.v[i], a.r[i]);
}

__global__ void __launch_bounds__(kThreads, kStagedBlocksPerSm) spmv_t_kernel(Args a) {
    State* st = a.st;
    if (st->done) return;
    extern __shared__ __align__(16) unsigned char stage_smem[];
    double acc[3] = {0.0, 0.0, 0.0};
    const double* sv = a.s;
    walk_rows(a, stage_smem, [sv](int j) { return __ldg(sv + j); }, [&](long long i, double ti) {
        const double si = sv[i];
        a.t[i] = ti;
        acc[0] = fma(ti, si, acc[0]);
        acc[1] = fma(ti, ti, acc[1]);
        acc[2] = fma(si, si, acc[2]);
    });
    double tot[3];
    if (!grid_sum<3>(acc, a, tot) || threadIdx.x != 0) return;
    if (tot[2] <= st->thresh2) {
        st->omega = 0.0;  // s is small enough: u += alpha p finishes the solve
    } else if (tot[1] == 0.0 || !is_fin(tot[1]) || !is_fin(tot[0])) {
        st->omega = 0.0;
        st->pending_breakdown = 1;
    } else {
        st->omega = tot[0] / tot[1];
    }
    st->arrive = 0;
}

__global__ void __launch_bounds__(kThreads, kBlocksPerSm) update_kernel(Args a) {
    State* st = a.st;
    if (st->done) return;
    const double alpha = st->alpha, omega = st->omega;
    double acc[2] = {0.0, 0.0};
    const long long stride = static_cast<long long>(gridDim.x) * kThreads;
    for (long long i = static_cast<long long>(blockIdx.x) * kThreads + threadIdx.x; i < a.n;
         i += stride) {
        const double si = a.s[i];
        a.u[i] = fma(omega, si, fma(alpha, a.p[i], a.u[i]));
        const double ri = fma(-omega, a.t[i], si);
        a.r[i] = ri;
        acc[0] = fma(a.rh[i], ri, acc[0]);
        acc[1] = fma(ri, ri, acc[1]);
    }
    double tot[2];
    if (!grid_sum<2>(acc, a, tot) || threadIdx.x != 0) return;
    const double rho_new = tot[0], rr = tot[1];
    st->iter += 1;
    st->rr = rr;
    int done = RUNNING;
    if (!is_fin(rr))
        done = BREAKDOWN;
    else if (rr <= st->thresh2)
        done = CONVERGED;
    else if (st->pending_breakdown || omega == 0.0)
        done = BREAKDOWN;
    else if (st->iter >= st->maxit)
        done = MAXIT;
    else if (rho_new == 0.0 || !is_fin(rho_new))
        done = BREAKDOWN;
    if (done == RUNNING) {
        st->beta = (rho_new / st->rho) * (alpha / omega);
        st->rho = rho_new;
    }
    st->done = done;
    st->arrive = 0;
}

int grid_of(const rbfb_ctx* ctx, int n) {
    const long long want = (static_cast<long long>(n) + kThreads - 1) / kThreads;
    return static_cast<int>(std::max(1LL, std::min(want, 1LL * kBlocksPerSm * ctx->sms)));
}

void release(Workspace* w) {
    if (!w) return;
    if (w->graph) cudaGraphExecDestroy(w->graph);
    if (w->vec) cudaFree(w->vec);
    if (w->bflag) cudaFree(w->bflag);
    if (w->part) cudaFree(w->part);
    if (w->st) cudaFree(w->st);
    if (w->st_h) cudaFreeHost(w->st_h);
    delete w;
}

int ensure(rbfb_ctx* ctx, int n, int grid) {
    auto* w = static_cast<Workspace*>(ctx->solve);
    if (!w) {
        w = new Workspace();
        ctx->solve = w;
        RBFB_CUDA(ctx, cudaMalloc(&w->st, sizeof(State)));
        RBFB_CUDA(ctx, cudaMallocHost(&w->st_h, sizeof(State)));
        // the operator passes' staging slabs (above the 48 KB default)
        RBFB_CUDA(ctx, cudaFuncSetAttribute(spmv_v_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kStageBytes)));
        RBFB_CUDA(ctx, cudaFuncSetAttribute(spmv_t_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kStageBytes)));
    }
    if (static_cast<size_t>(n) > w->cap) {
        if (w->graph) cudaGraphExecDestroy(w->graph);
        w->graph = nullptr;
        if (w->vec) cudaFree(w->vec);
        if (w->bflag) cudaFree(w->bflag);
        w->vec = nullptr;
        w->bflag = nullptr;
        w->cap = 0;
        if (cudaMalloc(&w->vec, 6 * sizeof(double) * n) != cudaSuccess ||
            cudaMalloc(&w->bflag, n) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, RBFB_ENOMEM, "solve workspace");
        }
        w->cap = n;
    }
    if (grid > w->grid_cap) {
        if (w->graph) cudaGraphExecDestroy(w->graph);
        w->graph = nullptr;
        if (w->part) cudaFree(w->part);
        w->part = nullptr;
        w->grid_cap = 0;
        if (cudaMalloc(&w->part, 3 * sizeof(double) * grid) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, RBFB_ENOMEM, "solve workspace");
        }
        w->grid_cap = grid;
    }
    return RBFB_OK;
}

// Enqueues kChunk iterations (5 launches each).
int enqueue_chunk(rbfb_ctx* ctx, const Args& a, int grid, cudaStream_t st) {
    for (int it = 0; it < kChunk; ++it) {
        p_kernel<<<grid, kThreads, 0, st>>>(a);
        spmv_v_kernel<<<grid, kThreads, kStageBytes, st>>>(a);
        s_kernel<<<grid, kThreads, 0, st>>>(a);
        spmv_t_kernel<<<grid, kThreads, kStageBytes, st>>>(a);
        update_kernel<<<grid, kThreads, 0, st>>>(a);
        ctx->launches += 5;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RBFB_OK : cuda_fail(ctx, e, "solve kernels");
}

}  // namespace solve
}  // namespace rbfb

extern "C" void rbfb_release_solve(rbfb_ctx* ctx) {
    rbfb::solve::release(static_cast<rbfb::solve::Workspace*>(ctx->solve));
    ctx->solve = nullptr;
}

extern "C" int rbfb_solve_bicgstab(rbfb_ctx* ctx, int n, int k, const int* ia, const int* ja,
                                   const double* values, const int* bnd, int nbnd, const double* f,
                                   double* u, double tol, int maxit, int* iters_h,
                                   double* relres_h, void* stream) {
    using namespace rbfb;
    using namespace rbfb::solve;
    if (iters_h) *iters_h = 0;
    if (relres_h) *relres_h = 0.0;
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n < 0 || nbnd < 0 || maxit < 0 || !(tol >= 0.0) || !std::isfinite(tol) || (!ia && k < 1))
        return fail(ctx, RBFB_EINVAL, "n >= 0, nbnd >= 0, maxit >= 0, finite tol >= 0 and k >= 1 "
                                      "(fixed width) required");
    if (n == 0) return RBFB_OK;
    if (!ja || !values || !f || !u || (nbnd > 0 && !bnd))
        return fail(ctx, RBFB_EINVAL, "null array argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    const int grid = grid_of(ctx, n);
    int rc = ensure(ctx, n, grid);
    if (rc) return rc;
    auto* w = static_cast<Workspace*>(ctx->solve);
    Args a{};
    a.n = n;
    a.k = k;
    a.ia = ia;
    a.ja = ja;
    a.values = values;
    a.vec = rows_vectorizable(ja, values);
    a.bflag = w->bflag;
    a.f = f;
    a.u = u;
    double* vec = w->vec;
    a.r = vec;
    a.rh = vec + static_cast<size_t>(n);
    a.p = vec + 2 * static_cast<size_t>(n);
    a.v = vec + 3 * static_cast<size_t>(n);
    a.s = vec + 4 * static_cast<size_t>(n);
    a.t = vec + 5 * static_cast<size_t>(n);
    a.part = w->part;
    a.st = w->st;

    RBFB_CUDA(ctx, cudaMemsetAsync(w->st, 0, sizeof(State), st));
    RBFB_CUDA(ctx, cudaMemsetAsync(w->bflag, 0, n, st));
    if (nbnd > 0) {
        const int fb = std::min((nbnd + kThreads - 1) / kThreads, 4 * ctx->sms);
        flag_kernel<<<fb, kThreads, 0, st>>>(n, nbnd, bnd, w->bflag, w->st);
        ++ctx->launches;
    }
    init_kernel<<<grid, kThreads, 0, st>>>(a, tol, maxit);
    ++ctx->launches;
    RBFB_CUDA(ctx, cudaGetLastError());

    // The chunk is a CUDA graph on a non-default stream (kernel arguments are
    // pointers and sizes, so one capture serves while they stay the same).
    std::vector<unsigned char> key(sizeof(Args) + sizeof(grid));
    std::memcpy(key.data(), &a, sizeof(Args));
    std::memcpy(key.data() + sizeof(Args), &grid, sizeof(grid));
    if (st != nullptr && (!w->graph || key != w->key)) {
        if (w->graph) cudaGraphExecDestroy(w->graph);
        w->graph = nullptr;
        const long long l0 = ctx->launches.load();
        RBFB_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_chunk(ctx, a, grid, st);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(st, &g);
        w->graph_launches = ctx->launches.load() - l0;
        ctx->launches -= w->graph_launches;  // counted when the graph runs
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ec != cudaSuccess) return cuda_fail(ctx, ec, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&w->graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            w->graph = nullptr;
            return cuda_fail(ctx, ei, "cudaGraphInstantiate");
        }
        w->key = key;
    }

    // Every chunk either advances the iteration count by kChunk or sets the
    // stop flag, so maxit / kChunk + 2 chunks always reach a stop.
    const long long max_chunks = static_cast<long long>(maxit) / kChunk + 2;
    State h{};
    for (long long c = 0; c < max_chunks; ++c) {
        if (st != nullptr) {
            RBFB_CUDA(ctx, cudaGraphLaunch(w->graph, st));
            ctx->launches += w->graph_launches;
        } else {
            rc = enqueue_chunk(ctx, a, grid, st);
            if (rc) return rc;
        }
        RBFB_CUDA(ctx, cudaMemcpyAsync(w->st_h, w->st, sizeof(State), cudaMemcpyDeviceToHost, st));
        RBFB_CUDA(ctx, cudaStreamSynchronize(st));
        h = *w->st_h;
        if (h.done != RUNNING) break;
    }
    if (h.done == BAD_INPUT || h.bad_bnd)
        return fail(ctx, RBFB_EINVAL, "boundary index outside [0, n)");
    if (iters_h) *iters_h = h.iter;
    if (h.done == ZERO_RHS) {
        RBFB_CUDA(ctx, cudaMemsetAsync(u, 0, sizeof(double) * n, st));
        RBFB_CUDA(ctx, cudaStreamSynchronize(st));
        return RBFB_OK;
    }
    if (relres_h) *relres_h = h.ff > 0.0 ? std::sqrt(h.rr / h.ff) : 0.0;
    switch (h.done) {
        case CONVERGED: return RBFB_OK;
        case MAXIT: return fail(ctx, RBFB_ENOCONV, "BiCGSTAB: maxit reached");
        case BREAKDOWN: return fail(ctx, RBFB_EBREAKDOWN, "BiCGSTAB: breakdown");
        default: return fail(ctx, RBFB_ETIMEOUT, "BiCGSTAB: no stop after maxit iterations");
    }
}
