// lbm.cu -- D2Q9 lattice Boltzmann kernels on sm_100a: equilibrium, moments,
// BGK collision, and semi-Lagrangian streaming through assembled RBF-FD
// interpolation operators, fused with the collision.
//
// Replaces feq_kernel, macros_kernel, bgk_kernel and bgk_kernel_split of
// src/lbm/d2q9_kernels.cu:13-150 (C++ twins of src/lbm/d2q9_kernels.cuf:
// 55-257). Same lattice (direction 0 at rest; 1-4 E, N, W, S; 5-8 NE, NW, SW,
// SE), same planar storage (direction a of node i at pdf[i + n*a]), same
// arithmetic: every product, sum and quotient of the reference's expressions
// in its order, each rounded once (no contraction into fused multiply-adds),
// for float and double. The results are bit-identical to the reference's
// kernels compiled without contraction and to the oracle's CPU restatement.
//
// Streaming is what the reference's assembly exists for (semi-Lagrangian
// streaming with interpolation operators, src/rbf_operators.h:292-298) but
// does not ship: population a of node s after streaming is the interpolation
// of the post-collision field f_a at the departure point x_s - c_a dt,
// sum_j W_a[s*k + j] * f_a[ja[s*k + j]], with W_a the weights of the
// interpolation right-hand side at that point (rbfb_assemble with
// RBFB_OP_INTERP and the 8 departure points). The sum runs in entry order,
// j = 0 first: the first product rounded, then one fused multiply-add an
// entry, as a CSR row product does. A warp stages 32 nodes' rows in shared
// memory and each lane sums its own node's row; the oracle restates that
// order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "rbf_b200.h"
#include "stream_copy.cuh"

namespace rbfb {
namespace lbm {

// Arithmetic rounded once per operation, per type.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double quo(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float quo(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// D2Q9 constants in the working precision, formed as the reference forms
// them (src/lbm/d2q9_kernels.h:16-31): a quotient of two small integers, and
// 3 times a weight, each rounded in T.
template <typename T>
struct Lattice {
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

// Density and velocity of populations f[0..8].
template <typename T>
__device__ __forceinline__ void moments(const T (&f)[9], T& rho, T& ux, T& uy) {
    rho = add(add(add(add(f[5], f[7]), add(f[6], f[8])), add(add(f[1], f[3]), add(f[2], f[4]))),
              f[0]);
    const T invrho = quo(T(1), rho);
    ux = mul(invrho, add(add(sub(f[5], f[7]), sub(f[8], f[6])), sub(f[1], f[3])));
    uy = mul(invrho, add(add(sub(f[5], f[7]), sub(f[6], f[8])), sub(f[2], f[4])));
}

// The direction-independent part of the equilibrium, 1/3 - u.u/2.
template <typename T>
__device__ __forceinline__ T indp_of(T uxsq, T uysq) {
    using L = Lattice<T>;
    return sub(L::one_third, mul(L::one_half, add(uxsq, uysq)));
}

// The equilibrium terms: e[a] = 3 w_a rho (indp + c_a.u + 3/2 (c_a.u)^2)
// without the factor 3 w_a rho, as pairs of opposite directions share them.
template <typename T>
struct EqTerms {
    T t13p, t13m, t24p, t24m, t57p, t57m, t68m, t68p;
};
template <typename T>
__device__ __forceinline__ EqTerms<T> eq_terms(T ux, T uy, T uxsq, T uysq, T indp) {
    using L = Lattice<T>;
    EqTerms<T> e;
    const T v13 = add(indp, mul(L::three_halves, uxsq));
    e.t13p = add(v13, ux);
    e.t13m = sub(v13, ux);
    const T v24 = add(indp, mul(L::three_halves, uysq));
    e.t24p = add(v24, uy);
    e.t24m = sub(v24, uy);
    const T xpy = add(ux, uy);
    const T v57 = add(indp, mul(mul(L::three_halves, xpy), xpy));
    e.t57p = add(v57, xpy);
    e.t57m = sub(v57, xpy);
    const T xmy = sub(ux, uy);
    const T v68 = add(indp, mul(mul(L::three_halves, xmy), xmy));
    e.t68m = sub(v68, xmy);
    e.t68p = add(v68, xmy);
    return e;
}

// BGK relaxation of f towards the equilibrium of its own moments: out[a] =
// (1 - omega) f[a] + omega 3 w_a rho (...), the reference's bgk_kernel body.
template <typename T>
__device__ __forceinline__ void collide(const T (&f)[9], T omega, T (&out)[9], T& rho, T& ux,
                                        T& uy, T& indp) {
    using L = Lattice<T>;
    const T omegabar = sub(T(1), omega);
    const T ow0 = mul(omega, L::three_w0);
    const T ows = mul(omega, L::three_ws);
    const T owd = mul(omega, L::three_wd);
    moments(f, rho, ux, uy);
    const T uxsq = mul(ux, ux);
    const T uysq = mul(uy, uy);
    indp = indp_of(uxsq, uysq);
    const EqTerms<T> e = eq_terms(ux, uy, uxsq, uysq, indp);
    out[0] = add(mul(omegabar, f[0]), mul(mul(ow0, rho), indp));
    out[1] = add(mul(omegabar, f[1]), mul(mul(ows, rho), e.t13p));
    out[3] = add(mul(omegabar, f[3]), mul(mul(ows, rho), e.t13m));
    out[2] = add(mul(omegabar, f[2]), mul(mul(ows, rho), e.t24p));
    out[4] = add(mul(omegabar, f[4]), mul(mul(ows, rho), e.t24m));
    out[5] = add(mul(omegabar, f[5]), mul(mul(owd, rho), e.t57p));
    out[7] = add(mul(omegabar, f[7]), mul(mul(owd, rho), e.t57m));
    out[6] = add(mul(omegabar, f[6]), mul(mul(owd, rho), e.t68m));
    out[8] = add(mul(omegabar, f[8]), mul(mul(owd, rho), e.t68p));
}

template <typename T>
__global__ void feq_kernel(int n, const T* __restrict__ rho, const T* __restrict__ ux,
                           const T* __restrict__ uy, T* __restrict__ pdf) {
    using L = Lattice<T>;
    const size_t N = static_cast<size_t>(n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T r = rho[i], u = ux[i], v = uy[i];
        const T uxsq = mul(u, u), uysq = mul(v, v);
        const T indp = indp_of(uxsq, uysq);
        const EqTerms<T> e = eq_terms(u, v, uxsq, uysq, indp);
        pdf[i] = mul(mul(L::three_w0, r), indp);
        pdf[i + N * 1] = mul(mul(L::three_ws, r), e.t13p);
        pdf[i + N * 3] = mul(mul(L::three_ws, r), e.t13m);
        pdf[i + N * 2] = mul(mul(L::three_ws, r), e.t24p);
        pdf[i + N * 4] = mul(mul(L::three_ws, r), e.t24m);
        pdf[i + N * 5] = mul(mul(L::three_wd, r), e.t57p);
        pdf[i + N * 7] = mul(mul(L::three_wd, r), e.t57m);
        pdf[i + N * 6] = mul(mul(L::three_wd, r), e.t68m);
        pdf[i + N * 8] = mul(mul(L::three_wd, r), e.t68p);
    }
}

template <typename T>
__global__ void macros_kernel(int n, const T* __restrict__ pdf, T* __restrict__ rho,
                              T* __restrict__ ux, T* __restrict__ uy) {
    const size_t N = static_cast<size_t>(n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T f[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) f[a] = pdf[i + N * a];
        T r, u, v;
        moments(f, r, u, v);
        rho[i] = r;
        ux[i] = u;
        uy[i] = v;
    }
}

// bgk_kernel (indp == nullptr) and bgk_kernel_split: collision in place.
template <typename T>
__global__ void bgk_kernel(int n, T omega, T* __restrict__ pdf, T* __restrict__ rho,
                           T* __restrict__ ux, T* __restrict__ uy, T* __restrict__ indp) {
    const size_t N = static_cast<size_t>(n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T f[9], o[9], r, u, v, d;
#pragma unroll
        for (int a = 0; a < 9; ++a) f[a] = pdf[i + N * a];
        collide(f, omega, o, r, u, v, d);
        rho[i] = r;
        ux[i] = u;
        uy[i] = v;
        if (indp) indp[i] = d;
#pragma unroll
        for (int a = 0; a < 9; ++a) pdf[i + N * a] = o[a];
    }
}

constexpr int kTileWarps = 4;  // warps a CTA; each warp owns a 32-node tile at a time

// Shared memory of one warp: DEPTH weight slabs (the directions in flight)
// and the tile's index slab, 32 rows of ks entries each; ks = k for odd k,
// k + 1 for even k, so that row r of lane r is bank-conflict free.
inline int tile_stride(int k) { return (k & 1) ? k : k + 1; }
inline size_t tile_smem_bytes(int k, int depth, bool jreg) {
    return static_cast<size_t>(kTileWarps) * 32 * tile_stride(k) *
           (depth * sizeof(double) + (jreg ? 0 : sizeof(int)));
}

// Copies the tile's m = cnt * k consecutive entries (element e to row e / k,
// column e % k of a ks-strided slab); lane takes e = lane + 32 i. (r, c) is
// the row and column of the lane's current element, advanced by 32 entries.
// VEC (unpadded slabs, 16-byte aligned source and destination): 16-byte
// copies, the odd tail entries one by one.
template <bool PAD, bool VEC, typename V>
__device__ __forceinline__ void copy_slab(V* dst, const V* src, int m, int k, int ks, int lane,
                                          int r, int c, int q32, int r32,
                                          unsigned long long pol) {
    if constexpr (VEC && !PAD) {
        constexpr int per = 16 / sizeof(V);
        const int chunks = m / per;
        for (int q = lane; q < chunks; q += 32)
            cp_async_stream<16>(dst + q * per, src + q * per, pol);
        for (int e = chunks * per + lane; e < m; e += 32)
            cp_async_stream<sizeof(V)>(dst + e, src + e, pol);
    } else {
        for (int e = lane; e < m; e += 32) {
            cp_async_stream<sizeof(V)>(dst + (PAD ? r * ks + c : e), src + e, pol);
            if (PAD) {
                r += q32;
                c += r32;
                if (c >= k) {
                    c -= k;
                    ++r;
                }
            }
        }
    }
}

// Semi-Lagrangian streaming of the post-collision field pdf_in through the
// interpolation operators W (8 arrays of n*k weights, direction a at
// W + (a-1)*n*k, rows like ja), then the BGK collision, into pdf_out. The
// moments of the streamed populations go to rho, ux, uy (any may be null).
// A warp takes a tile of 32 consecutive nodes: it copies the tile's index
// rows and the first DEPTH - 1 directions' weight rows into shared memory;
// for each direction it starts the copy of the direction DEPTH - 1 ahead and
// has each lane sum its own node's row in entry order (the first product
// rounded, then one fused multiply-add an entry), gathering pdf_in through
// the indices. Then every lane collides its node and the warp writes 32
// consecutive entries of each direction, as streaming stores. KT > 0 fixes
// k at compile time (the row's gathers all in flight at once). JREG (with
// KT): the index rows land in the second weight buffer and each lane keeps
// its own row in registers for the tile, so no index slab is kept.
template <typename T, bool PAD, int KT, int DEPTH, bool VEC, bool JREG = false>
__global__ void __launch_bounds__(kTileWarps * 32) stream_collide_kernel(
    int n, int k, const int* __restrict__ ja, const double* __restrict__ W, T omega,
    const T* __restrict__ pdf_in, T* __restrict__ pdf_out, T* __restrict__ rho,
    T* __restrict__ ux, T* __restrict__ uy) {
    static_assert(DEPTH >= 2 && DEPTH <= 4, "prefetch depth");
    static_assert(!JREG || (KT > 0 && !PAD && DEPTH == 2), "index rows in registers");
    extern __shared__ __align__(16) unsigned char tile_smem[];
    if (KT > 0) k = KT;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ks = PAD ? k + 1 : k;
    const int slab = 32 * ks;
    double* wbuf =
        reinterpret_cast<double*>(tile_smem) + static_cast<size_t>(wid) * DEPTH * slab;
    int* jbuf = JREG ? reinterpret_cast<int*>(wbuf + slab)
                     : reinterpret_cast<int*>(reinterpret_cast<double*>(tile_smem) +
                                              static_cast<size_t>(kTileWarps) * DEPTH * slab) +
                           static_cast<size_t>(wid) * slab;
    const size_t N = static_cast<size_t>(n);
    const size_t nnz = N * static_cast<size_t>(k);
    const unsigned long long pol = evict_first_policy();
    const int r0 = lane / k, c0 = lane - r0 * k, q32 = 32 / k, r32 = 32 - q32 * k;
    const int tiles = (n + 31) >> 5;
    for (int tile = blockIdx.x * kTileWarps + wid; tile < tiles; tile += gridDim.x * kTileWarps) {
        const int s0 = tile << 5;
        const int cnt = min(32, n - s0);
        const int m = cnt * k;
        const size_t base = static_cast<size_t>(s0) * k;
        copy_slab<PAD, VEC>(jbuf, ja + base, m, k, ks, lane, r0, c0, q32, r32, pol);
#pragma unroll
        for (int d = 1; d < DEPTH; ++d) {
            copy_slab<PAD, VEC>(wbuf + (d - 1) * slab, W + static_cast<size_t>(d - 1) * nnz + base,
                                m, k, ks, lane, r0, c0, q32, r32, pol);
            cp_async_commit();
        }
        int jrow[JREG ? KT : 1];
        if constexpr (JREG) {  // the lane's index row, then the buffer is free
            cp_async_wait<0>();
            __syncwarp();
            if (lane < cnt)
#pragma unroll
                for (int j = 0; j < KT; ++j) jrow[j] = jbuf[lane * ks + j];
            __syncwarp();
        }
        T f[9];
#pragma unroll
        for (int a = 1; a < 9; ++a) {
            const int nxt = a + DEPTH - 1;  // the direction whose copy starts now
            if (nxt <= 8) {
                copy_slab<PAD, VEC>(wbuf + ((nxt - 1) % DEPTH) * slab,
                                    W + static_cast<size_t>(nxt - 1) * nnz + base, m, k, ks, lane,
                                    r0, c0, q32, r32, pol);
                cp_async_commit();
            }
            cp_async_wait_pending(min(DEPTH - 1, 8 - a));
            __syncwarp();
            if (lane < cnt) {
                const double* wr = wbuf + ((a - 1) % DEPTH) * slab + lane * ks;
                const int* jr = jbuf + lane * ks;
                const T* pa = pdf_in + N * a;
                T v;
                if constexpr (JREG) {
                    v = mul(static_cast<T>(wr[0]), pa[jrow[0]]);
#pragma unroll
                    for (int j = 1; j < KT; ++j) v = fmaT(static_cast<T>(wr[j]), pa[jrow[j]], v);
                } else if constexpr (KT > 0) {
                    v = mul(static_cast<T>(wr[0]), pa[jr[0]]);
#pragma unroll
                    for (int j = 1; j < KT; ++j) v = fmaT(static_cast<T>(wr[j]), pa[jr[j]], v);
                } else {
                    v = mul(static_cast<T>(wr[0]), pa[jr[0]]);
#pragma unroll 8
                    for (int j = 1; j < k; ++j) v = fmaT(static_cast<T>(wr[j]), pa[jr[j]], v);
                }
                f[a] = v;
            }
            __syncwarp();  // every lane is done with this buffer before it is refilled
        }
        const int s = s0 + lane;
        if (lane < cnt) {
            f[0] = pdf_in[s];  // the rest population does not move
            T o[9], r, u, v, d;
            collide(f, omega, o, r, u, v, d);
#pragma unroll
            for (int a = 0; a < 9; ++a) __stcs(pdf_out + s + N * a, o[a]);
            if (rho) __stcs(rho + s, r);
            if (ux) __stcs(ux + s, u);
            if (uy) __stcs(uy + s, v);
        }
    }
}

template <typename T, bool PAD, int KT, int DEPTH, bool VEC, bool JREG = false>
int launch_stream_collide(int n, int k, const int* ja, const double* W, T omega, const T* pin,
                          T* pout, T* rho, T* ux, T* uy, cudaStream_t st) {
    auto kern = stream_collide_kernel<T, PAD, KT, DEPTH, VEC, JREG>;
    const size_t smem = tile_smem_bytes(k, DEPTH, JREG);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
        return RBFB_ECUDA;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileWarps * 32, smem) !=
            cudaSuccess ||
        per_sm < 1)
        return RBFB_ECUDA;
    const int tiles = (n + 31) / 32;
    const int blocks = std::max(1, std::min((tiles + kTileWarps - 1) / kTileWarps,
                                            std::max(sms, 1) * per_sm));
    kern<<<blocks, kTileWarps * 32, smem, st>>>(n, k, ja, W, omega, pin, pout, rho, ux, uy);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

template <typename T>
int stream_collide(int n, int k, const int* ja, const double* W, T omega, const T* pin, T* pout,
                   T* rho, T* ux, T* uy, cudaStream_t st) {
    // 16-byte copies need 16-byte aligned rows: ja, W and every direction's
    // array (n*k even). Odd k: unpadded slabs; k = 21 (the D2Q9 operators'
    // usual stencil) fixed at compile time, with the index rows held in
    // registers. Even k: padded slabs, 8-byte copies.
    const bool vec = ((reinterpret_cast<uintptr_t>(ja) | reinterpret_cast<uintptr_t>(W)) & 15) == 0 &&
                     ((static_cast<long long>(n) * k) & 1) == 0;
    if (!(k & 1))
        return launch_stream_collide<T, true, 0, 2, false>(n, k, ja, W, omega, pin, pout, rho, ux,
                                                           uy, st);
    if (vec && k == 21)  // index rows in registers: no index slab, 20 warps per SM
        return launch_stream_collide<T, false, 21, 2, true, true>(n, k, ja, W, omega, pin, pout,
                                                                  rho, ux, uy, st);
    if (vec)
        return launch_stream_collide<T, false, 0, 2, true>(n, k, ja, W, omega, pin, pout, rho, ux,
                                                           uy, st);
    return launch_stream_collide<T, false, 0, 2, false>(n, k, ja, W, omega, pin, pout, rho, ux,
                                                        uy, st);
}

int blocks_for(int n) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min((n + 255) / 256, std::max(sms, 1) * 16));
}

}  // namespace lbm
}  // namespace rbfb

using namespace rbfb::lbm;

extern "C" {

int rbfb_lbm_feq(int n, int precision, const void* rho, const void* ux, const void* uy, void* pdf,
                 void* stream) {
    if (n < 0 || !rho || !ux || !uy || !pdf) return RBFB_EINVAL;
    if (n == 0) return RBFB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == RBFB_FP64)
        feq_kernel<double><<<blocks_for(n), 256, 0, st>>>(
            n, static_cast<const double*>(rho), static_cast<const double*>(ux),
            static_cast<const double*>(uy), static_cast<double*>(pdf));
    else if (precision == RBFB_LBM_FP32)
        feq_kernel<float><<<blocks_for(n), 256, 0, st>>>(
            n, static_cast<const float*>(rho), static_cast<const float*>(ux),
            static_cast<const float*>(uy), static_cast<float*>(pdf));
    else
        return RBFB_EINVAL;
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_lbm_macros(int n, int precision, const void* pdf, void* rho, void* ux, void* uy,
                    void* stream) {
    if (n < 0 || !rho || !ux || !uy || !pdf) return RBFB_EINVAL;
    if (n == 0) return RBFB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == RBFB_FP64)
        macros_kernel<double><<<blocks_for(n), 256, 0, st>>>(
            n, static_cast<const double*>(pdf), static_cast<double*>(rho),
            static_cast<double*>(ux), static_cast<double*>(uy));
    else if (precision == RBFB_LBM_FP32)
        macros_kernel<float><<<blocks_for(n), 256, 0, st>>>(
            n, static_cast<const float*>(pdf), static_cast<float*>(rho), static_cast<float*>(ux),
            static_cast<float*>(uy));
    else
        return RBFB_EINVAL;
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_lbm_bgk(int n, int precision, double omega, void* pdf, void* rho, void* ux, void* uy,
                 void* indp, void* stream) {
    if (n < 0 || !rho || !ux || !uy || !pdf) return RBFB_EINVAL;
    if (n == 0) return RBFB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == RBFB_FP64)
        bgk_kernel<double><<<blocks_for(n), 256, 0, st>>>(
            n, omega, static_cast<double*>(pdf), static_cast<double*>(rho),
            static_cast<double*>(ux), static_cast<double*>(uy), static_cast<double*>(indp));
    else if (precision == RBFB_LBM_FP32)
        bgk_kernel<float><<<blocks_for(n), 256, 0, st>>>(
            n, static_cast<float>(omega), static_cast<float*>(pdf), static_cast<float*>(rho),
            static_cast<float*>(ux), static_cast<float*>(uy), static_cast<float*>(indp));
    else
        return RBFB_EINVAL;
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_lbm_stream_collide(int n, int precision, int k, const int* ja, const double* W,
                            double omega, const void* pdf_in, void* pdf_out, void* rho, void* ux,
                            void* uy, void* stream) {
    if (n < 0 || k < 1 || k > 64 || !ja || !W || !pdf_in || !pdf_out || pdf_in == pdf_out)
        return RBFB_EINVAL;
    if (n == 0) return RBFB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == RBFB_FP64)
        return stream_collide<double>(n, k, ja, W, omega, static_cast<const double*>(pdf_in),
                                      static_cast<double*>(pdf_out), static_cast<double*>(rho),
                                      static_cast<double*>(ux), static_cast<double*>(uy), st);
    if (precision == RBFB_LBM_FP32)
        return stream_collide<float>(n, k, ja, W, static_cast<float>(omega),
                                     static_cast<const float*>(pdf_in),
                                     static_cast<float*>(pdf_out), static_cast<float*>(rho),
                                     static_cast<float*>(ux), static_cast<float*>(uy), st);
    return RBFB_EINVAL;
}

}  // extern "C"
