// reorder.cu -- node renumbering on the device: space-filling-curve keys and
// orders, the boundary-last partition, and the renumbering of stencil graphs.
//
// Replaces the host-side locality tools of the reference:
//   rbf_morton_keys / rbf_hilbert_keys, zidx / hidx   src/rbf_ordering.F90:31-63,82-218
//   morton_order / hilbert_order (stable key sort)    src/rbf_reorder.h:210-230,180-185
//   boundary_last_by_flag (stable partition)          src/rbf_reorder.h:232-244
//   renumber_stencils / renumber_csr                  src/rbf_reorder.h:256-303
//   Permutation::permute (gather form)                src/rbf_reorder.h:68-80
// A renumbering that follows a space-filling curve makes the stencil
// gather of the assembly (and the cell walk of the k-NN search) local.
//
// Keys restate the Fortran arithmetic with every operation rounded on its
// own (the midpoint cx = x0 + 0.5 * (x1 - x0) is not fused). The sort is an
// LSD radix sort, 8-bit digits over the 2 * ndiv key bits, every pass
// stable, so equal keys keep the nodes' order -- std::stable_sort's result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <utility>

#include "asm_math.cuh"
#include "runtime.h"

namespace rbfb {
namespace reorder {

constexpr int kTpb = 256;             // threads per sort block
constexpr int kItems = 8;             // elements per thread per tile
constexpr int kTile = kTpb * kItems;  // elements per sort tile
constexpr int kScan = 1024;           // elements per scan block

// ---- bounding box (compute_bbox, src/rbf_reorder.h:60-66) ------------------------
// Doubles are ordered by their bit pattern once the sign is folded in:
// non-negative values keep theirs with the top bit set, negative ones are
// inverted. atomicMin / atomicMax on that image give exact minima / maxima.
__device__ __forceinline__ unsigned long long ord(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}
__global__ void bbox_init_kernel(unsigned long long* bb) {
    bb[0] = ~0ull;  // min x
    bb[1] = ~0ull;  // min y
    bb[2] = 0ull;   // max x
    bb[3] = 0ull;   // max y
}
__global__ void bbox_kernel(const double* x, const double* y, int n, unsigned long long* bb) {
    unsigned long long mnx = ~0ull, mny = ~0ull, mxx = 0ull, mxy = 0ull;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long ox = ord(x[i]), oy = ord(y[i]);
        mnx = min(mnx, ox);
        mny = min(mny, oy);
        mxx = max(mxx, ox);
        mxy = max(mxy, oy);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(bb + 0, mnx);
        atomicMin(bb + 1, mny);
        atomicMax(bb + 2, mxx);
        atomicMax(bb + 3, mxy);
    }
}
// bbox as doubles {xmin, ymin, xmax, ymax}, the layout of rbf::BBox2<double>
__global__ void bbox_final_kernel(const unsigned long long* bb, double* box) {
    box[0] = unord(bb[0]);
    box[1] = unord(bb[1]);
    box[2] = unord(bb[2]);
    box[3] = unord(bb[3]);
}

// ---- curve keys (zidx / hidx, src/rbf_ordering.F90:82-218) ------------------------
// Hilbert state tables of hidx: the key digit and the next rotation for
// quadrant q in rotation state rot, indexed [rot][q] (the Fortran arrays
// table(q, rot) and tr(q, rot), stored column-major).
__constant__ int c_hdigit[4][4] = {{0, 3, 1, 2}, {2, 3, 1, 0}, {2, 1, 3, 0}, {0, 1, 3, 2}};
__constant__ int c_hnext[4][4] = {{3, 1, 0, 0}, {1, 0, 1, 2}, {2, 2, 3, 1}, {0, 3, 2, 3}};

__global__ void keys_kernel(const double* x, const double* y, int n, const double* box, int ndiv,
                            int curve, unsigned long long* keys, int* vals) {
    const double bx0 = box[0], by0 = box[1], bx1 = box[2], by1 = box[3];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double px = x[i], py = y[i];
        double x0 = bx0, y0 = by0, x1 = bx1, y1 = by1;
        unsigned long long z = 0;
        int rot = 0;
        for (int l = 0; l < ndiv; ++l) {
            z <<= 2;
            const double cx = dadd(x0, dmul(0.5, dsub(x1, x0)));
            const double cy = dadd(y0, dmul(0.5, dsub(y1, y0)));
            const int q = (px > cx ? 1 : 0) + (py > cy ? 2 : 0);
            if (curve == 0) {
                z += q;  // Morton: 2 | 3 over 0 | 1
            } else {
                z += c_hdigit[rot][q];
                rot = c_hnext[rot][q];
            }
            if (px > cx) x0 = cx; else x1 = cx;
            if (py > cy) y0 = cy; else y1 = cy;
        }
        keys[i] = z;
        vals[i] = i;
    }
}

// ---- device-wide exclusive scan of int (three kernels) ----------------------------
__global__ void scan_block_kernel(const int* in, int* out, int n, int* sums) {
    __shared__ int ws[32];
    const int i = blockIdx.x * kScan + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int s = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += t;
    }
    if (lane == 31) ws[w] = s;
    __syncthreads();
    if (w == 0) {
        int t = ws[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        ws[lane] = t;
    }
    __syncthreads();
    const int excl = s - v + (w > 0 ? ws[w - 1] : 0);
    if (i < n) out[i] = excl;
    if (threadIdx.x == kScan - 1) sums[blockIdx.x] = excl + v;
}
// one block: exclusive scan of the nb block sums in chunks of 1024, carrying
// the running total; total[0] = the grand total
__global__ void scan_sums_kernel(int* sums, int nb, int* total) {
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += kScan) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        int s = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        if (lane == 31) ws[w] = s;
        __syncthreads();
        if (w == 0) {
            int t = ws[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += u;
            }
            ws[lane] = t;
        }
        __syncthreads();
        const int c = carry;
        if (i < nb) sums[i] = c + s - v + (w > 0 ? ws[w - 1] : 0);
        __syncthreads();
        if (threadIdx.x == kScan - 1) carry = c + s + (w > 0 ? ws[w - 1] : 0);
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}
__global__ void scan_add_kernel(int* out, int n, const int* sums) {
    const int i = blockIdx.x * kScan + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

// ---- stable LSD radix sort of (key, value) pairs ----------------------------------
__global__ void digit_hist_kernel(const unsigned long long* keys, int n, int shift, int nblocks,
                                  int* hist) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const int i = base + r * kTpb + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];  // digit-major
}

// Each tile scatters its elements in element order: round r handles
// elements r * 256 + t, and within a round an element's place among the
// equal digits before it is (earlier warps' counts) + (earlier lanes in its
// warp with the same digit, from __match_any_sync).
__global__ void digit_scatter_kernel(const unsigned long long* keys, const int* vals, int n,
                                     int shift, int nblocks, const int* off,
                                     unsigned long long* keys_out, int* vals_out) {
    constexpr int W = kTpb / 32;
    __shared__ int run[256];       // elements of each digit placed by earlier rounds
    __shared__ int wc[W][256];     // this round: count of each digit per warp
    __shared__ int base_of[256];   // the tile's first output position per digit
    base_of[threadIdx.x] = off[threadIdx.x * nblocks + blockIdx.x];
    run[threadIdx.x] = 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int tile = blockIdx.x * kTile;
    for (int r = 0; r < kItems; ++r) {
#pragma unroll
        for (int u = 0; u < W; ++u) wc[u][threadIdx.x] = 0;
        __syncthreads();
        const int i = tile + r * kTpb + threadIdx.x;
        const bool ok = i < n;
        unsigned long long key = 0;
        int val = 0;
        int dg = 256;  // out of range: a digit of its own, never written
        if (ok) {
            key = keys[i];
            val = vals[i];
            dg = (int)((key >> shift) & 255u);
        }
        const unsigned same = __match_any_sync(0xffffffffu, dg);
        const int rank = __popc(same & lt);
        if (ok && rank == 0) wc[w][dg] = __popc(same);
        __syncthreads();
        if (ok) {
            int before = 0;
            for (int u = 0; u < w; ++u) before += wc[u][dg];
            const int dst = base_of[dg] + run[dg] + before + rank;
            keys_out[dst] = key;
            vals_out[dst] = val;
        }
        __syncthreads();
        int tot = 0;
#pragma unroll
        for (int u = 0; u < W; ++u) tot += wc[u][threadIdx.x];
        run[threadIdx.x] += tot;
        __syncthreads();
    }
}

__global__ void inverse_kernel(const int* perm, int n, int* inv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        inv[perm[i]] = i;
}

// ---- boundary last (stable partition) --------------------------------------------
__global__ void flag_kernel(const int* flag, int n, int* b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        b[i] = flag[i] != 0;
}
// excl_b[i] = boundary nodes before i; interior nodes go to i - excl_b[i],
// boundary nodes to (n - nbnd) + excl_b[i]
__global__ void partition_kernel(const int* flag, const int* excl_b, int n, const int* nbnd,
                                 int* perm, int* inv) {
    const int nint = n - *nbnd;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int pos = flag[i] != 0 ? nint + excl_b[i] : i - excl_b[i];
        perm[pos] = i;
        if (inv) inv[i] = pos;
    }
}

// ---- renumbering of stencil graphs and node data ---------------------------------
__global__ void renumber_fixed_kernel(int n, int k, const int* ja, const int* perm, const int* inv,
                                      int* out) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long s = t / k, j = t - s * k;
        out[t] = inv[ja[(long long)perm[s] * k + j]];
    }
}
__global__ void row_len_kernel(int n, const int* ia, const int* perm, int* len) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        len[i] = ia[perm[i] + 1] - ia[perm[i]];
}
__global__ void renumber_csr_kernel(int n, const int* ia, const int* ja, const int* perm,
                                    const int* inv, const int* ia_out, int* ja_out) {
    // one warp per row, lanes over the row's entries (coalesced)
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const int a = ia[perm[i]], len = ia[perm[i] + 1] - a, d = ia_out[i];
        for (int j = lane; j < len; j += 32) ja_out[d + j] = inv[ja[a + j]];
    }
}
template <typename E>
__global__ void gather_kernel(int n, const int* perm, const E* in, E* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = in[perm[i]];
}

int grid_of(rbfb_ctx* ctx, long long work, int tpb) {
    const long long b = (work + tpb - 1) / tpb;
    return (int)std::max(1ll, std::min(b, (long long)ctx->sms * 16));
}

// exclusive scan of n ints (in -> out, may alias); tmp: >= n / kScan + 1 ints
// total (device, may be null) receives the sum
int scan(rbfb_ctx* ctx, const int* in, int* out, int n, int* tmp, int* total, cudaStream_t st) {
    const int nb = (n + kScan - 1) / kScan;
    scan_block_kernel<<<nb, kScan, 0, st>>>(in, out, n, tmp);
    scan_sums_kernel<<<1, kScan, 0, st>>>(tmp, nb, total);
    scan_add_kernel<<<nb, kScan, 0, st>>>(out, n, tmp);
    ctx->launches += 3;
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

// Scratch of one call, from the stream-ordered pool (freed on the stream).
struct Scratch {
    cudaStream_t st;
    void* p = nullptr;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch() {
        if (p) cudaFreeAsync(p, st);
    }
};
size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace reorder
}  // namespace rbfb

using namespace rbfb;
using namespace rbfb::reorder;

extern "C" {

int rbfb_curve_order(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* bbox_h,
                     int ndiv, int curve, int64_t* keys_out, int* perm, int* inv, void* stream);

int rbfb_curve_keys(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* bbox_h,
                    int ndiv, int curve, int64_t* keys, void* stream) {
    return rbfb_curve_order(ctx, n, x, y, bbox_h, ndiv, curve, keys, nullptr, nullptr, stream);
}

int rbfb_curve_order(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* bbox_h,
                     int ndiv, int curve, int64_t* keys_out, int* perm, int* inv, void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (ndiv < 1 || ndiv > 31) return fail(ctx, RBFB_EINVAL, "ndiv must be between 1 and 31");
    if (curve != 0 && curve != 1) return fail(ctx, RBFB_EINVAL, "curve: 0 (Morton) or 1 (Hilbert)");
    if (n < 0) return fail(ctx, RBFB_EINVAL, "negative size");
    if (n == 0) return RBFB_OK;  // nothing to order: pointers may be null
    if (!x || !y || (!keys_out && !perm)) return fail(ctx, RBFB_EINVAL, "null pointer argument");
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool sort = perm != nullptr;
    const int nblocks = (n + kTile - 1) / kTile;
    const size_t nh = (size_t)256 * nblocks;
    // scratch: box (4 doubles) + bb (4 u64) + keys/vals x2 + hist + scan sums + total
    const size_t o_box = 0, o_bb = 64, o_k0 = 128;
    const size_t o_v0 = o_k0 + al256(8ull * n);
    const size_t o_k1 = o_v0 + al256(4ull * n);
    const size_t o_v1 = o_k1 + (sort ? al256(8ull * n) : 0);
    const size_t o_h = o_v1 + (sort ? al256(4ull * n) : 0);
    const size_t o_s = o_h + (sort ? al256(4 * nh) : 0);
    const size_t bytes = o_s + al256(4 * (nh / kScan + 2));
    Scratch s(st);
    RBFB_CUDA(ctx, cudaMallocAsync(&s.p, bytes, st));
    char* base = static_cast<char*>(s.p);
    double* box = reinterpret_cast<double*>(base + o_box);
    auto* bb = reinterpret_cast<unsigned long long*>(base + o_bb);
    auto* k0 = reinterpret_cast<unsigned long long*>(base + o_k0);
    int* v0 = reinterpret_cast<int*>(base + o_v0);
    auto* k1 = reinterpret_cast<unsigned long long*>(base + o_k1);
    int* v1 = reinterpret_cast<int*>(base + o_v1);
    int* hist = reinterpret_cast<int*>(base + o_h);
    int* sums = reinterpret_cast<int*>(base + o_s);
    if (bbox_h) {
        RBFB_CUDA(ctx, cudaMemcpyAsync(box, bbox_h, 4 * sizeof(double), cudaMemcpyHostToDevice, st));
    } else {
        bbox_init_kernel<<<1, 1, 0, st>>>(bb);
        bbox_kernel<<<grid_of(ctx, n, 256), 256, 0, st>>>(x, y, n, bb);
        bbox_final_kernel<<<1, 1, 0, st>>>(bb, box);
        ctx->launches += 3;
    }
    keys_kernel<<<grid_of(ctx, n, 256), 256, 0, st>>>(x, y, n, box, ndiv, curve, k0, v0);
    ctx->launches += 1;
    RBFB_CUDA(ctx, cudaGetLastError());
    if (keys_out && !sort) {
        RBFB_CUDA(ctx, cudaMemcpyAsync(keys_out, k0, 8ull * n, cudaMemcpyDeviceToDevice, st));
        return RBFB_OK;
    }
    const int passes = (2 * ndiv + 7) / 8;
    for (int ps = 0; ps < passes; ++ps) {
        const int shift = 8 * ps;
        digit_hist_kernel<<<nblocks, kTpb, 0, st>>>(k0, n, shift, nblocks, hist);
        ctx->launches += 1;
        if (int r = scan(ctx, hist, hist, (int)nh, sums, nullptr, st)) return r;
        digit_scatter_kernel<<<nblocks, kTpb, 0, st>>>(k0, v0, n, shift, nblocks, hist, k1, v1);
        ctx->launches += 1;
        std::swap(k0, k1);
        std::swap(v0, v1);
    }
    RBFB_CUDA(ctx, cudaGetLastError());
    RBFB_CUDA(ctx, cudaMemcpyAsync(perm, v0, 4ull * n, cudaMemcpyDeviceToDevice, st));
    if (keys_out)
        RBFB_CUDA(ctx, cudaMemcpyAsync(keys_out, k0, 8ull * n, cudaMemcpyDeviceToDevice, st));
    if (inv) {
        inverse_kernel<<<grid_of(ctx, n, 256), 256, 0, st>>>(v0, n, inv);
        ctx->launches += 1;
    }
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

int rbfb_boundary_last(rbfb_ctx* ctx, int n, const int* flag, int* perm, int* inv, void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n < 0) return fail(ctx, RBFB_EINVAL, "negative size");
    if (n == 0) return RBFB_OK;
    if (!flag || !perm) return fail(ctx, RBFB_EINVAL, "null pointer argument");
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Scratch s(st);
    const size_t o_b = 0, o_s = al256(4ull * n), o_t = o_s + al256(4ull * (n / kScan + 2));
    RBFB_CUDA(ctx, cudaMallocAsync(&s.p, o_t + 256, st));
    char* base = static_cast<char*>(s.p);
    int* b = reinterpret_cast<int*>(base + o_b);
    int* sums = reinterpret_cast<int*>(base + o_s);
    int* total = reinterpret_cast<int*>(base + o_t);
    flag_kernel<<<grid_of(ctx, n, 256), 256, 0, st>>>(flag, n, b);
    ctx->launches += 1;
    if (int r = scan(ctx, b, b, n, sums, total, st)) return r;
    partition_kernel<<<grid_of(ctx, n, 256), 256, 0, st>>>(flag, b, n, total, perm, inv);
    ctx->launches += 1;
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

int rbfb_renumber_stencils(int n, int k, const int* ja, const int* perm, const int* inv,
                           int* ja_out, void* stream) {
    if (n < 0 || k < 1 || (n > 0 && (!ja || !perm || !inv || !ja_out)) || ja == ja_out)
        return RBFB_EINVAL;
    if (n == 0) return RBFB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long total = (long long)n * k;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148ll * 32);
    renumber_fixed_kernel<<<blocks, 256, 0, st>>>(n, k, ja, perm, inv, ja_out);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_renumber_csr(rbfb_ctx* ctx, int n, const int* ia, const int* ja, const int* perm,
                      const int* inv, int* ia_out, int* ja_out, void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n < 0 || (n > 0 && (!ia || !ja || !perm || !inv || !ia_out || !ja_out)) || ja == ja_out ||
        ia == ia_out)
        return fail(ctx, RBFB_EINVAL, "null or aliased pointer, or negative size");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        RBFB_CUDA(ctx, cudaMemsetAsync(ia_out, 0, sizeof(int), st));
        return RBFB_OK;
    }
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    Scratch s(st);
    RBFB_CUDA(ctx, cudaMallocAsync(&s.p, al256(4ull * (n / kScan + 2)), st));
    int* sums = static_cast<int*>(s.p);
    // ia_out[0..n-1] = lengths, scanned in place; ia_out[n] = the total
    row_len_kernel<<<grid_of(ctx, n, 256), 256, 0, st>>>(n, ia, perm, ia_out);
    ctx->launches += 1;
    if (int r = scan(ctx, ia_out, ia_out, n, sums, ia_out + n, st)) return r;
    renumber_csr_kernel<<<grid_of(ctx, 32ll * n, 256), 256, 0, st>>>(n, ia, ja, perm, inv, ia_out,
                                                                     ja_out);
    ctx->launches += 1;
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

int rbfb_permute(int n, const int* perm, const void* in, void* out, int elem_bytes, void* stream) {
    if (n < 0 || (n > 0 && (!perm || !in || !out)) || in == out ||
        (elem_bytes != 4 && elem_bytes != 8))
        return RBFB_EINVAL;
    if (n == 0) return RBFB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = std::min((n + 255) / 256, 148 * 32);
    if (elem_bytes == 8)
        gather_kernel<unsigned long long><<<blocks, 256, 0, st>>>(
            n, perm, static_cast<const unsigned long long*>(in), static_cast<unsigned long long*>(out));
    else
        gather_kernel<int><<<blocks, 256, 0, st>>>(n, perm, static_cast<const int*>(in),
                                                   static_cast<int*>(out));
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

}  // extern "C"
