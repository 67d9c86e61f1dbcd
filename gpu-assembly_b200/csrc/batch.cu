// batch.cu -- uneven stencils: rbfb_assemble_csr.
//
// FP64 batches (up to 3 right-hand sides) run as ONE persistent launch of the
// uneven kernel (asm_blocked.cuh, blk_csr_kernel): warps claim stencils of
// any size and degree from a device counter, walking a list sorted by class
// on the device (largest systems first); systems of up to 45 unknowns are
// solved in shared memory, larger ones (up to 96) in an L2-resident global
// scratch region per warp.
//
// Other batches (the FP32-refinement form, more right-hand sides) are
// bucketed on the device by the compiled kernel shape that fits them
// (smallest padded system size >= k + npoly(P)), counting-sorted into one
// stencil list, and each bucket's persistent kernel walks its slice of the
// list. Bucket sizes and offsets stay on the device (kernels read them
// through pointers), so the whole call is a fixed sequence of launches with
// no host round trip; the sequence is captured once into a CUDA graph and
// replayed for the same batch.
//
// The reference's only CSR-driven assembly is the Fortran fill_kernel over
// ia/ja (src/rbf_cuda.f90:36-99); its C++ kernel takes one fixed stencil size
// per launch (src/rbf_operators.h:187-210).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <vector>

#include "asm_blocked.cuh"
#include "runtime.h"

namespace rbfb {
namespace {

// The single-launch FP64 kernel for uneven batches: systems of up to 45
// unknowns (degree 3 with k = 35, the largest interior stencil in common
// use) in a 19 KB shared-memory slot, 11 CTAs of one warp per SM; up to 96
// in global scratch. Its n > 45 body (three list slots a lane) would set
// the register count of every path (230); bounded to 11 CTAs per SM it fits
// in 168 registers, spilling only on that rare path.
constexpr int kOneNS = 45, kOneNG = 96, kOneBlock = 32, kOnePB = 8, kOneMinB = 11;
using OneCfg = CsrCfg<double, kOneNS, kOneNG, 3, kOnePB>;
constexpr int kOneSmem = OneCfg::SmemL::bytes * (kOneBlock / 32);
// The launch walks the stencils sorted by class (system size descending,
// then degree): warps on one SM then run the same fill and elimination
// bodies (the instruction cache holds one at a time), and the largest
// systems go first instead of forming the tail. kOneKeys classes.
constexpr int kOneKeys = (kOneNG + 2) * 5;
__host__ __device__ constexpr int one_key(int n, int P) { return (kOneNG + 1 - n) * 5 + P; }

constexpr int kMaxVariants = 64;
constexpr int kTabN = 161;  // system sizes 0..160

struct BatchState {
    int* table = nullptr;     // [5][kTabN] variant per (P, n), -1 = none
    int table_mixed = -1, table_phs = -1, table_pmin = -1, table_pmax = -1;
    size_t table_tuned = 0;   // size of the context's tuned table when built
    std::vector<int> table_used;
    int* counts = nullptr;    // [kMaxVariants] x 3: counts | offsets | cursors
    DevCounters* ctrs = nullptr;  // per bucket
    int* err = nullptr;
    size_t cap = 0;
    int* bucket_of = nullptr;
    int* list = nullptr;
    // the single-launch kernel: persistent grid, its global scratch, and the
    // class counts | offsets | cursors of its sorted stencil list
    int one_grid = 0;
    int* one_counts = nullptr;
    char* gscratch = nullptr;
    size_t gscratch_bytes = 0;
    // cached graph of the last batch
    cudaGraphExec_t graph = nullptr;
    std::vector<unsigned char> graph_key;
    long long graph_launches = 0;  // kernels in the graph
};

BatchState* state(rbfb_ctx* ctx) {
    if (!ctx->batch) ctx->batch = new BatchState();
    return static_cast<BatchState*>(ctx->batch);
}

__global__ void assign_kernel(int nst, const int* ia, const int8_t* degree, int P0, const int* table,
                              int* bucket_of, int* counts, int* err) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nst; s += gridDim.x * blockDim.x) {
        const int ks = ia[s + 1] - ia[s];
        const int P = degree ? degree[s] : P0;
        int b = -1;
        if (P >= 0 && P <= 4 && ks >= 1) {
            const int n = ks + npoly(P);
            if (n < kTabN) b = table[P * kTabN + n];
        }
        bucket_of[s] = b;
        if (b >= 0) atomicAdd(counts + b, 1);
        else atomicExch(err, 1);
    }
}

__global__ void offsets_kernel(int* counts, int nb) {
    int acc = 0;
    for (int b = 0; b < nb; ++b) {
        counts[kMaxVariants + b] = acc;   // offsets
        counts[2 * kMaxVariants + b] = 0; // cursors
        acc += counts[b];
    }
}

// Class of every stencil of the single launch (an invalid one gets the
// last class; the kernel flags it) and the class counts.
__global__ void one_assign_kernel(int nst, const int* ia, const int8_t* degree, int P0,
                                  int* key_of, int* counts) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nst; s += gridDim.x * blockDim.x) {
        const int ks = ia[s + 1] - ia[s];
        const int P = degree ? degree[s] : P0;
        int key = kOneKeys - 1;
        if (P >= 0 && P <= 4 && ks >= 1 && ks + npoly(P) <= kOneNG) key = one_key(ks + npoly(P), P);
        key_of[s] = key;
        atomicAdd(counts + key, 1);
    }
}

__global__ void one_offsets_kernel(int* counts) {
    __shared__ int part[kOneKeys];
    for (int i = threadIdx.x; i < kOneKeys; i += blockDim.x) part[i] = counts[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int i = 0; i < kOneKeys; ++i) {
            const int c = part[i];
            part[i] = acc;
            acc += c;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kOneKeys; i += blockDim.x) {
        counts[kOneKeys + i] = part[i];  // offsets
        counts[2 * kOneKeys + i] = 0;    // cursors
    }
}

__global__ void one_scatter_kernel(int nst, const int* key_of, int* counts, int* list) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nst; s += gridDim.x * blockDim.x) {
        const int key = key_of[s];
        list[counts[kOneKeys + key] + atomicAdd(counts + 2 * kOneKeys + key, 1)] = s;
    }
}

__global__ void scatter_kernel(int nst, const int* bucket_of, int* counts, int* list) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nst; s += gridDim.x * blockDim.x) {
        const int b = bucket_of[s];
        if (b < 0) continue;
        list[counts[kMaxVariants + b] + atomicAdd(counts + 2 * kMaxVariants + b, 1)] = s;
    }
}

int ensure(rbfb_ctx* ctx, BatchState* b, size_t n) {
    if (!b->counts) {
        RBFB_CUDA(ctx, cudaMalloc(&b->counts, 3 * kMaxVariants * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&b->ctrs, kMaxVariants * sizeof(DevCounters)));
        RBFB_CUDA(ctx, cudaMalloc(&b->err, sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&b->table, 5 * kTabN * sizeof(int)));
    }
    if (b->cap < n) {
        cudaFree(b->bucket_of);
        cudaFree(b->list);
        b->bucket_of = b->list = nullptr;
        b->cap = 0;
        RBFB_CUDA(ctx, cudaMalloc(&b->bucket_of, n * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&b->list, n * sizeof(int)));
        b->cap = n;
    }
    return ensure_fb(ctx, n);
}

// The (P, n) -> variant table for one precision and PHS rule; also returns
// the set of variants that can occur for the allowed degrees.
int build_table(rbfb_ctx* ctx, BatchState* b, bool mixed, int phs, int Pmin, int Pmax,
                std::vector<int>& used) {
    if (b->table_mixed == (mixed ? 1 : 0) && b->table_phs == phs && b->table_pmin == Pmin &&
        b->table_pmax == Pmax && b->table_tuned == ctx->tuned.size()) {
        used = b->table_used;  // unchanged: no upload
        return RBFB_OK;
    }
    std::vector<int> tab(5 * kTabN, -1);
    used.clear();
    for (int P = 0; P <= 4; ++P)
        for (int n = 1; n < kTabN; ++n) {
            const int Q = phs ? phs : 2 * P - 1;
            if (Q < 1) continue;
            const int v = pick_variant(ctx, mixed, P, Q, n);
            tab[P * kTabN + n] = v;
            if (v >= 0 && P >= Pmin && P <= Pmax &&
                std::find(used.begin(), used.end(), v) == used.end())
                used.push_back(v);
        }
    RBFB_CUDA(ctx, cudaMemcpy(b->table, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice));
    b->table_mixed = mixed ? 1 : 0;
    b->table_phs = phs;
    b->table_pmin = Pmin;
    b->table_pmax = Pmax;
    b->table_tuned = ctx->tuned.size();
    b->table_used = used;
    return RBFB_OK;
}

// Grid and global scratch of the single-launch kernel (set up outside any
// stream capture).
int ensure_one(rbfb_ctx* ctx, BatchState* b) {
    const void* k = reinterpret_cast<const void*>(
        &blk_csr_kernel<double, kOneNS, kOneNG, 3, kOneBlock, kOnePB, kOneMinB>);
    if (!b->one_counts) RBFB_CUDA(ctx, cudaMalloc(&b->one_counts, 3 * kOneKeys * sizeof(int)));
    if (b->one_grid == 0) {
        RBFB_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kOneSmem));
        int nb = 0;
        RBFB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kOneBlock, kOneSmem));
        if (nb < 1) return fail(ctx, RBFB_EUNSUPPORTED, "uneven kernel does not fit an SM");
        b->one_grid = nb * ctx->sms;
    }
    const size_t need = static_cast<size_t>(b->one_grid) * (kOneBlock / 32) * OneCfg::gbytes;
    if (b->gscratch_bytes < need) {
        cudaFree(b->gscratch);
        b->gscratch = nullptr;
        b->gscratch_bytes = 0;
        RBFB_CUDA(ctx, cudaMalloc(&b->gscratch, need));
        b->gscratch_bytes = need;
    }
    return RBFB_OK;
}

void release(BatchState* b) {
    cudaFree(b->gscratch);
    cudaFree(b->one_counts);
    cudaFree(b->table); cudaFree(b->counts); cudaFree(b->ctrs); cudaFree(b->err);
    cudaFree(b->bucket_of); cudaFree(b->list);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    delete b;
}

}  // namespace
}  // namespace rbfb

using namespace rbfb;

extern "C" {

void rbfb_release_batch(rbfb_ctx* ctx) {
    if (ctx->batch) release(static_cast<BatchState*>(ctx->batch));
    ctx->batch = nullptr;
}

int rbfb_assemble_csr(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                      const double* y, const int* ia, const int* ja, const int8_t* degree,
                      double* const* values_h, int* info, rbfb_stats* stats, void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int rc = check_desc(ctx, desc);
    if (rc) return rc;
    if (nstencils < 0 || !ia || !ja || !x || !y || !values_h)
        return fail(ctx, RBFB_EINVAL, "null pointer argument");
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BatchState* b = state(ctx);
    rc = ensure(ctx, b, static_cast<size_t>(std::max(nstencils, 1)));
    if (rc) return rc;
    const bool mixed = desc->precision == RBFB_FP32_IR;

    // the parameters every bucket shares
    AsmParams p;
    std::memset(&p, 0, sizeof(p));
    const int nrhs = rhs_columns(desc, p);
    if (nrhs < 0) return fail(ctx, nrhs, "bad operator mask / interpolation points");
    // FP64 with up to 3 right-hand sides: the whole batch in ONE persistent
    // launch of the uneven kernel; otherwise bucketed launches
    const bool one = !mixed && nrhs <= 3 &&
                     (desc->phs == 0 || desc->phs == 3 || desc->phs == 5 || desc->phs == 7 ||
                      desc->phs == 9);
    std::vector<int> used;
    if (one) {
        rc = ensure_one(ctx, b);
        if (rc) return rc;
    } else {
        rc = build_table(ctx, b, mixed, desc->phs, degree ? 0 : desc->degree,
                         degree ? 4 : desc->degree, used);
        if (rc) return rc;
        if (used.empty()) return fail(ctx, RBFB_EUNSUPPORTED, "no compiled kernel for these degrees");
    }
    for (int q = 0; q < nrhs; ++q) {
        if (!values_h[q]) return fail(ctx, RBFB_EINVAL, "null values pointer");
        p.values[q] = values_h[q];
    }
    p.x = x;
    p.y = y;
    p.ja = ja;
    p.ia = ia;
    p.Lx = desc->period[0];
    p.Ly = desc->period[1];
    p.scale = desc->scale;
    p.info = info;
    p.max_sweeps = desc->max_sweeps > 0 ? desc->max_sweeps : 6;
    p.ir_tol = desc->ir_tol > 0 ? desc->ir_tol : 1e-11;
    p.list = b->list;

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        RBFB_CUDA(ctx, cudaEventCreate(&e0));
        RBFB_CUDA(ctx, cudaEventCreate(&e1));
        RBFB_CUDA(ctx, cudaEventRecord(e0, st));
    }
    const int nb = static_cast<int>(variants().size());
    if (nb > kMaxVariants) return fail(ctx, RBFB_EUNSUPPORTED, "too many compiled shapes");
    // occupancy queries and shared-memory opt-ins before any capture
    for (int v : used) {
        if (grid_for(ctx, v) < 0) return RBFB_ECUDA;
        if (mixed) {
            const auto& var = variants()[v];
            const int v64 = pick_variant(ctx, false, var.P, var.Q, var.ntp);
            if (v64 < 0) return fail(ctx, RBFB_EUNSUPPORTED, "no FP64 fallback kernel");
            if (grid_for(ctx, v64) < 0) return RBFB_ECUDA;
        }
        if (nrhs > variants()[v].nrhs) return fail(ctx, RBFB_EUNSUPPORTED, "too many right-hand sides");
    }
    // the whole batch in one launch: warps claim stencils from a counter
    auto enqueue_one = [&](cudaStream_t s) -> int {
        RBFB_CUDA(ctx, cudaMemsetAsync(b->ctrs, 0, kMaxVariants * sizeof(DevCounters), s));
        RBFB_CUDA(ctx, cudaMemsetAsync(b->err, 0, sizeof(int), s));
        if (nstencils == 0) return RBFB_OK;
        // the stencils sorted by class (counting sort on the device)
        RBFB_CUDA(ctx, cudaMemsetAsync(b->one_counts, 0, kOneKeys * sizeof(int), s));
        const int blocks = std::max(1, std::min((nstencils + 255) / 256, ctx->sms * 8));
        one_assign_kernel<<<blocks, 256, 0, s>>>(nstencils, ia, degree, desc->degree, b->bucket_of,
                                                 b->one_counts);
        one_offsets_kernel<<<1, 256, 0, s>>>(b->one_counts);
        one_scatter_kernel<<<blocks, 256, 0, s>>>(nstencils, b->bucket_of, b->one_counts, b->list);
        AsmParams q = p;
        q.list = b->list;
        q.item_base = 0;
        q.nitems = nstencils;
        q.work = &b->ctrs[0].work[0];
        blk_csr_kernel<double, kOneNS, kOneNG, 3, kOneBlock, kOnePB, kOneMinB>
            <<<b->one_grid, kOneBlock, kOneSmem, s>>>(q, degree, desc->degree, desc->phs,
                                                       b->gscratch, b->err);
        ctx->launches += 4;
        RBFB_CUDA(ctx, cudaGetLastError());
        return RBFB_OK;
    };
    // the whole batch: a fixed sequence of launches, sizes read on the device
    auto enqueue_buckets = [&](cudaStream_t s) -> int {
        RBFB_CUDA(ctx, cudaMemsetAsync(b->counts, 0, 3 * kMaxVariants * sizeof(int), s));
        RBFB_CUDA(ctx, cudaMemsetAsync(b->ctrs, 0, kMaxVariants * sizeof(DevCounters), s));
        RBFB_CUDA(ctx, cudaMemsetAsync(b->err, 0, sizeof(int), s));
        if (nstencils == 0) return RBFB_OK;
        const int blocks = std::max(1, std::min((nstencils + 255) / 256, ctx->sms * 8));
        assign_kernel<<<blocks, 256, 0, s>>>(nstencils, ia, degree, desc->degree, b->table,
                                             b->bucket_of, b->counts, b->err);
        offsets_kernel<<<1, 1, 0, s>>>(b->counts, nb);
        scatter_kernel<<<blocks, 256, 0, s>>>(nstencils, b->bucket_of, b->counts, b->list);
        ctx->launches += 3;
        RBFB_CUDA(ctx, cudaGetLastError());
        for (int v : used) {
            AsmParams q = p;
            q.nitems_dev = b->counts + v;
            q.list_off_dev = b->counts + kMaxVariants + v;
            q.fb_list = ctx->fb_list;
            q.fb_count = &b->ctrs[v].fb_count;
            q.sweeps_max = &b->ctrs[v].sweeps_max;
            q.sweeps_sum = &b->ctrs[v].sweeps_sum;
            int r = launch_variant(ctx, v, q, s);
            if (r) return r;
            if (mixed) {
                const auto& var = variants()[v];
                AsmParams f = q;
                f.list = ctx->fb_list;
                f.nitems_dev = &b->ctrs[v].fb_count;
                f.fb_list = nullptr;
                r = launch_variant(ctx, pick_variant(ctx, false, var.P, var.Q, var.ntp), f, s);
                if (r) return r;
            }
        }
        return RBFB_OK;
    };
    auto enqueue = [&](cudaStream_t s) -> int { return one ? enqueue_one(s) : enqueue_buckets(s); };
    // Captured into a CUDA graph on a non-default stream, replayed while the
    // arguments (and the context's buffers) stay the same.
    if (st != nullptr) {
        std::vector<unsigned char> key;
        auto put = [&](const void* q, size_t len) {
            const auto* c = static_cast<const unsigned char*>(q);
            key.insert(key.end(), c, c + len);
        };
        const void* ptrs[] = {x, y, ia, ja, degree, info, b->list, b->bucket_of, b->counts,
                              b->ctrs, ctx->fb_list, b->table, b->gscratch, b->one_counts};
        put(ptrs, sizeof(ptrs));
        put(p.values, sizeof(p.values));
        put(&nstencils, sizeof(nstencils));
        put(desc, offsetof(rbfb_desc, nc));
        put(&desc->nc, sizeof(desc->nc));
        put(&one, sizeof(one));
        if (!b->graph || key != b->graph_key) {
            if (b->graph) cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
            const long long l0 = ctx->launches.load();
            RBFB_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            rc = enqueue(st);
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(st, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ec != cudaSuccess) return cuda_fail(ctx, ec, "cudaStreamEndCapture");
            const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) {
                b->graph = nullptr;
                return cuda_fail(ctx, ei, "cudaGraphInstantiate");
            }
            b->graph_key = key;
            b->graph_launches = ctx->launches.load() - l0;
            ctx->launches -= b->graph_launches;  // counted when the graph runs
        }
        RBFB_CUDA(ctx, cudaGraphLaunch(b->graph, st));
        ctx->launches += b->graph_launches;
    } else {
        rc = enqueue(st);
        if (rc) return rc;
    }
    if (!stats) return RBFB_OK;
    std::vector<DevCounters> h(nb);
    int herr = 0;
    rc = count_singular(ctx, info, nstencils, &b->ctrs[0].singular, st);
    if (rc) return rc;
    RBFB_CUDA(ctx, cudaEventRecord(e1, st));
    RBFB_CUDA(ctx, cudaMemcpyAsync(h.data(), b->ctrs, nb * sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
    RBFB_CUDA(ctx, cudaMemcpyAsync(&herr, b->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    RBFB_CUDA(ctx, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::memset(stats, 0, sizeof(*stats));
    stats->stencils = nstencils;
    stats->singular = static_cast<long long>(h[0].singular);
    for (const auto& c : h) {
        stats->fallback += c.fb_count;
        stats->sweeps += static_cast<long long>(c.sweeps_sum);
        stats->max_sweeps_used = std::max(stats->max_sweeps_used, c.sweeps_max);
    }
    stats->buckets = one ? 1 : static_cast<int>(used.size());
    stats->ms = ms;
    if (herr) return fail(ctx, RBFB_EUNSUPPORTED, "a stencil has no compiled kernel (size or degree)");
    return RBFB_OK;
}

}  // extern "C"
