// runtime.cu -- context, launch selection and the assembly entry points of
// the C ABI (include/rbf_b200.h).
//
// The reference launches assemble_interp_weights<Config><<<nstencils,
// block_dim, smem>>> after an optional cudaFuncSetAttribute opt-in
// (src/rbf_operators.h:317-328, usage sketched at src/main.cpp:38-45). Here
// the shape is chosen at run time from the compiled variants, the grid is
// persistent (SM count x resident CTAs), and the FP32-refinement path chains
// the FP64 kernel over the stencils it could not refine, on the same stream,
// without a host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "runtime.h"

namespace rbfb {

int fail(rbfb_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(rbfb_ctx* ctx, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    if (ctx) ctx->err = m;
    return e == cudaErrorMemoryAllocation ? RBFB_ENOMEM : RBFB_ECUDA;
}

int rhs_columns(const rbfb_desc* d, AsmParams& p) {
    int m = 0;
    if (d->ops & RBFB_OP_INTERP) {
        if (d->nc < 1 || !d->xc || !d->yc) return RBFB_EINVAL;
        for (int j = 0; j < d->nc; ++j) {
            if (m >= kMaxRhs) return RBFB_EUNSUPPORTED;
            p.col_op[m] = RBFB_OP_INTERP;
            p.col_ic[m] = j;
            ++m;
        }
    }
    for (int bit = RBFB_OP_LAPLACE; bit <= RBFB_OP_DXY; bit <<= 1) {
        if (d->ops & bit) {
            if (m >= kMaxRhs) return RBFB_EUNSUPPORTED;
            p.col_op[m] = bit;
            p.col_ic[m] = 0;
            ++m;
        }
    }
    if (d->ops & ~(RBFB_OP_INTERP | RBFB_OP_LAPLACE | RBFB_OP_DX | RBFB_OP_DY | RBFB_OP_DXX |
                   RBFB_OP_DYY | RBFB_OP_DXY))
        return RBFB_EINVAL;
    if (m == 0) return RBFB_EINVAL;
    p.nrhs = m;
    p.xc = d->xc;
    p.yc = d->yc;
    return m;
}

int pick_variant(rbfb_ctx* ctx, bool mixed, int P, int Q, int n, int nrhs) {
    const auto& vs = variants();
    auto serves = [&](const Variant& v) {
        return v.mixed == mixed && v.P == P && v.Q == Q && v.nrhs >= nrhs;
    };
    int best_ntp = 1 << 30;
    for (const auto& v : vs)
        if (serves(v) && v.ntp >= n) best_ntp = std::min(best_ntp, v.ntp);
    if (best_ntp == (1 << 30)) return -1;
    if (ctx) {
        auto it = ctx->tuned.find({mixed ? 1 : 0, P, Q, best_ntp});
        if (it != ctx->tuned.end() && it->second.variant >= 0 && serves(vs[it->second.variant]) &&
            vs[it->second.variant].ntp >= n)
            return it->second.variant;
    }
    for (size_t i = 0; i < vs.size(); ++i)
        if (serves(vs[i]) && vs[i].ntp == best_ntp) return static_cast<int>(i);
    return -1;
}

int grid_for(rbfb_ctx* ctx, int v, int bps_override) {
    const auto& var = variants()[v];
    if (ctx->occ.size() != variants().size()) ctx->occ.assign(variants().size(), -1);
    if (ctx->occ[v] < 0) {
        cudaError_t e = cudaFuncSetAttribute(var.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             var.smem_block);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaFuncSetAttribute");
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, var.kernel, var.block,
                                                          var.smem_block);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        if (nb < 1) return fail(ctx, RBFB_EUNSUPPORTED, std::string("variant does not fit an SM: ") + var.name);
        ctx->occ[v] = nb;
    }
    int bps = ctx->occ[v];
    if (bps_override > 0) bps = std::min(bps, bps_override);
    return bps * ctx->sms;
}

int launch_variant(rbfb_ctx* ctx, int v, const AsmParams& p, cudaStream_t st, int blocks) {
    const auto& var = variants()[v];
    if (blocks <= 0) {
        // a tuned CTAs-per-SM for this shape, if the autotuner chose one (the
        // entry sits under the smallest system size of its class)
        for (const auto& kv : ctx->tuned) {
            if (kv.second.variant == v && kv.second.blocks_per_sm > 0) {
                const int g = grid_for(ctx, v, kv.second.blocks_per_sm);
                if (g < 0) return g;
                blocks = g;
                break;
            }
        }
    }
    int grid = blocks > 0 ? blocks : grid_for(ctx, v);
    if (grid < 0) return grid;
    if (blocks > 0) {
        int g2 = grid_for(ctx, v);  // ensure the opt-in happened
        if (g2 < 0) return g2;
    }
    var.launch(dim3(grid), var.block, var.smem_block, st, p);
    ctx->launches.fetch_add(1, std::memory_order_relaxed);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, (std::string("launch of ") + var.name).c_str());
    return RBFB_OK;
}

int ensure_fb(rbfb_ctx* ctx, size_t n) {
    if (ctx->fb_cap >= n) return RBFB_OK;
    if (ctx->fb_list) cudaFree(ctx->fb_list);
    ctx->fb_list = nullptr;
    ctx->fb_cap = 0;
    const size_t cap = std::max<size_t>(n, 1024);
    RBFB_CUDA(ctx, cudaMalloc(&ctx->fb_list, cap * sizeof(int)));
    ctx->fb_cap = cap;
    return RBFB_OK;
}

__global__ void count_nonzero_kernel(const int* info, int n, unsigned long long* out) {
    unsigned long long c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        c += (info[i] != 0);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

int count_singular(rbfb_ctx* ctx, const int* info, int n, unsigned long long* out, cudaStream_t st) {
    if (n <= 0 || !info) return RBFB_OK;
    const int blocks = std::min((n + 255) / 256, ctx->sms * 4);
    count_nonzero_kernel<<<blocks, 256, 0, st>>>(info, n, out);
    ctx->launches.fetch_add(1, std::memory_order_relaxed);
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

int check_desc(rbfb_ctx* ctx, const rbfb_desc* d) {
    if (!d) return fail(ctx, RBFB_EINVAL, "null descriptor");
    if (d->degree < 0 || d->degree > 4) return fail(ctx, RBFB_EINVAL, "degree must be 0..4");
    if (d->phs != 0 && (d->phs < 1 || d->phs % 2 == 0)) return fail(ctx, RBFB_EINVAL, "phs must be odd");
    if (d->precision != RBFB_FP64 && d->precision != RBFB_FP32_IR)
        return fail(ctx, RBFB_EINVAL, "unknown precision");
    return RBFB_OK;
}

namespace {

// Common set-up of the parameters of one call.
int base_params(rbfb_ctx* ctx, const rbfb_desc* d, int nstencils, const double* x, const double* y,
                const int* ja, double* const* values_h, double* const* values_d, int* info,
                DevCounters* ctr, AsmParams& p) {
    std::memset(&p, 0, sizeof(p));
    int rc = rhs_columns(d, p);
    if (rc < 0) return fail(ctx, rc, "bad operator mask / interpolation points");
    if (!x || !y || !ja || (!values_h && !values_d))
        return fail(ctx, RBFB_EINVAL, "null pointer argument");
    if (values_d) {
        p.values_dev = values_d;  // read by the kernels
    } else {
        for (int q = 0; q < p.nrhs; ++q) {
            if (!values_h[q]) return fail(ctx, RBFB_EINVAL, "null values pointer");
            p.values[q] = values_h[q];
        }
    }
    p.nitems = nstencils;
    p.x = x;
    p.y = y;
    p.ja = ja;
    p.Lx = d->period[0];
    p.Ly = d->period[1];
    p.scale = d->scale;
    p.info = info;
    p.max_sweeps = d->max_sweeps > 0 ? d->max_sweeps : 6;
    p.ir_tol = d->ir_tol > 0 ? d->ir_tol : 1e-11;
    p.fb_count = &ctr->fb_count;
    p.sweeps_max = &ctr->sweeps_max;
    p.sweeps_sum = &ctr->sweeps_sum;
    return RBFB_OK;
}

int finish_stats(rbfb_ctx* ctx, const int* info, int nstencils, rbfb_stats* stats, cudaStream_t st,
                 cudaEvent_t ev0, cudaEvent_t ev1, int buckets) {
    if (!stats) return RBFB_OK;
    int rc = count_singular(ctx, info, nstencils, &ctx->ctr->singular, st);
    if (rc) return rc;
    RBFB_CUDA(ctx, cudaEventRecord(ev1, st));
    DevCounters h{};
    RBFB_CUDA(ctx, cudaMemcpyAsync(&h, ctx->ctr, sizeof(h), cudaMemcpyDeviceToHost, st));
    RBFB_CUDA(ctx, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    stats->stencils = nstencils;
    stats->singular = static_cast<long long>(h.singular);
    stats->fallback = h.fb_count;
    stats->sweeps = static_cast<long long>(h.sweeps_sum);
    stats->max_sweeps_used = h.sweeps_max;
    stats->buckets = buckets;
    stats->ms = ms;
    return RBFB_OK;
}

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

}  // namespace

int enqueue_fixed(rbfb_ctx* ctx, const rbfb_desc* desc, int first, int count, const double* x,
                  const double* y, int k, const int* ja, double* const* values, int* info,
                  DevCounters* ctr, int* fb, cudaStream_t st, int row_base,
                  double* const* values_d) {
    const int P = desc->degree;
    const int Q = desc->phs ? desc->phs : 2 * P - 1;
    const int n = k + npoly(P);
    const bool mixed = desc->precision == RBFB_FP32_IR;
    AsmParams p;
    int rc = base_params(ctx, desc, count, x, y, ja, values, values_d, info, ctr, p);
    if (rc) return rc;
    const int v = pick_variant(ctx, mixed, P, Q, n, p.nrhs);
    if (v < 0)
        return fail(ctx, RBFB_EUNSUPPORTED,
                    "no compiled kernel for P=" + std::to_string(P) + " Q=" + std::to_string(Q) +
                        " n=" + std::to_string(n) + " with " + std::to_string(p.nrhs) +
                        " right-hand sides");
    if (p.nrhs > variants()[v].nrhs)
        return fail(ctx, RBFB_EUNSUPPORTED, "more right-hand sides than the compiled kernels hold");
    p.k = k;
    p.item_base = first;
    p.row_base = row_base;
    if (count == 0) return RBFB_OK;
    if (!mixed) return launch_variant(ctx, v, p, st);
    p.fb_list = fb;
    rc = launch_variant(ctx, v, p, st);
    if (rc) return rc;
    // FP64 kernel over the stencils whose refinement stalled
    const int v64 = pick_variant(ctx, false, P, Q, n, p.nrhs);
    if (v64 < 0) return fail(ctx, RBFB_EUNSUPPORTED, "no FP64 fallback kernel for this shape");
    AsmParams f = p;
    f.list = fb;
    f.item_base = 0;
    f.nitems_dev = &ctr->fb_count;
    f.fb_list = nullptr;
    return launch_variant(ctx, v64, f, st);
}

}  // namespace rbfb

using namespace rbfb;

extern "C" {

const char* rbfb_status_string(int status) {
    switch (status) {
        case RBFB_OK: return "ok";
        case RBFB_EINVAL: return "invalid argument";
        case RBFB_ECUDA: return "CUDA error";
        case RBFB_ENOMEM: return "out of memory";
        case RBFB_EUNSUPPORTED: return "no compiled kernel for this shape";
        case RBFB_ETIMEOUT: return "timed out";
        case RBFB_EBUDGET: return "request exceeds the memory budget";
        case RBFB_ENOTFOUND: return "unknown ticket";
        case RBFB_EBUSY: return "not finished";
        case RBFB_ETOOBIG: return "problem exceeds the fixed scratch of the no-allocation call";
        case RBFB_ENOCONV: return "iterative solve did not converge within maxit";
        case RBFB_EBREAKDOWN: return "iterative solve broke down";
        default: return status > 0 ? "singular stencils" : "unknown status";
    }
}

const char* rbfb_last_error(const rbfb_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

long long rbfb_kernel_launches(const rbfb_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

int rbfb_create(rbfb_ctx** out, int device) {
    if (!out) return RBFB_EINVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return RBFB_ECUDA;
    if (device < 0 || device >= ndev) return RBFB_EINVAL;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return RBFB_ECUDA;
    auto* ctx = new rbfb_ctx();
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    e = cudaMalloc(&ctx->ctr, sizeof(DevCounters));
    if (e != cudaSuccess) {
        delete ctx;
        return RBFB_ENOMEM;
    }
    cudaMemset(ctx->ctr, 0, sizeof(DevCounters));
    *out = ctx;
    return RBFB_OK;
}

void rbfb_release_pipeline(rbfb_ctx* ctx);  // host_pipeline.cu
void rbfb_release_knn(rbfb_ctx* ctx);       // knn.cu
void rbfb_release_batch(rbfb_ctx* ctx);     // batch.cu
void rbfb_release_solve(rbfb_ctx* ctx);     // solve.cu

int rbfb_destroy(rbfb_ctx* ctx) {
    if (!ctx) return RBFB_OK;
    cudaSetDevice(ctx->device);
    rbfb_release_pipeline(ctx);
    rbfb_release_knn(ctx);
    rbfb_release_batch(ctx);
    rbfb_release_solve(ctx);
    if (ctx->fb_list) cudaFree(ctx->fb_list);
    if (ctx->ctr) cudaFree(ctx->ctr);
    delete ctx;
    return RBFB_OK;
}

namespace {

int assemble_fixed_call(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                        const double* y, int k, const int* ja, double* const* values_h,
                        double* const* values_d, int* info, rbfb_stats* stats, void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int rc = check_desc(ctx, desc);
    if (rc) return rc;
    if (nstencils < 0 || k < 1) return fail(ctx, RBFB_EINVAL, "nstencils >= 0 and k >= 1 required");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    EventPair ev;
    if (stats) {
        RBFB_CUDA(ctx, cudaEventCreate(&ev.a));
        RBFB_CUDA(ctx, cudaEventCreate(&ev.b));
        RBFB_CUDA(ctx, cudaEventRecord(ev.a, st));
    }
    RBFB_CUDA(ctx, cudaMemsetAsync(ctx->ctr, 0, sizeof(DevCounters), st));
    if (desc->precision == RBFB_FP32_IR) {
        rc = ensure_fb(ctx, static_cast<size_t>(std::max(nstencils, 1)));
        if (rc) return rc;
    }
    rc = enqueue_fixed(ctx, desc, 0, nstencils, x, y, k, ja, values_h, info, ctx->ctr,
                       ctx->fb_list, st, 0, values_d);
    if (rc) return rc;
    return finish_stats(ctx, info, nstencils, stats, st, ev.a, ev.b, 1);
}

}  // namespace

int rbfb_assemble(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                  const double* y, int k, const int* ja, double* const* values_h, int* info,
                  rbfb_stats* stats, void* stream) {
    return assemble_fixed_call(ctx, desc, nstencils, x, y, k, ja, values_h, nullptr, info, stats,
                               stream);
}

int rbfb_assemble_dtab(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                       const double* y, int k, const int* ja, double* const* values_d, int* info,
                       rbfb_stats* stats, void* stream) {
    if (!values_d) return ctx ? fail(ctx, RBFB_EINVAL, "null values table") : RBFB_EINVAL;
    return assemble_fixed_call(ctx, desc, nstencils, x, y, k, ja, nullptr, values_d, info, stats,
                               stream);
}

int rbfb_assemble_range(rbfb_ctx* ctx, const rbfb_desc* desc, int first, int count, int n,
                        const double* x, const double* y, int k, const int* ja_rows,
                        double* const* values_rows, int* info_rows, rbfb_stats* stats,
                        void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int rc = check_desc(ctx, desc);
    if (rc) return rc;
    if (first < 0 || count < 0 || first + count > n || k < 1)
        return fail(ctx, RBFB_EINVAL, "need 0 <= first, first + count <= n, k >= 1");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    EventPair ev;
    if (stats) {
        RBFB_CUDA(ctx, cudaEventCreate(&ev.a));
        RBFB_CUDA(ctx, cudaEventCreate(&ev.b));
        RBFB_CUDA(ctx, cudaEventRecord(ev.a, st));
    }
    RBFB_CUDA(ctx, cudaMemsetAsync(ctx->ctr, 0, sizeof(DevCounters), st));
    if (desc->precision == RBFB_FP32_IR) {
        rc = ensure_fb(ctx, static_cast<size_t>(std::max(count, 1)));
        if (rc) return rc;
    }
    rc = enqueue_fixed(ctx, desc, first, count, x, y, k, ja_rows, values_rows, info_rows, ctx->ctr,
                       ctx->fb_list, st, first);
    if (rc) return rc;
    return finish_stats(ctx, info_rows, count, stats, st, ev.a, ev.b, 1);
}

}  // extern "C"
