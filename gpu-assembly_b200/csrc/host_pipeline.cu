// host_pipeline.cu -- rbfb_assemble_host: the end-to-end call from host
// memory. Nodes go in once; the k-NN search runs on a compute stream, then
// the assembly in chunks of stencils, alternating between two compute
// streams so that a chunk's kernel fills the SMs its predecessor's last
// CTAs leave idle (the chunks' outputs are disjoint and their kernels
// assign stencils statically). Each chunk's weights are copied back on a
// third stream as soon as the chunk is done, so the device->host transfer
// of the CSR values (the largest transfer of the call) overlaps the
// assembly of the next chunks. Copies are asynchronous, and overlap, when
// the host buffers are pinned (cudaHostAlloc / cudaHostRegister).
//
// No reference counterpart: the reference's caller copies and launches by
// hand (src/main.cpp:27-53, src/main.f90:25-57).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "runtime.h"

namespace rbfb {
namespace {

struct Pipe {
    size_t n_cap = 0, nk_cap = 0;
    int nrhs_cap = 0, nchunk_cap = 0;
    double* x = nullptr;
    double* y = nullptr;
    int* ja = nullptr;
    int* info = nullptr;
    int* fb = nullptr;
    double* vals[kMaxRhs] = {};
    DevCounters* ctrs = nullptr;
    cudaStream_t sc = nullptr, sc2 = nullptr, sd = nullptr;
    std::vector<cudaEvent_t> ev;
    cudaEvent_t t0 = nullptr, t1 = nullptr, kdone = nullptr;
};

Pipe* pipe_of(rbfb_ctx* ctx) {
    if (!ctx->pipe) ctx->pipe = new Pipe();
    return static_cast<Pipe*>(ctx->pipe);
}

int grow(rbfb_ctx* ctx, Pipe* p, size_t n, size_t nk, int nrhs, int nchunk) {
    if (!p->sc) {
        RBFB_CUDA(ctx, cudaStreamCreateWithFlags(&p->sc, cudaStreamNonBlocking));
        RBFB_CUDA(ctx, cudaStreamCreateWithFlags(&p->sc2, cudaStreamNonBlocking));
        RBFB_CUDA(ctx, cudaStreamCreateWithFlags(&p->sd, cudaStreamNonBlocking));
        RBFB_CUDA(ctx, cudaEventCreate(&p->t0));
        RBFB_CUDA(ctx, cudaEventCreate(&p->t1));
        RBFB_CUDA(ctx, cudaEventCreateWithFlags(&p->kdone, cudaEventDisableTiming));
    }
    if (p->n_cap < n) {
        cudaFree(p->x); cudaFree(p->y); cudaFree(p->info); cudaFree(p->fb);
        p->x = p->y = nullptr; p->info = p->fb = nullptr; p->n_cap = 0;
        RBFB_CUDA(ctx, cudaMalloc(&p->x, n * sizeof(double)));
        RBFB_CUDA(ctx, cudaMalloc(&p->y, n * sizeof(double)));
        RBFB_CUDA(ctx, cudaMalloc(&p->info, n * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&p->fb, n * sizeof(int)));
        p->n_cap = n;
    }
    if (p->nk_cap < nk || p->nrhs_cap < nrhs) {
        cudaFree(p->ja);
        p->ja = nullptr;
        for (auto& v : p->vals) { cudaFree(v); v = nullptr; }
        p->nk_cap = 0;
        p->nrhs_cap = 0;
        RBFB_CUDA(ctx, cudaMalloc(&p->ja, nk * sizeof(int)));
        for (int q = 0; q < nrhs; ++q) RBFB_CUDA(ctx, cudaMalloc(&p->vals[q], nk * sizeof(double)));
        p->nk_cap = nk;
        p->nrhs_cap = nrhs;
    }
    if (p->nchunk_cap < nchunk) {
        cudaFree(p->ctrs);
        p->ctrs = nullptr;
        RBFB_CUDA(ctx, cudaMalloc(&p->ctrs, nchunk * sizeof(DevCounters)));
        for (auto e : p->ev) cudaEventDestroy(e);
        p->ev.assign(nchunk, nullptr);
        for (auto& e : p->ev) RBFB_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        p->nchunk_cap = nchunk;
    }
    return RBFB_OK;
}

}  // namespace
}  // namespace rbfb

using namespace rbfb;

extern "C" {

void rbfb_release_pipeline(rbfb_ctx* ctx) {
    auto* p = static_cast<Pipe*>(ctx->pipe);
    if (!p) return;
    cudaFree(p->x); cudaFree(p->y); cudaFree(p->ja); cudaFree(p->info); cudaFree(p->fb);
    for (auto v : p->vals) cudaFree(v);
    cudaFree(p->ctrs);
    for (auto e : p->ev) cudaEventDestroy(e);
    if (p->t0) cudaEventDestroy(p->t0);
    if (p->t1) cudaEventDestroy(p->t1);
    if (p->kdone) cudaEventDestroy(p->kdone);
    if (p->sc) cudaStreamDestroy(p->sc);
    if (p->sc2) cudaStreamDestroy(p->sc2);
    if (p->sd) cudaStreamDestroy(p->sd);
    delete p;
    ctx->pipe = nullptr;
}

int rbfb_assemble_host(rbfb_ctx* ctx, const rbfb_desc* desc, int n, const double* x_h,
                       const double* y_h, int k, const int* ja_h, int* ja_out_h,
                       double* const* values_h, int* info_h, rbfb_stats* stats) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int rc = check_desc(ctx, desc);
    if (rc) return rc;
    if (n < 1 || k < 1 || k > n || !x_h || !y_h || !values_h)
        return fail(ctx, RBFB_EINVAL, "need n >= 1, 1 <= k <= n and host arrays");
    AsmParams probe;
    std::memset(&probe, 0, sizeof(probe));
    const int nrhs = rhs_columns(desc, probe);
    if (nrhs < 0) return fail(ctx, nrhs, "bad operator mask");
    for (int q = 0; q < nrhs; ++q)
        if (!values_h[q]) return fail(ctx, RBFB_EINVAL, "null host values pointer");
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t nk = static_cast<size_t>(n) * k;
    const int chunk = std::max(16384, (n + 63) / 64);
    const int nchunk = (n + chunk - 1) / chunk;
    Pipe* p = pipe_of(ctx);
    rc = grow(ctx, p, n, nk, nrhs, nchunk);
    if (rc) return rc;
    cudaStream_t sc = p->sc, sc2 = p->sc2, sd = p->sd;
    RBFB_CUDA(ctx, cudaEventRecord(p->t0, sc));
    RBFB_CUDA(ctx, cudaMemcpyAsync(p->x, x_h, n * sizeof(double), cudaMemcpyHostToDevice, sc));
    RBFB_CUDA(ctx, cudaMemcpyAsync(p->y, y_h, n * sizeof(double), cudaMemcpyHostToDevice, sc));
    if (ja_h) {
        RBFB_CUDA(ctx, cudaMemcpyAsync(p->ja, ja_h, nk * sizeof(int), cudaMemcpyHostToDevice, sc));
    } else {
        const double per[2] = {desc->period[0], desc->period[1]};
        const bool periodic = per[0] > 0 && per[1] > 0;
        rc = knn::build(ctx, n, p->x, p->y, periodic ? per : nullptr, sc);
        if (rc < 0) return rc;
        rc = knn::query(ctx, n, nullptr, nullptr, k, p->ja, sc);
        if (rc) return rc;
    }
    if (ja_out_h) {
        RBFB_CUDA(ctx, cudaEventRecord(p->kdone, sc));
        RBFB_CUDA(ctx, cudaStreamWaitEvent(sd, p->kdone, 0));
        RBFB_CUDA(ctx, cudaMemcpyAsync(ja_out_h, p->ja, nk * sizeof(int), cudaMemcpyDeviceToHost, sd));
    }
    RBFB_CUDA(ctx, cudaMemsetAsync(p->ctrs, 0, nchunk * sizeof(DevCounters), sc));
    // the second compute stream starts after the stencils and counters
    RBFB_CUDA(ctx, cudaEventRecord(p->kdone, sc));
    RBFB_CUDA(ctx, cudaStreamWaitEvent(sc2, p->kdone, 0));
    for (int c = 0; c < nchunk; ++c) {
        const int c0 = c * chunk, cnt = std::min(chunk, n - c0);
        cudaStream_t s = (c & 1) ? sc2 : sc;
        rc = enqueue_fixed(ctx, desc, c0, cnt, p->x, p->y, k, p->ja, p->vals, p->info,
                           p->ctrs + c, p->fb + c0, s);
        if (rc) return rc;
        RBFB_CUDA(ctx, cudaEventRecord(p->ev[c], s));
        RBFB_CUDA(ctx, cudaStreamWaitEvent(sd, p->ev[c], 0));
        const size_t o = static_cast<size_t>(c0) * k, len = static_cast<size_t>(cnt) * k;
        for (int q = 0; q < nrhs; ++q)
            RBFB_CUDA(ctx, cudaMemcpyAsync(values_h[q] + o, p->vals[q] + o, len * sizeof(double),
                                           cudaMemcpyDeviceToHost, sd));
        if (info_h)
            RBFB_CUDA(ctx, cudaMemcpyAsync(info_h + c0, p->info + c0, cnt * sizeof(int),
                                           cudaMemcpyDeviceToHost, sd));
    }
    // both compute streams done: singular count on the device, then the
    // counters of every chunk
    RBFB_CUDA(ctx, cudaEventRecord(p->kdone, sc2));
    RBFB_CUDA(ctx, cudaStreamWaitEvent(sc, p->kdone, 0));
    rc = count_singular(ctx, p->info, n, &p->ctrs[0].singular, sc);
    if (rc) return rc;
    std::vector<DevCounters> h(nchunk);
    RBFB_CUDA(ctx, cudaMemcpyAsync(h.data(), p->ctrs, nchunk * sizeof(DevCounters),
                                   cudaMemcpyDeviceToHost, sc));
    RBFB_CUDA(ctx, cudaEventRecord(p->kdone, sd));
    RBFB_CUDA(ctx, cudaStreamWaitEvent(sc, p->kdone, 0));
    RBFB_CUDA(ctx, cudaEventRecord(p->t1, sc));
    RBFB_CUDA(ctx, cudaStreamSynchronize(sc));
    long long singular = static_cast<long long>(h[0].singular);
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p->t0, p->t1);
        std::memset(stats, 0, sizeof(*stats));
        stats->stencils = n;
        stats->singular = singular;
        for (const auto& c : h) {
            stats->fallback += c.fb_count;
            stats->sweeps += static_cast<long long>(c.sweeps_sum);
            stats->max_sweeps_used = std::max(stats->max_sweeps_used, c.sweeps_max);
        }
        stats->buckets = 1;
        stats->ms = ms;
    }
    return static_cast<int>(std::min<long long>(singular, 0x7fffffff));
}

}  // extern "C"
