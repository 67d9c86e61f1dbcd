// serve.cu -- continuous-batching assembly server (rbfb_server_*).
//
// Requests (node sets of any size, with k and an operator descriptor) are
// queued at submit. A worker thread admits them into free slots, first fit
// in arrival order, as long as the device memory held by admitted requests
// stays within the HBM budget. Each slot owns a stream and its own rbfb_ctx
// (its own k-NN and fallback workspace), so admitted requests run their
// k-NN search and assembly concurrently on the device and never share
// scratch. Buffers come from the stream-ordered allocator (cudaMallocAsync)
// on the slot's stream; completion is signalled by a host callback on that
// stream, which frees the slot at once. Nodes, stencils and weights stay
// resident on the device until rbfb_server_release, and count against the
// budget until then. A request is assembled by exactly the same kernels as
// rbfb_assemble, so its result does not depend on what runs beside it.
//
// No reference counterpart (the reference has no serving path).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "runtime.h"

namespace {

using Clock = std::chrono::steady_clock;

enum class State { Queued, Running, Done, Failed };

struct Slot;

struct Req {
    long long ticket = 0;
    int n = 0, k = 0, nrhs = 0;
    rbfb_desc desc{};
    double* xh = nullptr;  // pinned host copies of the nodes (from the server's cache)
    double* yh = nullptr;
    size_t xh_cap = 0, yh_cap = 0;
    State state = State::Queued;
    int status = RBFB_OK;
    size_t bytes = 0;
    // device, resident until release
    double* x = nullptr;
    double* y = nullptr;
    int* ja = nullptr;
    int* info = nullptr;
    double* vals[RBFB_MAX_RHS] = {};
    rbfb::DevCounters* ctr = nullptr;
    int* fb = nullptr;
    unsigned long long* sing = nullptr;
    long long singular = 0, fallback = 0;
    bool counted = false;
    double t_submit = 0, t_start = 0, t_end = 0;
    // device clock: events around the request's work on its stream, read
    // against the server's origin event once the request is done
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double dev_start = -1.0, dev_end = -1.0;
    Slot* slot = nullptr;
    cudaStream_t stream = nullptr;
};

struct Slot {
    rbfb_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    Req* busy = nullptr;
};

}  // namespace

struct rbfb_server {
    int device = 0;
    size_t budget = 0;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv;       // worker wake-ups
    std::condition_variable done_cv;  // poll waiters
    std::thread worker;
    bool stop = false;
    long long next = 1;
    size_t resident = 0;
    std::map<long long, std::unique_ptr<Req>> reqs;
    std::deque<long long> queue;
    Clock::time_point t0 = Clock::now();
    cudaStream_t io = nullptr;  // fetch copies
    cudaEvent_t origin = nullptr;  // device-clock origin of the requests' timings
    // Pinned staging buffers for submitted node sets, reused: page-locking
    // and unlocking host memory per request costs milliseconds (and
    // unlocking may wait for the device). Blocks are never returned to the
    // system before destroy. Own mutex, taken by the completion callback;
    // like the server mutex it is never held across a CUDA call.
    std::mutex pin_mu;
    std::multimap<size_t, void*> pin_free;  // capacity -> block
    std::vector<void*> pin_all;
    double now_ms() const {
        return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    }
};

namespace {

size_t request_bytes(int n, int k, int nrhs) {
    const size_t nk = static_cast<size_t>(n) * k;
    return 16 * static_cast<size_t>(n) + 4 * nk + 8 * nk * nrhs + 8 * static_cast<size_t>(n) +
           sizeof(rbfb::DevCounters) + 1024;
}

// A pinned block of at least `bytes` (capacity in *cap), or nullptr. The
// cache mutex is never held across the CUDA call: a completion callback
// (pin_release) may run meanwhile, and the CUDA call may wait for it.
void* pin_acquire(rbfb_server* s, size_t bytes, size_t* cap) {
    {
        std::lock_guard<std::mutex> l(s->pin_mu);
        auto it = s->pin_free.lower_bound(bytes);
        if (it != s->pin_free.end() && it->first <= 4 * bytes + (1u << 20)) {
            void* p = it->second;
            *cap = it->first;
            s->pin_free.erase(it);
            return p;
        }
    }
    size_t c = 1u << 16;
    while (c < bytes) c <<= 1;
    void* p = nullptr;
    if (cudaHostAlloc(&p, c, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    {
        std::lock_guard<std::mutex> l(s->pin_mu);
        s->pin_all.push_back(p);
    }
    *cap = c;
    return p;
}
// Back to the cache (no CUDA call: allowed in a stream callback).
void pin_release(rbfb_server* s, void* p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> l(s->pin_mu);
    s->pin_free.emplace(cap, p);
}

struct CallbackArg {
    rbfb_server* srv;
    Req* req;
};

void CUDART_CB on_done(void* p) {
    auto* a = static_cast<CallbackArg*>(p);
    // the node copies ran before the kernels on this stream: staging is free
    pin_release(a->srv, a->req->xh, a->req->xh_cap);
    pin_release(a->srv, a->req->yh, a->req->yh_cap);
    a->req->xh = a->req->yh = nullptr;
    {
        std::lock_guard<std::mutex> l(a->srv->mu);
        a->req->t_end = a->srv->now_ms();
        if (a->req->state == State::Running) a->req->state = State::Done;
        if (a->req->slot) a->req->slot->busy = nullptr;
        a->req->slot = nullptr;
    }
    a->srv->cv.notify_all();
    a->srv->done_cv.notify_all();
    delete a;
}

// Enqueue one admitted request on its slot (the worker, without the lock).
int launch(rbfb_server* s, Slot& sl, Req* r) {
    cudaStream_t st = sl.stream;
    r->stream = st;
    const size_t n = r->n, nk = n * r->k;
    auto alloc = [&](void** p, size_t b) { return cudaMallocAsync(p, b, st); };
    cudaError_t e = cudaSuccess;
    e = e ? e : alloc(reinterpret_cast<void**>(&r->x), n * 8);
    e = e ? e : alloc(reinterpret_cast<void**>(&r->y), n * 8);
    e = e ? e : alloc(reinterpret_cast<void**>(&r->ja), nk * 4);
    e = e ? e : alloc(reinterpret_cast<void**>(&r->info), n * 4);
    e = e ? e : alloc(reinterpret_cast<void**>(&r->fb), n * 4);
    e = e ? e : alloc(reinterpret_cast<void**>(&r->ctr), sizeof(rbfb::DevCounters));
    for (int q = 0; q < r->nrhs && !e; ++q) e = alloc(reinterpret_cast<void**>(&r->vals[q]), nk * 8);
    if (e) return RBFB_ENOMEM;
    e = cudaMemcpyAsync(r->x, r->xh, n * 8, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync(r->y, r->yh, n * 8, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemsetAsync(r->ctr, 0, sizeof(rbfb::DevCounters), st);
    e = e ? e : cudaEventCreate(&r->ev0);
    e = e ? e : cudaEventCreate(&r->ev1);
    e = e ? e : cudaEventRecord(r->ev0, st);  // the request's kernels start after this point
    if (e) return RBFB_ECUDA;
    rbfb_ctx* ctx = sl.ctx;
    const double per[2] = {r->desc.period[0], r->desc.period[1]};
    const bool periodic = per[0] > 0 && per[1] > 0;
    int rc;
    {
        std::lock_guard<std::mutex> cl(ctx->mu);
        rc = rbfb::knn::build(ctx, r->n, r->x, r->y, periodic ? per : nullptr, st);
        if (rc >= 0) rc = rbfb::knn::query(ctx, r->n, nullptr, nullptr, r->k, r->ja, st);
        if (rc >= 0)
            rc = rbfb::enqueue_fixed(ctx, &r->desc, 0, r->n, r->x, r->y, r->k, r->ja, r->vals,
                                     r->info, r->ctr, r->fb, st);
        if (rc >= 0) rc = rbfb::count_singular(ctx, r->info, r->n, &r->ctr->singular, st);
    }
    if (rc < 0) return rc;
    e = cudaEventRecord(r->ev1, st);
    e = e ? e : cudaLaunchHostFunc(st, on_done, new CallbackArg{s, r});
    return e ? RBFB_ECUDA : RBFB_OK;
}

// The worker admits one request at a time under the lock, then launches it
// with the lock released: no thread holds the server lock across a CUDA
// call, so the completion callback (which takes the lock) can never wait on
// a thread that waits on CUDA.
void worker_loop(rbfb_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        Req* r = nullptr;
        Slot* slot = nullptr;
        {
            std::unique_lock<std::mutex> l(s->mu);
            if (s->stop) return;
            for (auto& sl : s->slots)
                if (!sl.busy) {
                    slot = &sl;
                    break;
                }
            if (slot) {
                for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
                    Req* c = s->reqs[*it].get();
                    if (s->resident + c->bytes > s->budget) continue;  // first fit
                    r = c;
                    s->resident += c->bytes;
                    s->queue.erase(it);
                    r->state = State::Running;
                    r->slot = slot;
                    slot->busy = r;
                    r->t_start = s->now_ms();
                    break;
                }
            }
            if (!r) {
                s->cv.wait_for(l, std::chrono::milliseconds(1));
                continue;
            }
        }
        const int rc = launch(s, *slot, r);
        if (rc != RBFB_OK) {
            {
                std::lock_guard<std::mutex> l(s->mu);
                r->status = rc;
                r->state = State::Failed;
                slot->busy = nullptr;
                r->slot = nullptr;
            }
            s->done_cv.notify_all();
        }
    }
}

void free_request(rbfb_server* s, Req* r) {
    cudaStream_t st = r->stream;
    auto fr = [&](void* p) {
        if (p) cudaFreeAsync(p, st);
    };
    fr(r->x); fr(r->y); fr(r->ja); fr(r->info); fr(r->fb); fr(r->ctr);
    for (auto& v : r->vals) fr(v);
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    r->ev0 = r->ev1 = nullptr;
    // staging of a request that never completed (failed or never launched)
    pin_release(s, r->xh, r->xh_cap);
    pin_release(s, r->yh, r->yh_cap);
    r->xh = r->yh = nullptr;
}

}  // namespace

extern "C" {

int rbfb_server_create(rbfb_server** out, int device, size_t budget, int max_slots) {
    if (!out || max_slots < 1 || budget == 0) return RBFB_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return RBFB_ECUDA;
    auto* s = new rbfb_server();
    s->device = device;
    s->budget = budget;
    s->slots.resize(max_slots);
    for (auto& sl : s->slots) {
        if (rbfb_create(&sl.ctx, device) != RBFB_OK ||
            cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess) {
            for (auto& t : s->slots) {
                if (t.ctx) rbfb_destroy(t.ctx);
                if (t.stream) cudaStreamDestroy(t.stream);
            }
            delete s;
            return RBFB_ECUDA;
        }
    }
    cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking);
    if (cudaEventCreate(&s->origin) != cudaSuccess || cudaEventRecord(s->origin, s->io) != cudaSuccess ||
        cudaEventSynchronize(s->origin) != cudaSuccess) {
        for (auto& t : s->slots) {
            rbfb_destroy(t.ctx);
            cudaStreamDestroy(t.stream);
        }
        delete s;
        return RBFB_ECUDA;
    }
    // Requests allocate from the device's default stream-ordered pool; let it
    // keep up to the budget cached between requests instead of handing memory
    // back to the driver at every synchronisation (an attribute of this
    // process's pool, not a setting of the GPU).
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return RBFB_OK;
}

int rbfb_server_submit(rbfb_server* s, const rbfb_request* req, long long* ticket) {
    if (!s || !req || !ticket || !req->x_h || !req->y_h) return RBFB_EINVAL;
    if (req->n < 1 || req->k < 1 || req->k > req->n) return RBFB_EINVAL;
    rbfb_desc d = req->desc;
    if (d.ops & RBFB_OP_INTERP) return RBFB_EUNSUPPORTED;  // interpolation points are per call
    rbfb::AsmParams probe;
    std::memset(&probe, 0, sizeof(probe));
    const int nrhs = rbfb::rhs_columns(&d, probe);
    if (nrhs < 0) return nrhs;
    // shape check up front: a request no kernel serves is refused at submit
    const int P = d.degree, Q = d.phs ? d.phs : 2 * P - 1;
    if (rbfb::pick_variant(nullptr, d.precision == RBFB_FP32_IR, P, Q, req->k + rbfb::npoly(P)) < 0)
        return RBFB_EUNSUPPORTED;
    auto r = std::make_unique<Req>();
    r->n = req->n;
    r->k = req->k;
    r->nrhs = nrhs;
    r->desc = d;
    r->bytes = request_bytes(req->n, req->k, nrhs);
    if (r->bytes > s->budget) return RBFB_EBUDGET;
    r->xh = static_cast<double*>(pin_acquire(s, r->n * 8, &r->xh_cap));
    r->yh = static_cast<double*>(pin_acquire(s, r->n * 8, &r->yh_cap));
    if (!r->xh || !r->yh) {
        pin_release(s, r->xh, r->xh_cap);
        pin_release(s, r->yh, r->yh_cap);
        return RBFB_ENOMEM;
    }
    std::memcpy(r->xh, req->x_h, r->n * 8);
    std::memcpy(r->yh, req->y_h, r->n * 8);
    {
        std::lock_guard<std::mutex> l(s->mu);
        r->ticket = s->next++;
        r->t_submit = s->now_ms();
        *ticket = r->ticket;
        s->queue.push_back(r->ticket);
        s->reqs[r->ticket] = std::move(r);
    }
    s->cv.notify_all();
    return RBFB_OK;
}

int rbfb_server_poll(rbfb_server* s, long long ticket, int wait_ms, rbfb_result* res) {
    if (!s) return RBFB_EINVAL;
    Req* r = nullptr;
    {
        std::unique_lock<std::mutex> l(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return RBFB_ENOTFOUND;
        r = it->second.get();
        auto finished = [&] { return r->state == State::Done || r->state == State::Failed; };
        if (!finished()) {
            if (wait_ms == 0) return RBFB_EBUSY;
            if (wait_ms < 0) s->done_cv.wait(l, finished);
            else if (!s->done_cv.wait_for(l, std::chrono::milliseconds(wait_ms), finished))
                return RBFB_ETIMEOUT;
        }
    }
    // the request's stream has finished: its counters are final (read once,
    // without the lock)
    if (r->state == State::Done && !r->counted && r->ctr) {
        rbfb::DevCounters h{};
        float a = -1.f, b = -1.f;
        if (r->ev0 && r->ev1) {
            if (cudaEventElapsedTime(&a, s->origin, r->ev0) != cudaSuccess) a = -1.f;
            if (cudaEventElapsedTime(&b, s->origin, r->ev1) != cudaSuccess) b = -1.f;
        }
        if (cudaMemcpy(&h, r->ctr, sizeof(h), cudaMemcpyDeviceToHost) == cudaSuccess) {
            std::lock_guard<std::mutex> l(s->mu);
            r->singular = static_cast<long long>(h.singular);
            r->fallback = h.fb_count;
            r->dev_start = a;
            r->dev_end = b;
            r->counted = true;
        }
    }
    std::lock_guard<std::mutex> l(s->mu);
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->status = r->state == State::Failed ? r->status : RBFB_OK;
        res->n = r->n;
        res->k = r->k;
        res->nrhs = r->nrhs;
        res->singular = r->singular;
        res->fallback = r->fallback;
        res->ja = r->ja;
        for (int q = 0; q < r->nrhs; ++q) res->values[q] = r->vals[q];
        res->submit_ms = r->t_submit;
        res->start_ms = r->t_start;
        res->end_ms = r->t_end;
        res->dev_start_ms = r->dev_start;
        res->dev_end_ms = r->dev_end;
    }
    return r->state == State::Failed ? r->status : RBFB_OK;
}

int rbfb_server_fetch(rbfb_server* s, long long ticket, int* ja_h, double* const* values_h) {
    if (!s || !values_h) return RBFB_EINVAL;
    Req* r = nullptr;
    {
        std::lock_guard<std::mutex> l(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return RBFB_ENOTFOUND;
        r = it->second.get();
        if (r->state != State::Done) return r->state == State::Failed ? r->status : RBFB_EBUSY;
    }
    const size_t nk = static_cast<size_t>(r->n) * r->k;
    cudaSetDevice(s->device);
    for (int q = 0; q < r->nrhs; ++q)
        if (cudaMemcpyAsync(values_h[q], r->vals[q], nk * 8, cudaMemcpyDeviceToHost, s->io))
            return RBFB_ECUDA;
    if (ja_h && cudaMemcpyAsync(ja_h, r->ja, nk * 4, cudaMemcpyDeviceToHost, s->io))
        return RBFB_ECUDA;
    return cudaStreamSynchronize(s->io) == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

int rbfb_server_release(rbfb_server* s, long long ticket) {
    if (!s) return RBFB_EINVAL;
    std::unique_ptr<Req> r;
    {
        std::lock_guard<std::mutex> l(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return RBFB_ENOTFOUND;
        if (it->second->state == State::Running || it->second->state == State::Queued)
            return RBFB_EBUSY;
        r = std::move(it->second);
        s->reqs.erase(it);
        s->resident -= std::min(s->resident, r->bytes);
    }
    cudaSetDevice(s->device);
    free_request(s, r.get());
    s->cv.notify_all();
    return RBFB_OK;
}

size_t rbfb_server_resident_bytes(const rbfb_server* s) {
    if (!s) return 0;
    auto* m = const_cast<rbfb_server*>(s);
    std::lock_guard<std::mutex> l(m->mu);
    return m->resident;
}

int rbfb_server_destroy(rbfb_server* s) {
    if (!s) return RBFB_OK;
    {
        std::lock_guard<std::mutex> l(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    for (auto& sl : s->slots) cudaStreamSynchronize(sl.stream);
    for (auto& kv : s->reqs) free_request(s, kv.second.get());
    for (auto& sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
        rbfb_destroy(sl.ctx);
    }
    if (s->io) cudaStreamDestroy(s->io);
    if (s->origin) cudaEventDestroy(s->origin);
    for (void* p : s->pin_all) cudaFreeHost(p);
    delete s;
    return RBFB_OK;
}

}  // extern "C"
