// runtime.h -- internal state behind the C ABI: the context (workspace,
// launch table, counters) and the helpers the entry points share.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "rbf_b200.h"
#include "asm_kernel.cuh"
#include "asm_variants.h"

namespace rbfb {

// Device counters of one assembly call.
struct DevCounters {
    int fb_count;      // stencils queued for the FP64 kernel
    int sweeps_max;    // largest refinement sweep count
    int work[2];       // dynamic work counters (mixed, fallback)
    unsigned long long sweeps_sum;
    unsigned long long singular;
};

struct LaunchShape {
    int variant = -1;
    int blocks_per_sm = 0;  // 0 = occupancy maximum
};

}  // namespace rbfb

struct rbfb_ctx {
    int device = 0;
    int sms = 0;
    std::string err;
    std::atomic<long long> launches{0};
    std::mutex mu;
    // scratch owned by the context
    int* fb_list = nullptr;
    size_t fb_cap = 0;
    rbfb::DevCounters* ctr = nullptr;
    // occupancy of each compiled variant (blocks per SM), lazily queried
    std::vector<int> occ;
    // tuned launch table: (mixed, P, Q, ntp) -> shape
    std::map<std::tuple<int, int, int, int>, rbfb::LaunchShape> tuned;
    // k-NN workspace
    void* knn_ws = nullptr;
    size_t knn_ws_bytes = 0;
    // CSR batching state (batch.cu)
    void* batch = nullptr;
    // host-pipeline staging (pinned) and device buffers
    void* pipe = nullptr;
    // iterative-solve workspace and its replay graph (solve.cu)
    void* solve = nullptr;
};

namespace rbfb {

// error helpers: record a message in the context and return the code
int fail(rbfb_ctx* ctx, int code, const std::string& msg);
int cuda_fail(rbfb_ctx* ctx, cudaError_t e, const char* where);
#define RBFB_CUDA(ctx, call)                                        \
    do {                                                            \
        cudaError_t e__ = (call);                                   \
        if (e__ != cudaSuccess) return ::rbfb::cuda_fail(ctx, e__, #call); \
    } while (0)

// Fills col_op / col_ic of params from the descriptor; returns nrhs or < 0.
int rhs_columns(const rbfb_desc* d, AsmParams& p);

// Variant for (mixed, P, Q) that fits a system of n unknowns with nrhs
// right-hand sides, honouring the tuned table; -1 when none is compiled.
int pick_variant(rbfb_ctx* ctx, bool mixed, int P, int Q, int n, int nrhs = 1);

// Persistent grid size of a variant (blocks), after the shared-memory opt-in.
int grid_for(rbfb_ctx* ctx, int v, int blocks_per_sm_override = 0);

// Launch a variant over p (grid: persistent). Counts the launch.
int launch_variant(rbfb_ctx* ctx, int v, const AsmParams& p, cudaStream_t st, int blocks = 0);

// Ensure the fallback list holds n entries.
int ensure_fb(rbfb_ctx* ctx, size_t n);

// Count nonzero entries of info into *out (one kernel launch).
int count_singular(rbfb_ctx* ctx, const int* info, int n, unsigned long long* out, cudaStream_t st);

// Fixed-width assembly of stencils [first, first + count) on `st` with the
// counters `ctr` and the fallback region fb (count entries). No sync.
// values: host table of device pointers, or nullptr when values_d (a table in
// device memory) is given.
int enqueue_fixed(rbfb_ctx* ctx, const rbfb_desc* desc, int first, int count, const double* x,
                  const double* y, int k, const int* ja, double* const* values, int* info,
                  DevCounters* ctr, int* fb, cudaStream_t st, int row_base = 0,
                  double* const* values_d = nullptr);

int check_desc(rbfb_ctx* ctx, const rbfb_desc* d);

namespace knn {
// Bins the nodes (returns the number of cells or < 0), then answers queries
// (xq == nullptr: the nodes themselves). Both enqueue on `st`, no sync.
int build(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* period,
          cudaStream_t st);
int query(rbfb_ctx* ctx, int nq, const double* xq, const double* yq, int k, int* ja,
          cudaStream_t st);
}  // namespace knn

}  // namespace rbfb
