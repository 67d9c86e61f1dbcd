// knn.cu -- k-nearest-neighbour stencils on a uniform cell grid (sm_100a).
//
// Replaces the reference's tree searches: NodeSet::stencils(k) over a
// nanoflann k-d tree in the open plane (src/rbf_nodeset.h:155-181) and
// KdTree::knn_stencils(k) over SciPy's ckdtree in a periodic box
// (src/rbf_spatial.cpp:193-260). A tree walk is pointer chasing; on the GPU
// the nodes are binned instead:
//
//   1. bounding box (open plane, device reduction) or the box [0,L)^2;
//   2. cell of every node on a C x C grid (about kPerCell nodes per cell),
//      counting sort by cell: cell_start[] and the nodes' coordinates and
//      indices in cell order (coalesced candidate reads);
//   3. one warp per query, queries in cell order: walk the nodes of the
//      (2R+1)^2 cells around the query's cell (their runs of cells laid out
//      flat over the lanes) and keep, in shared memory with their squared
//      distances, those closer than the distance from the query to the edge
//      of the searched block. If at least k are kept, the k nearest nodes
//      are among them: rank them by (squared distance, index) and write the
//      k smallest. Otherwise R grows and the warp searches again. More
//      candidates than the buffer holds are merged chunk by chunk.
//
// Distances use the reference's arithmetic exactly: dx*dx + dy*dy of the
// plain differences, each operation rounded (nanoflann L2_Simple_Adaptor,
// nanoflann.hpp:690-699), and in a periodic box of ckdtree's wrapped
// differences (wrap_distance, ckdtree/src/distance.h:262-272) with both
// the nodes and the queries folded into [0, L) first (rbf_spatial.h:39-48,
// ckdtree wrap_position). Neighbours are ordered by (squared distance,
// index), which equals the reference's order wherever no two candidates tie.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "asm_math.cuh"
#include "runtime.h"

namespace rbfb {
namespace knn {

constexpr int kPerCell = 2;   // target nodes per cell
constexpr int kCap = 256;     // candidate buffer per warp (entries)
constexpr int kWarps = 4;     // warps per CTA in the query kernel
constexpr int kMaxK = 128;

struct Grid {
    double x0, y0;     // origin of the cell grid
    double hx, hy;     // cell sides
    int cx, cy;        // cells per axis
    double Lx, Ly;     // periods (> 0) or 0
};

// detail::fold of the reference (src/rbf_spatial.h:39-48), rounded per op.
__device__ __forceinline__ double fold(double x, double L) {
    if (!(L > 0.0)) return x;
    x = dsub(x, dmul(L, floor(ddiv(x, L))));
    while (x >= L) x = dsub(x, L);
    while (x < 0.0) x = dadd(x, L);
    return x;
}

// ckdtree wrap_distance.
__device__ __forceinline__ double wrap_d(double d, double L) {
    if (!(L > 0.0)) return d;
    const double hb = 0.5 * L;
    if (d < -hb) return dadd(L, d);
    if (d > hb) return dsub(d, L);
    return d;
}

__device__ __forceinline__ double sqdist(double qx, double qy, double px, double py, double Lx,
                                         double Ly) {
    const double dx = wrap_d(dsub(qx, px), Lx);
    const double dy = wrap_d(dsub(qy, py), Ly);
    return dadd(dmul(dx, dx), dmul(dy, dy));
}

__device__ __forceinline__ int cell_coord(double v, double o, double h, int c) {
    int i = static_cast<int>(floor((v - o) / h));
    return i < 0 ? 0 : (i >= c ? c - 1 : i);
}

// ---- 1. bounding box ---------------------------------------------------------
__global__ void bbox_kernel(const double* x, const double* y, int n, double* out /*4*/) {
    double mnx = 1e308, mny = 1e308, mxx = -1e308, mxy = -1e308;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        mnx = fmin(mnx, x[i]);
        mxx = fmax(mxx, x[i]);
        mny = fmin(mny, y[i]);
        mxy = fmax(mxy, y[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mnx = fmin(mnx, __shfl_down_sync(0xffffffffu, mnx, o));
        mxx = fmax(mxx, __shfl_down_sync(0xffffffffu, mxx, o));
        mny = fmin(mny, __shfl_down_sync(0xffffffffu, mny, o));
        mxy = fmax(mxy, __shfl_down_sync(0xffffffffu, mxy, o));
    }
    if ((threadIdx.x & 31) == 0) {
        // order-preserving integer images of doubles for atomic min/max
        auto key = [](double v) {
            long long b = __double_as_longlong(v);
            return b >= 0 ? (unsigned long long)b | 0x8000000000000000ull
                          : ~(unsigned long long)b;
        };
        unsigned long long* o = reinterpret_cast<unsigned long long*>(out);
        atomicMin(o + 0, key(mnx));
        atomicMax(o + 1, key(mxx));
        atomicMin(o + 2, key(mny));
        atomicMax(o + 3, key(mxy));
    }
}

__device__ __forceinline__ double unkey(unsigned long long k) {
    return (k & 0x8000000000000000ull) ? __longlong_as_double((long long)(k & 0x7fffffffffffffffull))
                                       : __longlong_as_double((long long)~k);
}

__global__ void bbox_init_kernel(unsigned long long* bb) {
    bb[0] = ~0ull;
    bb[1] = 0ull;
    bb[2] = ~0ull;
    bb[3] = 0ull;
}

__global__ void set_grid_kernel(Grid g, Grid* out) { *out = g; }

// Turns the bbox keys into the grid geometry (one thread).
__global__ void grid_kernel(const unsigned long long* bb, int cx, int cy, Grid* g) {
    const double xmin = unkey(bb[0]), xmax = unkey(bb[1]);
    const double ymin = unkey(bb[2]), ymax = unkey(bb[3]);
    double wx = xmax - xmin, wy = ymax - ymin;
    if (!(wx > 0)) wx = 1.0;
    if (!(wy > 0)) wy = 1.0;
    g->x0 = xmin;
    g->y0 = ymin;
    g->hx = wx / cx * (1.0 + 1e-12);
    g->hy = wy / cy * (1.0 + 1e-12);
    g->cx = cx;
    g->cy = cy;
    g->Lx = 0.0;
    g->Ly = 0.0;
}

// ---- 2. binning ----------------------------------------------------------------
__global__ void cell_count_kernel(const double* x, const double* y, int n, const Grid* gp,
                                  int* cell_of, int* count, double* fx, double* fy) {
    const Grid g = *gp;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double px = fold(x[i], g.Lx), py = fold(y[i], g.Ly);
        fx[i] = px;
        fy[i] = py;
        const int c = cell_coord(py, g.y0, g.hy, g.cy) * g.cx + cell_coord(px, g.x0, g.hx, g.cx);
        cell_of[i] = c;
        atomicAdd(count + c, 1);
    }
}

// exclusive scan, three phases: per-block totals, scan of totals, add
constexpr int kScanBlock = 1024;
__global__ void scan_block_kernel(const int* in, int* out, int n, int* block_sums) {
    __shared__ int warp_sums[32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int v = i < n ? in[i] : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int s = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += t;
    }
    if (lane == 31) warp_sums[w] = s;
    __syncthreads();
    if (w == 0) {
        int ws = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += t;
        }
        warp_sums[lane] = ws;
    }
    __syncthreads();
    const int excl = s - v + (w > 0 ? warp_sums[w - 1] : 0);
    if (i < n) out[i] = excl;
    if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = excl + v;
}
__global__ void scan_sums_kernel(int* sums, int nb, int* total) {
    // single thread: nb is small (cells / 1024)
    int acc = 0;
    for (int b = 0; b < nb; ++b) {
        const int t = sums[b];
        sums[b] = acc;
        acc += t;
    }
    *total = acc;
}
__global__ void scan_add_kernel(int* out, int n, const int* sums) {
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

__global__ void scatter_kernel(const int* cell_of, int n, const int* start, int* cursor,
                               const double* fx, const double* fy, int* sidx, double* sx,
                               double* sy) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = cell_of[i];
        const int pos = start[c] + atomicAdd(cursor + c, 1);
        sidx[pos] = i;
        sx[pos] = fx[i];
        sy[pos] = fy[i];
    }
}

// ---- 3. queries --------------------------------------------------------------------
struct QueryArgs {
    const Grid* g;
    const int* start;  // cells + 1 entries
    const int* sidx;
    const double* sx;
    const double* sy;
    int nq;
    const double* qx;  // query coordinates (folded); nullptr: the nodes themselves
    const double* qy;
    const int* qorder;  // query visiting order (cell order), or nullptr
    int k;
    int* ja;
    int* status;  // set to 1 when a query could not be completed
};

__device__ __forceinline__ bool key_less(unsigned long long da, int ia, unsigned long long db,
                                         int ib) {
    return da < db || (da == db && ia < ib);
}

// Bounded to 8 CTAs (32 warps) per SM: 64 registers and a few spilled bytes
// instead of 96 registers and about 20 warps; the search is issue-bound, and
// the extra warps fill the issue slots (2.75 -> 2.60 ms for 1M nodes, k = 35).
__global__ void __launch_bounds__(kWarps * 32, 8) query_kernel(QueryArgs a) {
    __shared__ unsigned long long sd[kWarps][kCap];
    __shared__ int si[kWarps][kCap];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* d = sd[w];
    int* id = si[w];
    const Grid g = *a.g;
    const int k = a.k;
    for (int t = blockIdx.x * kWarps + w; t < a.nq; t += gridDim.x * kWarps) {
        const int q = a.qorder ? a.qorder[t] : t;
        double qx, qy;
        if (a.qx) {
            qx = fold(a.qx[q], g.Lx);
            qy = fold(a.qy[q], g.Ly);
        } else {
            qx = a.sx[t];  // nodes in cell order: t-th sorted node is node q
            qy = a.sy[t];
        }
        const int ccx = cell_coord(qx, g.x0, g.hx, g.cx);
        const int ccy = cell_coord(qy, g.y0, g.hy, g.cy);
        int R = 1;
        // initial ring from the density
        {
            const double want = (k + 1.0) / kPerCell;
            R = max(1, (int)ceil(0.5 * (sqrt(want * 1.27) - 1.0)) + 1);
        }
        bool done = false;
        // First try a tighter radius than the block bound: the distance at
        // which k + 1 nodes are expected at the grid's mean density (kPerCell
        // per cell), with a 30% margin. Exactness does not depend on it: if
        // fewer than k nodes lie inside, the block is walked again with the
        // full bound.
        const double est2 = 1.69 * (k + 1) * g.hx * g.hy / (3.141592653589793 * kPerCell);
        bool tight = true;
        for (int attempt = 0; attempt < 64 && !done; ++attempt) {
            // periodic axes: never more than one period (no cell twice); open
            // axes: up to the whole grid (the clamp below keeps it in range)
            const int Rx = g.Lx > 0 ? min(R, (g.cx - 1) / 2 + 1) : min(R, g.cx);
            const int Ry = g.Ly > 0 ? min(R, (g.cy - 1) / 2 + 1) : min(R, g.cy);
            const bool fullx = g.Lx > 0 ? (2 * Rx + 1 >= g.cx) : false;
            const bool fully = g.Ly > 0 ? (2 * Ry + 1 >= g.cy) : false;
            // x/y cell ranges (periodic: wrapped, never more than the grid)
            int xlo = ccx - Rx, xhi = ccx + Rx, ylo = ccy - Ry, yhi = ccy + Ry;
            if (g.Lx > 0) {
                if (fullx) { xlo = 0; xhi = g.cx - 1; }
            } else {
                xlo = max(xlo, 0);
                xhi = min(xhi, g.cx - 1);
            }
            if (g.Ly > 0) {
                if (fully) { ylo = 0; yhi = g.cy - 1; }
            } else {
                ylo = max(ylo, 0);
                yhi = min(yhi, g.cy - 1);
            }
            // distance from the query to the edge of the searched block
            double bx = 1e300, by = 1e300;
            if (g.Lx > 0) {
                if (!fullx) bx = fmin(qx - (ccx - Rx) * g.hx, (ccx + Rx + 1) * g.hx - qx);
            } else {
                if (ccx - Rx > 0) bx = fmin(bx, qx - (g.x0 + (ccx - Rx) * g.hx));
                if (ccx + Rx < g.cx - 1) bx = fmin(bx, g.x0 + (ccx + Rx + 1) * g.hx - qx);
            }
            if (g.Ly > 0) {
                if (!fully) by = fmin(qy - (ccy - Ry) * g.hy, (ccy + Ry + 1) * g.hy - qy);
            } else {
                if (ccy - Ry > 0) by = fmin(by, qy - (g.y0 + (ccy - Ry) * g.hy));
                if (ccy + Ry < g.cy - 1) by = fmin(by, g.y0 + (ccy + Ry + 1) * g.hy - qy);
            }
            double bound = fmin(bx, by);
            bound = bound * (1.0 - 1e-9) - 1e-15 * fmax(fabs(qx), fabs(qy));
            // Only candidates inside a circle of radius at most `bound`
            // (inscribed in the searched block) are kept: when at least k of
            // them are found, the k nearest nodes are among them, since every
            // node outside is farther than all of these; otherwise the radius
            // widens to the bound, then the block grows. (A block that covers
            // the whole domain keeps everything.)
            const double bound2 = bound >= 1e299 ? INFINITY : (bound > 0.0 ? bound * bound : 0.0);
            const double keep2 = tight ? fmin(bound2, est2) : bound2;
            // gather candidates chunk by chunk; the current best k stay at the front.
            // The block is a list of runs of consecutive cells (one per row, two
            // where a periodic row wraps). A batch of up to 32 runs is laid out
            // flat: lane t loads run t's bounds (all loads in flight at once),
            // a warp scan gives each run its offset, and the flat candidate
            // list is walked 32 at a time, each lane finding its run by a
            // shuffle binary search. The candidate set and its order are those
            // of a row-by-row walk.
            int have = 0;  // entries in the buffer (best-so-far first)
            int total = 0;
            const int nrows = yhi - ylo + 1;
            const int nruns = 2 * nrows;
            for (int rb = 0; rb < nruns; rb += 32) {
                int rbeg = 0, rlen = 0;  // this lane's run: first candidate, length
                {
                    const int run = rb + lane;
                    if (run < nruns) {
                        const int rr = run >> 1, part = run & 1;
                        int cyy = ylo + rr;
                        if (g.Ly > 0) cyy = ((cyy % g.cy) + g.cy) % g.cy;
                        int c0 = 0, c1 = -1;  // empty unless set below
                        if (g.Lx > 0 && !fullx) {
                            const int a0 = xlo, a1 = xhi;
                            if (a0 < 0) {
                                if (part == 0) { c0 = a0 + g.cx; c1 = g.cx - 1; } else { c0 = 0; c1 = a1; }
                            } else if (a1 >= g.cx) {
                                if (part == 0) { c0 = a0; c1 = g.cx - 1; } else { c0 = 0; c1 = a1 - g.cx; }
                            } else if (part == 0) {
                                c0 = a0; c1 = a1;
                            }
                        } else if (part == 0) {
                            c0 = xlo; c1 = xhi;
                        }
                        if (c1 >= c0) {
                            rbeg = a.start[cyy * g.cx + c0];
                            rlen = a.start[cyy * g.cx + c1 + 1] - rbeg;
                        }
                    }
                }
                int incl = rlen;  // inclusive scan of the run lengths
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int excl = incl - rlen;
                const int btotal = __shfl_sync(0xffffffffu, incl, 31);
                for (int base = 0; base < btotal; base += 32) {
                    const int f = base + lane;
                    // the run holding flat index f: the number of runs ending at or
                    // before it (incl is non-decreasing over the lanes)
                    int r = 0;
#pragma unroll
                    for (int sh = 16; sh > 0; sh >>= 1) {
                        const int v = __shfl_sync(0xffffffffu, incl, r + sh - 1);
                        if (v <= f) r += sh;
                    }
                    const int jb = __shfl_sync(0xffffffffu, rbeg, r);
                    const int jx = __shfl_sync(0xffffffffu, excl, r);
                    const int j = jb + (f - jx);
                    bool ok = f < btotal;
                    unsigned long long dk = 0;
                    int ik = 0;
                    if (ok) {
                        const double d2 = sqdist(qx, qy, a.sx[j], a.sy[j], g.Lx, g.Ly);
                        ok = d2 < keep2;
                        dk = (unsigned long long)__double_as_longlong(d2);
                        ik = a.sidx[j];
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, ok);
                    const int cnt = __popc(bal);
                    if (have + cnt > kCap) {
                        // merge: keep the k best of the buffer
                        __syncwarp();
                        int keepd[kCap / 32];
#pragma unroll
                        for (int u = 0; u < kCap / 32; ++u) {
                            const int c = lane + 32 * u;
                            int rank = kCap;
                            if (c < have) {
                                rank = 0;
                                for (int v = 0; v < have; ++v)
                                    rank += key_less(d[v], id[v], d[c], id[c]);
                            }
                            keepd[u] = rank;
                        }
                        unsigned long long td[kCap / 32];
                        int ti[kCap / 32];
#pragma unroll
                        for (int u = 0; u < kCap / 32; ++u) {
                            const int c = lane + 32 * u;
                            td[u] = c < have ? d[c] : 0;
                            ti[u] = c < have ? id[c] : 0;
                        }
                        __syncwarp();
#pragma unroll
                        for (int u = 0; u < kCap / 32; ++u)
                            if (keepd[u] < k) {
                                d[keepd[u]] = td[u];
                                id[keepd[u]] = ti[u];
                            }
                        __syncwarp();
                        have = min(have, k);
                    }
                    const int pos = have + __popc(bal & ((1u << lane) - 1u));
                    if (ok) {
                        d[pos] = dk;
                        id[pos] = ik;
                    }
                    have += cnt;
                    total += cnt;
                    __syncwarp();
                }
            }
            if (total < k) {
                if (tight && keep2 < bound2) {
                    tight = false;  // same block, full bound
                    continue;
                }
                R += max(1, R / 2);
                continue;
            }
            // rank the buffer, write the k best: one pass over the buffer, each
            // (broadcast) entry compared with all of the lane's own entries
            int myrank[kCap / 32];
            unsigned long long mine_d[kCap / 32];
            int mine_i[kCap / 32];
            const int nslot = (have + 31) / 32;  // warp-uniform
#pragma unroll
            for (int u = 0; u < kCap / 32; ++u) {
                const int c = lane + 32 * u;
                myrank[u] = 0;
                mine_d[u] = (u < nslot && c < have) ? d[c] : 0ull;
                mine_i[u] = (u < nslot && c < have) ? id[c] : 0;
            }
            // the slot count is warp-uniform: one loop body per count, so only
            // the live slots are compared
            auto rank_with = [&](auto ns) {
                constexpr int NS = decltype(ns)::value;
                for (int v = 0; v < have; ++v) {
                    const unsigned long long dv = d[v];
                    const int iv = id[v];
#pragma unroll
                    for (int u = 0; u < NS; ++u) myrank[u] += key_less(dv, iv, mine_d[u], mine_i[u]);
                }
            };
            switch (nslot) {
                case 1: rank_with(std::integral_constant<int, 1>{}); break;
                case 2: rank_with(std::integral_constant<int, 2>{}); break;
                case 3: rank_with(std::integral_constant<int, 3>{}); break;
                case 4: rank_with(std::integral_constant<int, 4>{}); break;
                case 5: rank_with(std::integral_constant<int, 5>{}); break;
                case 6: rank_with(std::integral_constant<int, 6>{}); break;
                case 7: rank_with(std::integral_constant<int, 7>{}); break;
                default: rank_with(std::integral_constant<int, kCap / 32>{}); break;
            }
#pragma unroll
            for (int u = 0; u < kCap / 32; ++u)
                if (lane + 32 * u >= have) myrank[u] = kCap;
            // k-th distance: the entry of rank k-1, broadcast by two max-reductions
            unsigned long long dkth = 0;
#pragma unroll
            for (int u = 0; u < kCap / 32; ++u)
                if (myrank[u] == k - 1) dkth = d[lane + 32 * u];
            const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)(dkth >> 32));
            const unsigned lo =
                __reduce_max_sync(0xffffffffu, ((unsigned)(dkth >> 32) == hi) ? (unsigned)dkth : 0u);
            const unsigned long long dk_all = ((unsigned long long)hi << 32) | lo;
            const double dk2 = __longlong_as_double((long long)dk_all);
            if (dk2 < bound * bound || (bound >= 1e299)) {
#pragma unroll
                for (int u = 0; u < kCap / 32; ++u)
                    if (myrank[u] < k) a.ja[(size_t)q * k + myrank[u]] = id[lane + 32 * u];
                done = true;
            } else {
                R += max(1, R / 2);
            }
            __syncwarp();
        }
        if (!done && lane == 0) atomicExch(a.status, 1);
    }
}

struct Workspace {
    size_t n_cap = 0, cells_cap = 0;
    int* cell_of = nullptr;
    int* count = nullptr;   // cells + 1
    int* start = nullptr;   // cells + 1
    int* cursor = nullptr;  // cells
    int* block_sums = nullptr;
    int* sidx = nullptr;
    double* sx = nullptr;
    double* sy = nullptr;
    double* fx = nullptr;
    double* fy = nullptr;
    double* qf = nullptr;  // folded queries (2 * nq)
    size_t nq_cap = 0;
    Grid* grid = nullptr;
    unsigned long long* bbox = nullptr;
    int* status = nullptr;
    int* total = nullptr;
};

Workspace* ws_of(rbfb_ctx* ctx) { return static_cast<Workspace*>(ctx->knn_ws); }

int ensure_ws(rbfb_ctx* ctx, size_t n, size_t cells) {
    if (!ctx->knn_ws) ctx->knn_ws = new Workspace();
    Workspace* w = ws_of(ctx);
    if (!w->grid) {
        RBFB_CUDA(ctx, cudaMalloc(&w->grid, sizeof(Grid)));
        RBFB_CUDA(ctx, cudaMalloc(&w->bbox, 4 * sizeof(unsigned long long)));
        RBFB_CUDA(ctx, cudaMalloc(&w->status, sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&w->total, sizeof(int)));
    }
    if (w->n_cap < n) {
        cudaFree(w->cell_of); cudaFree(w->sidx); cudaFree(w->sx); cudaFree(w->sy);
        cudaFree(w->fx); cudaFree(w->fy);
        w->n_cap = 0;
        RBFB_CUDA(ctx, cudaMalloc(&w->cell_of, n * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&w->sidx, n * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&w->sx, n * sizeof(double)));
        RBFB_CUDA(ctx, cudaMalloc(&w->sy, n * sizeof(double)));
        RBFB_CUDA(ctx, cudaMalloc(&w->fx, n * sizeof(double)));
        RBFB_CUDA(ctx, cudaMalloc(&w->fy, n * sizeof(double)));
        w->n_cap = n;
    }
    if (w->cells_cap < cells) {
        cudaFree(w->count); cudaFree(w->start); cudaFree(w->cursor); cudaFree(w->block_sums);
        w->cells_cap = 0;
        RBFB_CUDA(ctx, cudaMalloc(&w->count, (cells + 1) * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&w->start, (cells + 1) * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&w->cursor, (cells + 1) * sizeof(int)));
        RBFB_CUDA(ctx, cudaMalloc(&w->block_sums, ((cells + 1) / kScanBlock + 2) * sizeof(int)));
        w->cells_cap = cells;
    }
    return RBFB_OK;
}

// Builds the binned node set. Returns the number of cells or < 0.
int build(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* period,
          cudaStream_t st) {
    const bool periodic = period && period[0] > 0 && period[1] > 0;
    int cx, cy;
    if (periodic) {
        const double aspect = period[0] / period[1];
        const double cells = std::max(1.0, static_cast<double>(n) / kPerCell);
        cx = std::max(1, static_cast<int>(std::sqrt(cells * aspect)));
        cy = std::max(1, static_cast<int>(std::sqrt(cells / aspect)));
    } else {
        cx = cy = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(n) / kPerCell)));
    }
    const size_t cells = static_cast<size_t>(cx) * cy;
    int rc = ensure_ws(ctx, n, cells);
    if (rc) return rc;
    Workspace* w = ws_of(ctx);
    const int tpb = 256;
    const int blocks = std::max(1, std::min((n + tpb - 1) / tpb, ctx->sms * 8));
    if (periodic) {
        Grid g{0.0, 0.0, period[0] / cx, period[1] / cy, cx, cy, period[0], period[1]};
        set_grid_kernel<<<1, 1, 0, st>>>(g, w->grid);
        ctx->launches += 1;
    } else {
        bbox_init_kernel<<<1, 1, 0, st>>>(w->bbox);
        bbox_kernel<<<blocks, tpb, 0, st>>>(x, y, n, reinterpret_cast<double*>(w->bbox));
        grid_kernel<<<1, 1, 0, st>>>(w->bbox, cx, cy, w->grid);
        ctx->launches += 3;
    }
    RBFB_CUDA(ctx, cudaMemsetAsync(w->count, 0, (cells + 1) * sizeof(int), st));
    RBFB_CUDA(ctx, cudaMemsetAsync(w->cursor, 0, (cells + 1) * sizeof(int), st));
    cell_count_kernel<<<blocks, tpb, 0, st>>>(x, y, n, w->grid, w->cell_of, w->count, w->fx, w->fy);
    const int ncell1 = static_cast<int>(cells) + 1;
    const int nsb = (ncell1 + kScanBlock - 1) / kScanBlock;
    scan_block_kernel<<<nsb, kScanBlock, 0, st>>>(w->count, w->start, ncell1, w->block_sums);
    scan_sums_kernel<<<1, 1, 0, st>>>(w->block_sums, nsb, w->total);
    scan_add_kernel<<<nsb, kScanBlock, 0, st>>>(w->start, ncell1, w->block_sums);
    scatter_kernel<<<blocks, tpb, 0, st>>>(w->cell_of, n, w->start, w->cursor, w->fx, w->fy,
                                          w->sidx, w->sx, w->sy);
    ctx->launches += 5;
    RBFB_CUDA(ctx, cudaGetLastError());
    return static_cast<int>(cells);
}

int query(rbfb_ctx* ctx, int nq, const double* xq, const double* yq, int k, int* ja,
          cudaStream_t st) {
    Workspace* w = ws_of(ctx);
    RBFB_CUDA(ctx, cudaMemsetAsync(w->status, 0, sizeof(int), st));
    QueryArgs a{};
    a.g = w->grid;
    a.start = w->start;
    a.sidx = w->sidx;
    a.sx = w->sx;
    a.sy = w->sy;
    a.nq = nq;
    a.qx = xq;
    a.qy = yq;
    a.qorder = xq ? nullptr : w->sidx;
    a.k = k;
    a.ja = ja;
    a.status = w->status;
    const int blocks = std::max(1, std::min((nq + kWarps - 1) / kWarps, ctx->sms * 16));
    query_kernel<<<blocks, kWarps * 32, 0, st>>>(a);
    ctx->launches += 1;
    RBFB_CUDA(ctx, cudaGetLastError());
    return RBFB_OK;
}

}  // namespace knn
}  // namespace rbfb

using namespace rbfb;

extern "C" {

void rbfb_release_knn(rbfb_ctx* ctx) {
    auto* w = static_cast<knn::Workspace*>(ctx->knn_ws);
    if (!w) return;
    cudaFree(w->cell_of); cudaFree(w->count); cudaFree(w->start); cudaFree(w->cursor);
    cudaFree(w->block_sums); cudaFree(w->sidx); cudaFree(w->sx); cudaFree(w->sy);
    cudaFree(w->fx); cudaFree(w->fy); cudaFree(w->grid); cudaFree(w->bbox);
    cudaFree(w->status); cudaFree(w->total);
    delete w;
    ctx->knn_ws = nullptr;
}

static int knn_check(rbfb_ctx* ctx, int n, const double* x, const double* y, int k, const int* ja,
                     const double* period) {
    if (!x || !y || !ja) return fail(ctx, RBFB_EINVAL, "null pointer argument");
    if (n < 1 || k < 1 || k > n) return fail(ctx, RBFB_EINVAL, "need 1 <= k <= n");
    if (k > knn::kMaxK) return fail(ctx, RBFB_EUNSUPPORTED, "k above the search limit (128)");
    if (period && ((period[0] > 0) != (period[1] > 0)))
        return fail(ctx, RBFB_EINVAL, "periodic in both axes or neither");
    return RBFB_OK;
}

int rbfb_knn_stencils(rbfb_ctx* ctx, int n, const double* x, const double* y, int k,
                      const double* period_h, int* ja, void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int rc = knn_check(ctx, n, x, y, k, ja, period_h);
    if (rc) return rc;
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rc = knn::build(ctx, n, x, y, period_h, st);
    if (rc < 0) return rc;
    return knn::query(ctx, n, nullptr, nullptr, k, ja, st);
}

int rbfb_knn_query(rbfb_ctx* ctx, int n, const double* x, const double* y, int nq,
                   const double* xq, const double* yq, int k, const double* period_h, int* ja,
                   void* stream) {
    if (!ctx) return RBFB_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int rc = knn_check(ctx, n, x, y, k, ja, period_h);
    if (rc) return rc;
    if (nq < 0 || (nq > 0 && (!xq || !yq))) return fail(ctx, RBFB_EINVAL, "bad query arrays");
    RBFB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rc = knn::build(ctx, n, x, y, period_h, st);
    if (rc < 0) return rc;
    if (nq == 0) return RBFB_OK;
    return knn::query(ctx, nq, xq, yq, k, ja, st) == RBFB_OK
               ? RBFB_OK
               : RBFB_ECUDA;
}

// Status of the last search on this context's stream: 0 complete, 1 when a
// query gave up (more than 64 widenings). Synchronises `stream`.
int rbfb_knn_status(rbfb_ctx* ctx, void* stream) {
    if (!ctx || !ctx->knn_ws) return RBFB_EINVAL;
    int h = 0;
    RBFB_CUDA(ctx, cudaMemcpyAsync(&h, knn::ws_of(ctx)->status, sizeof(int), cudaMemcpyDeviceToHost,
                                   static_cast<cudaStream_t>(stream)));
    RBFB_CUDA(ctx, cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    return h;
}

}  // extern "C"

// ---- no-allocation variant: rbfb_knn_stencils_static ------------------------------
//
// Some callers may not allocate device memory once they are running: a solver
// loop that claimed all its device memory in a set-up phase and must not call
// cudaMalloc/cudaFree afterwards (those calls can synchronise the device and
// fragment the caller's pool), or a host application whose device memory is
// owned by another framework's allocator. For them this search keeps its
// scratch in a fixed array in device memory, defined below, instead of in a
// context: every GPU that loads the library holds the array until the process
// exits, and no call allocates anything.
namespace rbfb {
namespace knn {

constexpr int kStaticMaxNodes = 65536;                   // largest node set served
constexpr int kStaticMaxCells = kStaticMaxNodes / kPerCell;  // largest cell grid served
constexpr size_t al256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kS_cell_of = 0;
constexpr size_t kS_count = kS_cell_of + al256(4ull * kStaticMaxNodes);
constexpr size_t kS_start = kS_count + al256(4ull * (kStaticMaxCells + 1));
constexpr size_t kS_cursor = kS_start + al256(4ull * (kStaticMaxCells + 1));
constexpr size_t kS_bsums = kS_cursor + al256(4ull * (kStaticMaxCells + 1));
constexpr size_t kS_sidx = kS_bsums + al256(4ull * ((kStaticMaxCells + 1) / kScanBlock + 2));
constexpr size_t kS_sx = kS_sidx + al256(4ull * kStaticMaxNodes);
constexpr size_t kS_sy = kS_sx + al256(8ull * kStaticMaxNodes);
constexpr size_t kS_fx = kS_sy + al256(8ull * kStaticMaxNodes);
constexpr size_t kS_fy = kS_fx + al256(8ull * kStaticMaxNodes);
constexpr size_t kS_grid = kS_fy + al256(8ull * kStaticMaxNodes);
constexpr size_t kS_bbox = kS_grid + al256(sizeof(Grid));
constexpr size_t kS_status = kS_bbox + al256(4 * sizeof(unsigned long long));
constexpr size_t kS_total = kS_status + al256(2 * sizeof(int));

// The scratch. In host code this name is only a stand-in for the device
// array, never a device address: host code takes the address with
// cudaGetSymbolAddress (per device) and passes it to the kernels.
static __device__ __align__(256) unsigned char g_knn_static[kS_total];

namespace {
std::mutex g_static_mu;
void* g_static_addr[64] = {};  // device address of the array, per device ordinal

// The array's device address on the current device: looked up once per
// device (cudaGetSymbolAddress, with that device current) and cached for the
// process. A cudaDeviceReset ends the context the address belongs to, so
// these entry points must not be used across one. nullptr on failure.
unsigned char* static_scratch(int* dev_out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    *dev_out = dev;
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_knn_static) != cudaSuccess || !p) return nullptr;
        g_static_addr[dev] = p;
    }
    return static_cast<unsigned char*>(g_static_addr[dev]);
}
}  // namespace

}  // namespace knn
}  // namespace rbfb

extern "C" int rbfb_knn_stencils_static(int n, const double* x, const double* y, int k,
                                        const double* period_h, int* ja, void* stream) {
    using namespace rbfb::knn;
    // the argument checks (and codes) of rbfb_knn_stencils
    if (!x || !y || !ja) return RBFB_EINVAL;
    if (n < 1 || k < 1 || k > n) return RBFB_EINVAL;
    if (k > kMaxK) return RBFB_EUNSUPPORTED;
    const bool periodic = period_h && period_h[0] > 0 && period_h[1] > 0;
    if (period_h && ((period_h[0] > 0) != (period_h[1] > 0))) return RBFB_EINVAL;
    if (n > kStaticMaxNodes) return RBFB_ETOOBIG;
    // the cell grid of the search, as build() forms it
    int cx, cy;
    if (periodic) {
        const double aspect = period_h[0] / period_h[1];
        const double cells = std::max(1.0, static_cast<double>(n) / kPerCell);
        cx = std::max(1, static_cast<int>(std::sqrt(cells * aspect)));
        cy = std::max(1, static_cast<int>(std::sqrt(cells / aspect)));
    } else {
        cx = cy = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(n) / kPerCell)));
    }
    const long long cells = static_cast<long long>(cx) * cy;
    if (cells > kStaticMaxCells) return RBFB_ETOOBIG;
    int dev = 0;
    unsigned char* base = static_scratch(&dev);
    if (!base) return RBFB_ECUDA;
    int* cell_of = reinterpret_cast<int*>(base + kS_cell_of);
    int* count = reinterpret_cast<int*>(base + kS_count);
    int* start = reinterpret_cast<int*>(base + kS_start);
    int* cursor = reinterpret_cast<int*>(base + kS_cursor);
    int* bsums = reinterpret_cast<int*>(base + kS_bsums);
    int* sidx = reinterpret_cast<int*>(base + kS_sidx);
    double* sx = reinterpret_cast<double*>(base + kS_sx);
    double* sy = reinterpret_cast<double*>(base + kS_sy);
    double* fx = reinterpret_cast<double*>(base + kS_fx);
    double* fy = reinterpret_cast<double*>(base + kS_fy);
    Grid* grid = reinterpret_cast<Grid*>(base + kS_grid);
    unsigned long long* bbox = reinterpret_cast<unsigned long long*>(base + kS_bbox);
    int* status = reinterpret_cast<int*>(base + kS_status);
    int* total = status + 1;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tpb = 256;
    const int blocks = std::max(1, std::min((n + tpb - 1) / tpb, std::max(sms, 1) * 8));
    if (periodic) {
        Grid g{0.0, 0.0, period_h[0] / cx, period_h[1] / cy, cx, cy, period_h[0], period_h[1]};
        set_grid_kernel<<<1, 1, 0, st>>>(g, grid);
    } else {
        bbox_init_kernel<<<1, 1, 0, st>>>(bbox);
        bbox_kernel<<<blocks, tpb, 0, st>>>(x, y, n, reinterpret_cast<double*>(bbox));
        grid_kernel<<<1, 1, 0, st>>>(bbox, cx, cy, grid);
    }
    // what must start at zero: the per-cell counters and the status word
    if (cudaMemsetAsync(count, 0, (cells + 1) * sizeof(int), st) != cudaSuccess ||
        cudaMemsetAsync(cursor, 0, (cells + 1) * sizeof(int), st) != cudaSuccess ||
        cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess)
        return RBFB_ECUDA;
    cell_count_kernel<<<blocks, tpb, 0, st>>>(x, y, n, grid, cell_of, count, fx, fy);
    const int ncell1 = static_cast<int>(cells) + 1;
    const int nsb = (ncell1 + kScanBlock - 1) / kScanBlock;
    scan_block_kernel<<<nsb, kScanBlock, 0, st>>>(count, start, ncell1, bsums);
    scan_sums_kernel<<<1, 1, 0, st>>>(bsums, nsb, total);
    scan_add_kernel<<<nsb, kScanBlock, 0, st>>>(start, ncell1, bsums);
    scatter_kernel<<<blocks, tpb, 0, st>>>(cell_of, n, start, cursor, fx, fy, sidx, sx, sy);
    QueryArgs a{};
    a.g = grid;
    a.start = start;
    a.sidx = sidx;
    a.sx = sx;
    a.sy = sy;
    a.nq = n;
    a.qorder = sidx;
    a.k = k;
    a.ja = ja;
    a.status = status;
    const int qblocks = std::max(1, std::min((n + kWarps - 1) / kWarps, std::max(sms, 1) * 16));
    query_kernel<<<qblocks, kWarps * 32, 0, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}

// Completion status of the last rbfb_knn_stencils_static search on the
// current device: reads the status word of the fixed array into a host
// local (no allocation) and synchronises `stream`.
extern "C" int rbfb_knn_static_status(void* stream) {
    int dev = 0;
    unsigned char* base = rbfb::knn::static_scratch(&dev);
    if (!base) return RBFB_ECUDA;
    int h = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(&h, base + rbfb::knn::kS_status, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return RBFB_ECUDA;
    return h;
}
