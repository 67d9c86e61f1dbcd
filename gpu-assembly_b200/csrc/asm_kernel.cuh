// asm_kernel.cuh -- batched RBF-FD assembly on sm_100a: gather + FP64 centre
// shift + radius scaling, FP64 fill of the saddle-point system, Gaussian
// elimination with partial pivoting in registers, back substitution,
// optional FP64 iterative refinement, and the CSR scatter.
//
// Replaces assemble_interp_weights<Config> (src/rbf_operators.h:292-376),
// whose solve is cuSolverDx gesv_partial_pivot with one stencil per CTA.
//
// Layout. A group of G = GR x GC lanes (G <= 32, inside one warp) owns one
// stencil; a CTA holds BLOCK / G groups and the grid is persistent. The
// system is padded to NTP unknowns and ordered polynomial block first:
// unknowns [lambda (NP), w (k), padding]; equations [P^T rows (NP), node
// rows (k), padding rows]. Padding rows/columns are identity, so the real
// unknowns see exactly the arithmetic of the unpadded system. Row r lives in
// lane-row r % GR, register slot r / GR; column c in lane-column c % GC,
// register column c / GC. Right-hand sides are replicated in the GC lanes of
// a lane-row. Rows are never swapped: pst[s] records the elimination step at
// which the row in slot s became the pivot row (kFree while unused).
//
// Phases of one stencil:
//   gather   lanes take ja and the neighbour coordinates (FP64) -- from
//            shared memory when the previous stencil's call prefetched them
//            with cp.async (PF shapes), else from global memory -- shift to
//            the centre (minimum image in a periodic box) and take the group
//            max of the binary exponents for the power-of-two radius scale;
//   fill     phi for each unordered node pair once, monomials per node, the
//            right-hand sides per row: all FP64, written (rounded to T) into
//            a shared-memory staging matrix S, then loaded into the row
//            registers (register shapes);
//   factor   register shapes: a runtime loop over blocks of GC*VEC steps,
//            the steps of a block unrolled (register indices static). Per
//            step: the pivot found by the look-ahead reduction (one 32-bit
//            key per candidate, pivot_key: the magnitude word without its 7
//            lowest bits, the row index in those bits, ties to the lowest row
//            as in the oracle); the pivot row's owner
//            lanes write it to a double-buffered shared row, __syncwarp,
//            every lane reads it back; l = a(r,c) * (1/pivot) for unused rows
//            (0 otherwise); a(r,j) = fma(-l, u(j), a(r,j)) for j > c and for
//            the right-hand sides; l is kept in a(r,c) (the L factor).
//            Shared-memory shapes (n up to 80): the same steps on S, blocked
//            right-looking in panels (eliminate_smem);
//   solve    the factors are in S; column-oriented back substitution from S:
//            x_c = y(p_c) * (1/pivot_c), then y(r) = fma(-u(r,c), x_c, y(r))
//            for rows pivoted before c;
//   refine   (MIXED: factor in FP32) residual b - M x in FP64 from the FP64
//            phi cache and monomials in shared memory, correction through
//            the FP32 factors in S, x += d in FP64, until the predicted
//            remaining error is below the tolerance; a stencil that stalls,
//            diverges or runs out of sweeps is queued for the FP64 kernel;
//   scatter  weights of the k node unknowns, rescaled by 2^(-order*e), to
//            values[q][row offset + j] (coalesced over j).
#pragma once

#include <cstdint>
#include <type_traits>

#include "asm_math.cuh"

namespace rbfb {

constexpr int kMaxRhs = 8;
constexpr int kFree = 0x3fffffff;  // pst of a row that is not yet a pivot row

struct AsmParams {
    int nitems;               // stencils to process (list entries, or 0..nitems-1)
    int item_base;            // first stencil id when list is nullptr
    const int* list;          // stencil ids, or nullptr
    const int* nitems_dev;    // device-side item count (overrides nitems when set)
    const int* list_off_dev;  // device-side offset into list and fb_list, or nullptr
    const double* x;
    const double* y;
    const int* ja;  // fixed width: row s at ja + s*k; CSR: ja + ia[s]
    const int* ia;  // nullptr for fixed width
    int k;          // fixed width stencil size
    int row_base;   // fixed width: ja, values and info hold rows row_base.. only
    double Lx, Ly;  // periods (<= 0: open axis)
    int scale;
    int nrhs;
    int col_op[kMaxRhs];  // RBFB_OP_* of every right-hand-side column
    int col_ic[kMaxRhs];  // interpolation point index of OP_INTERP columns
    const double* xc;
    const double* yc;
    double* values[kMaxRhs];
    double* const* values_dev;  // the same table in device memory (read when set)
    int* info;
    // refinement (MIXED)
    int max_sweeps;
    double ir_tol;
    int* fb_list;  // stencils handed to the FP64 kernel
    int* fb_count;
    unsigned long long* sweeps_sum;
    int* sweeps_max;
    int* work;  // dynamic work counter, or nullptr for a static stride
};

// Output array of right-hand side q: from the device-resident table when the
// caller passed one (the reference's T* const* A), else from the parameters.
__device__ __forceinline__ double* out_column(const AsmParams& p, int q) {
    return p.values_dev ? p.values_dev[q] : p.values[q];
}

// Asynchronous global -> shared copies (cp.async, no register staging):
// the next stencil's data is fetched while the current one is solved.
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Pivot keys. The magnitude word of a candidate: the bits of |v| for
// float, the high 32 bits of |v|'s binary64 representation (sign, exponent,
// 20 leading mantissa bits) for double. A key is that word without its 7
// lowest bits, plus one (an unused zero still counts), with the row index
// (as 127 - r, so ties go to the lowest row) in the freed bits: one 32-bit
// warp reduction finds the pivot. The oracle compares the same words.
__device__ __forceinline__ uint32_t mag32(float v) { return __float_as_uint(fabsf(v)); }
__device__ __forceinline__ uint32_t mag32(double v) {
    return (uint32_t)((unsigned long long)__double_as_longlong(fabs(v)) >> 32);
}
__device__ __forceinline__ uint32_t pivot_key(uint32_t mag, int r) {
    return (((mag >> 7) + 1u) << 7) | (uint32_t)(127 - r);
}
__device__ __forceinline__ float recip_rn(float v) { return __frcp_rn(v); }
__device__ __forceinline__ double recip_rn(double v) { return __drcp_rn(v); }

__device__ __forceinline__ unsigned group_mask(int G) {
    if (G == 32) return 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
}

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED, bool SMEM = false>
struct AsmCfg {
    static constexpr int G = GR * GC;
    static_assert(G <= 32 && (G & (G - 1)) == 0, "group is a power of two inside a warp");
    static_assert(NTP % GR == 0 && NTP % GC == 0, "padded size must tile the lanes");
    static_assert(!MIXED || sizeof(T) == 4, "refinement factors in FP32");
    static constexpr int NP = npoly(P);
    static constexpr int R = NTP / GR;   // row slots per lane
    static constexpr int CW = NTP / GC;  // register columns per lane
    static constexpr int KMAX = NTP - NP;
    static constexpr int NPAIR = KMAX * (KMAX - 1) / 2;  // packed strict upper triangle
    static constexpr int KPL = (KMAX + G - 1) / G;       // gathered nodes per lane
    static constexpr int VEC = 2;  // register tuples: float2 / double2
    static_assert(SMEM || CW % VEC == 0, "register columns must tile the vector width");
    static_assert(NTP <= 128, "pivot keys carry the row index in 7 bits");
    // pivot row buffer: NTP columns, NRHS right-hand sides, the pivot's reciprocal
    static constexpr int BW = ((NTP + NRHS + 1 + VEC - 1) / VEC) * VEC;
    // S row stride. The lanes of a group read S down a column (the back
    // substitution, the refinement sweeps, the shared-memory elimination) and
    // write it across rows (the fill), so consecutive rows must start in
    // different banks: an odd stride in elements for the shared-memory
    // elimination; for the register path, whose rows move as tuples,
    // an odd stride in tuples (at most two rows of a column share a bank).
    static constexpr int LDS = SMEM ? NTP + 1 : ((NTP / VEC) % 2 == 0 ? NTP + VEC : NTP);
    static constexpr int al16(int b) { return (b + 15) & ~15; }
    static constexpr int off_cx = 0;
    static constexpr int off_cy = off_cx + al16(8 * KMAX);
    static constexpr int off_s = off_cy + al16(8 * KMAX);
    static constexpr int off_x = off_s + al16(NTP * LDS * (int)sizeof(T));
    static constexpr int off_buf = off_x + al16(NTP * NRHS * (int)sizeof(T));
    static constexpr int off_phi = off_buf + al16(2 * BW * (int)sizeof(T));
    static constexpr int off_pm = off_phi + (MIXED ? al16(8 * NPAIR) : 0);
    static constexpr int off_x64 = off_pm + (MIXED ? al16(8 * KMAX * NP) : 0);
    static constexpr int off_b64 = off_x64 + (MIXED ? al16(8 * NTP * NRHS) : 0);
    static constexpr int off_piv = off_b64 + (MIXED ? al16(8 * NTP * NRHS) : 0);
    // next stencil, prefetched while this one is solved: its ja row, its
    // centre (x, y) and its CSR bounds ia[s], ia[s + 1]
    static constexpr int off_nja = off_piv + al16(4 * NTP);  // pivot row of each step before it
    static constexpr int off_nxy = off_nja + al16(4 * KMAX);
    static constexpr int off_nia = off_nxy + 16;
    static constexpr int bytes = off_nia + 16;
    // S position of column c (de-interleaved by lane-column)
    static __device__ __forceinline__ int scol(int c) { return (c % GC) * CW + c / GC; }
};

// Register rows are kept as two-element tuples (float2 / double2) so the
// pivot row goes to shared memory straight from aligned register pairs. A
// block of the elimination covers GC * 2 steps; for FP32, wider float4
// tuples would double the unrolled steps per block (and the code size)
// for no fewer shared-memory instructions that matter.
template <typename T>
struct Vec;
template <>
struct Vec<float> {
    using type = float2;
};
template <>
struct Vec<double> {
    using type = double2;
};
__device__ __forceinline__ float& comp(float2& v, int t) { return t == 0 ? v.x : v.y; }
__device__ __forceinline__ double& comp(double2& v, int t) { return t == 0 ? v.x : v.y; }

// Packed index of the pair (i, j), i < j, of a k-node stencil.
__device__ __forceinline__ int tri(int i, int j, int k) {
    return i * (2 * k - i - 1) / 2 + (j - i - 1);
}
__device__ __forceinline__ double phi_at(const double* phi, int i, int j, int k) {
    return i == j ? 0.0 : (i < j ? phi[tri(i, j, k)] : phi[tri(j, i, k)]);
}

// Right-hand sides of node row (xi, yi): every column q < nrhs, FP64, the
// PHS power r^(Q-2) shared by the derivative operators (one square root).
template <int P, int Q, int NRHS>
__device__ __forceinline__ void rhs_node(const AsmParams& p, double xi, double yi, int e,
                                         double* out) {
    const double r2 = dist2(xi, yi);
    const double rq2 = phs64<Q - 2>(r2);
    const double q = static_cast<double>(Q);
    const double qr = dmul(q, rq2);
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
        double v = 0.0;
        if (c < p.nrhs) {
            const int op = p.col_op[c];
            switch (op) {
                case kOpInterp: {
                    const double xe = scalbn(p.xc[p.col_ic[c]], -e);
                    const double ye = scalbn(p.yc[p.col_ic[c]], -e);
                    v = phs64<Q>(dist2(dsub(xe, xi), dsub(ye, yi)));
                    break;
                }
                case kOpLaplace: v = dmul(q * q, rq2); break;
                case kOpDx: v = -dmul(qr, xi); break;
                case kOpDy: v = -dmul(qr, yi); break;
                default: v = phs_op_origin<Q>(op, xi, yi); break;
            }
        }
        out[c] = v;
    }
}
template <int P>
__device__ __forceinline__ double rhs_poly(const AsmParams& p, int q, int m, int e) {
    const int op = p.col_op[q];
    if (op == kOpInterp) {
        int a, b;
        mono_exps(m, a, b);
        return mono_ab<P>(scalbn(p.xc[p.col_ic[q]], -e), scalbn(p.yc[p.col_ic[q]], -e), a, b);
    }
    return poly_op_origin(op, m);
}

// Gaussian elimination with row-implicit partial pivoting on the matrix in
// shared memory (systems too large for register rows), blocked right-looking.
// Lane (lr, lc) owns rows lr + GR*sl and columns c = lc (mod GC). The
// columns go in panels of PB:
//   A. the panel's PB steps, each: pivot search on the lanes' rows (the same
//      keys and reduction as the register path), multipliers
//      l = a(r,c) * (1/pivot) kept in place as the L factor, the update
//      a(r,j) -= l * a(p,j) confined to the panel's columns, and the
//      right-hand sides (X, shared);
//   B. the panel's pivot rows over the trailing columns: row p_t receives
//      the updates of steps t' < t, in order (a triangular pass spread over
//      all lanes by column);
//   C. every row not yet pivoted, over the trailing columns: the PB updates
//      of the panel, in order, with one load and one store per element.
// Each element sees exactly the fused multiply-adds of the unblocked
// elimination, in the same order, so the result is bit-identical to it; the
// shared-memory traffic of the trailing update drops by PB.
// On return yv holds the transformed right-hand sides of the lane's rows,
// pst/dinv/pivrow as the register path.
template <typename T, int GR, int GC, int NTP, int NRHS, typename C>
__device__ __forceinline__ void eliminate_smem(T* S, T* X, T* buf, int* pivrow, T (&yv)[C::R][NRHS],
                                               int (&pst)[C::R], T (&dinv)[C::R], int& info,
                                               int lr, int lc, int lg, unsigned gmask) {
    constexpr int R = C::R, LDS = C::LDS, G = C::G, BW = C::BW;
    constexpr int PB = 8;  // panel width
    static_assert(NTP % PB == 0, "whole panels");
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        pst[sl] = kFree;
        dinv[sl] = T(0);
    }
#pragma unroll 1
    for (int c0 = 0; c0 < NTP; c0 += PB) {
        // ---- A. the panel's steps
#pragma unroll 1
        for (int c = c0; c < c0 + PB; ++c) {
            const int sc = C::scol(c);
            // pivot search over the lanes' rows (lane-column 0 only; pivot_key)
            int prow;
            bool zero_pivot;
            T my_inv;
            {
                T lbest = T(1);
                uint32_t best = 0;
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    const int r = lr + GR * sl;
                    const T v = S[r * LDS + sc];
                    const uint32_t kk = (lc == 0 && pst[sl] == kFree) ? pivot_key(mag32(v), r) : 0u;
                    if (kk > best) {
                        best = kk;
                        lbest = v;
                    }
                }
                my_inv = recip_rn(lbest);
                const uint32_t m = __reduce_max_sync(gmask, best);
                prow = 127 - (int)(m & 127u);
                zero_pivot = (m >> 7) <= 1u;
            }
            if (zero_pivot && info == 0) info = c + 1;
            const int plr = prow % GR, psl = prow / GR;
            if (lg == 0) pivrow[c] = prow;
            // the owner publishes 1/pivot; everybody marks the pivot row used
            if (lr == plr && lc == 0) buf[BW - 1] = my_inv;
            __syncwarp(gmask);
            const T inv = buf[BW - 1];
#pragma unroll
            for (int sl = 0; sl < R; ++sl)
                if (lr == plr && sl == psl) {
                    pst[sl] = c;
                    dinv[sl] = inv;
                }
            // multipliers of the lane's unused rows
            T l[R];
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                const int r = lr + GR * sl;
                l[sl] = (pst[sl] == kFree) ? S[r * LDS + sc] * inv : T(0);
            }
            __syncwarp(gmask);  // everybody has read column c
            if (lc == 0) {
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
                    if (pst[sl] == kFree) S[(lr + GR * sl) * LDS + sc] = l[sl];
            }
            // update: the lane's rows over its panel columns j > c, then the
            // right-hand sides. All rows are loaded and updated branch-free
            // (independent chains the compiler can interleave); only the rows
            // not yet pivoted are stored back, so pivoted rows stay as they are.
            const T* Sp = S + prow * LDS;
            for (int j = c + 1 + ((lc - c - 1) % GC + GC) % GC; j < c0 + PB; j += GC) {
                const int sj = C::scol(j);
                const T u = Sp[sj];
                T v[R];
#pragma unroll
                for (int sl = 0; sl < R; ++sl) v[sl] = S[(lr + GR * sl) * LDS + sj];
#pragma unroll
                for (int sl = 0; sl < R; ++sl) v[sl] = fma(-l[sl], u, v[sl]);
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
                    if (pst[sl] == kFree) S[(lr + GR * sl) * LDS + sj] = v[sl];
            }
            if (lc == 0) {
                T uq[NRHS];
#pragma unroll
                for (int q = 0; q < NRHS; ++q) uq[q] = X[prow * NRHS + q];
                T v[R][NRHS];
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
#pragma unroll
                    for (int q = 0; q < NRHS; ++q) v[sl][q] = X[(lr + GR * sl) * NRHS + q];
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
#pragma unroll
                    for (int q = 0; q < NRHS; ++q) v[sl][q] = fma(-l[sl], uq[q], v[sl][q]);
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
                    if (pst[sl] == kFree) {
#pragma unroll
                        for (int q = 0; q < NRHS; ++q) X[(lr + GR * sl) * NRHS + q] = v[sl][q];
                    }
            }
            __syncwarp(gmask);
        }
        const int jt = c0 + PB;  // first trailing column
        if (jt >= NTP) break;
        int prw[PB];  // the panel's pivot rows
#pragma unroll
        for (int t = 0; t < PB; ++t) prw[t] = pivrow[c0 + t];
        // ---- B. the panel's pivot rows over the trailing columns
        for (int j = jt + lg; j < NTP; j += G) {
            const int sj = C::scol(j);
            T u[PB];
#pragma unroll
            for (int t = 0; t < PB; ++t) {
                T* e = S + prw[t] * LDS + sj;
                T v = *e;
#pragma unroll
                for (int tp = 0; tp < t; ++tp)
                    v = fma(-S[prw[t] * LDS + C::scol(c0 + tp)], u[tp], v);
                *e = v;
                u[t] = v;
            }
        }
        __syncwarp(gmask);
        // ---- C. the rows not yet pivoted over the trailing columns
        T lm[R][PB];
#pragma unroll
        for (int sl = 0; sl < R; ++sl)
#pragma unroll
            for (int t = 0; t < PB; ++t)
                lm[sl][t] = (pst[sl] == kFree) ? S[(lr + GR * sl) * LDS + C::scol(c0 + t)] : T(0);
        for (int j = jt + ((lc - jt) % GC + GC) % GC; j < NTP; j += GC) {
            const int sj = C::scol(j);
            T u[PB];
#pragma unroll
            for (int t = 0; t < PB; ++t) u[t] = S[prw[t] * LDS + sj];
            // R independent chains, interleaved step by step; each element
            // still takes the PB updates in order t = 0..PB-1
            T v[R];
#pragma unroll
            for (int sl = 0; sl < R; ++sl) v[sl] = S[(lr + GR * sl) * LDS + sj];
#pragma unroll
            for (int t = 0; t < PB; ++t)
#pragma unroll
                for (int sl = 0; sl < R; ++sl) v[sl] = fma(-lm[sl][t], u[t], v[sl]);
#pragma unroll
            for (int sl = 0; sl < R; ++sl)
                if (pst[sl] == kFree) S[(lr + GR * sl) * LDS + sj] = v[sl];
        }
        __syncwarp(gmask);
    }
#pragma unroll
    for (int sl = 0; sl < R; ++sl)
#pragma unroll
        for (int q = 0; q < NRHS; ++q) yv[sl][q] = X[(lr + GR * sl) * NRHS + q];
    __syncwarp(gmask);
}

// The prefetch of a group's first stencil, done up front (the stages that
// assemble_one spreads over a stencil's solve, back to back): centre and CSR
// bounds, then the ja row, then the neighbour coordinates into cx/cy.
template <class C>
__device__ __forceinline__ void prefetch_first(const AsmParams& p, int s, char* smem, int lg,
                                               unsigned gmask) {
    constexpr int G = C::G;
    double* cx = reinterpret_cast<double*>(smem + C::off_cx);
    double* cy = reinterpret_cast<double*>(smem + C::off_cy);
    int* nja = reinterpret_cast<int*>(smem + C::off_nja);
    double* nxy = reinterpret_cast<double*>(smem + C::off_nxy);
    int* nia = reinterpret_cast<int*>(smem + C::off_nia);
    if (lg == 0) {
        cp_async8(nxy, p.x + s);
        cp_async8(nxy + 1, p.y + s);
        if (p.ia) {
            cp_async4(nia, p.ia + s);
            cp_async4(nia + 1, p.ia + s + 1);
        }
    }
    cp_async_wait_all();
    __syncwarp(gmask);
    const int off = p.ia ? nia[0] : (s - p.row_base) * p.k;
    const int ks = p.ia ? nia[1] - off : p.k;
    for (int j = lg; j < ks; j += G) cp_async4(nja + j, p.ja + off + j);
    cp_async_wait_all();
    for (int j = lg; j < ks; j += G) {  // this lane's own ja slots
        const int nb = nja[j];
        cp_async8(cx + j, p.x + nb);
        cp_async8(cy + j, p.y + nb);
    }
}

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED, bool SMEM,
          bool PF>
__device__ __forceinline__ void assemble_one(const AsmParams& p, int s, int sn, char* smem,
                                             int lg, unsigned gmask) {
    using C = AsmCfg<T, GR, GC, NTP, NRHS, P, Q, MIXED, SMEM>;
    constexpr int G = C::G, NP = C::NP, R = C::R, CW = C::CW, BW = C::BW, VEC = C::VEC;
    constexpr int LDS = C::LDS;
    double* cx = reinterpret_cast<double*>(smem + C::off_cx);
    double* cy = reinterpret_cast<double*>(smem + C::off_cy);
    T* S = reinterpret_cast<T*>(smem + C::off_s);
    T* X = reinterpret_cast<T*>(smem + C::off_x);
    T* buf = reinterpret_cast<T*>(smem + C::off_buf);
    double* phi = reinterpret_cast<double*>(smem + C::off_phi);
    double* pm = reinterpret_cast<double*>(smem + C::off_pm);
    double* x64 = reinterpret_cast<double*>(smem + C::off_x64);
    double* b64 = reinterpret_cast<double*>(smem + C::off_b64);

    const int lr = lg / GC, lc = lg % GC;
    int* nja = reinterpret_cast<int*>(smem + C::off_nja);
    double* nxy = reinterpret_cast<double*>(smem + C::off_nxy);
    int* nia = reinterpret_cast<int*>(smem + C::off_nia);

    // With PF, stencil s was prefetched (by the previous call of this group,
    // or by prefetch_first): its neighbour coordinates wait in cx/cy (raw),
    // its centre in nxy, its CSR bounds in nia. Without PF everything comes
    // from global memory. (Every call of a shape takes the same branch, so
    // the stencil body exists once in the kernel's code.)
    int off, ks;
    double x0, y0;
    if constexpr (PF) {
        cp_async_wait_all();
        __syncwarp(gmask);
        x0 = nxy[0];
        y0 = nxy[1];
        off = p.ia ? nia[0] : (s - p.row_base) * p.k;
        ks = p.ia ? nia[1] - off : p.k;
        __syncwarp(gmask);  // read before the slots are refilled below
    } else {
        x0 = p.x[s];
        y0 = p.y[s];
        off = p.ia ? p.ia[s] : (s - p.row_base) * p.k;
        ks = p.ia ? p.ia[s + 1] - off : p.k;
    }
    const int n = NP + ks;
    // prefetch (PF), stage 1: the next stencil's centre and CSR bounds
    if (PF && sn >= 0 && lg == 0) {
        cp_async8(nxy, p.x + sn);
        cp_async8(nxy + 1, p.y + sn);
        if (p.ia) {
            cp_async4(nia, p.ia + sn);
            cp_async4(nia + 1, p.ia + sn + 1);
        }
    }

    // ---- gather + FP64 shift (+ minimum image), src/rbf_operators.h:354-358
    int e;
    {
        double gx[C::KPL], gy[C::KPL];
        int emax = -100000;
#pragma unroll
        for (int t = 0; t < C::KPL; ++t) {
            const int j = lg + t * G;
            gx[t] = 0.0;
            gy[t] = 0.0;
            if (j < ks) {
                double xn, yn;
                if constexpr (PF) {
                    xn = cx[j];  // this lane's own prefetched slots
                    yn = cy[j];
                } else {
                    const int nb = __ldg(p.ja + off + j);
                    xn = __ldg(p.x + nb);
                    yn = __ldg(p.y + nb);
                }
                gx[t] = min_image(dsub(xn, x0), p.Lx);
                gy[t] = min_image(dsub(yn, y0), p.Ly);
                if (gx[t] != 0.0) emax = max(emax, ilogb(fabs(gx[t])) + 1);
                if (gy[t] != 0.0) emax = max(emax, ilogb(fabs(gy[t])) + 1);
            }
        }
        e = __reduce_max_sync(gmask, emax);
        e = (p.scale && e > -100000) ? e : 0;
#pragma unroll
        for (int t = 0; t < C::KPL; ++t) {
            const int j = lg + t * G;
            if (j < ks) {
                cx[j] = scalbn(gx[t], -e);
                cy[j] = scalbn(gy[t], -e);
            }
        }
    }
    __syncwarp(gmask);

    // ---- fill the staging matrix S (permuted, padded) and the right-hand sides
    // phi block: each unordered pair once. The pairs (i < j) are walked as
    // one flat sequence, G at a time: every lane busy, iterations independent.
    {
        const int npair = ks * (ks - 1) / 2;
        // (i, j) of pair number lg; past the end of row i (j >= ks) the walk
        // continues in row i + 1 at j - ks + i + 2
        int i = 0, j = 1 + lg;
        while (i < ks - 1 && j >= ks) {
            j += i + 2 - ks;
            ++i;
        }
        for (int t = lg; t < npair; t += G) {
            const double v = phs64<Q>(dist2(dsub(cx[j], cx[i]), dsub(cy[j], cy[i])));
            S[(NP + i) * LDS + C::scol(NP + j)] = static_cast<T>(v);
            S[(NP + j) * LDS + C::scol(NP + i)] = static_cast<T>(v);
            if constexpr (MIXED) phi[t] = v;  // t = tri(i, j, ks)
            j += G;
            while (i < ks - 1 && j >= ks) {
                j += i + 2 - ks;
                ++i;
            }
        }
    }
    // node rows: monomials (the row and its transposed P^T column), the zero
    // diagonal of the phi block, the right-hand sides
    for (int i = lg; i < ks; i += G) {
        const int r = NP + i;
        T* Sr = S + r * LDS;
        const double xi = cx[i], yi = cy[i];
        double mon[NP];
        monomials<P>(xi, yi, mon);
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            Sr[C::scol(m)] = static_cast<T>(mon[m]);
            S[m * LDS + C::scol(r)] = static_cast<T>(mon[m]);
            if constexpr (MIXED) pm[i * NP + m] = mon[m];
        }
        Sr[C::scol(r)] = T(0);
        double rv[NRHS];
        rhs_node<P, Q, NRHS>(p, xi, yi, e, rv);
#pragma unroll
        for (int q = 0; q < NRHS; ++q) {
            X[r * NRHS + q] = static_cast<T>(rv[q]);
            if constexpr (MIXED) b64[r * NRHS + q] = rv[q];
        }
    }
    // P^T rows: right-hand sides (the polynomial reproduction conditions)
    for (int r = lg; r < NP; r += G) {
#pragma unroll
        for (int q = 0; q < NRHS; ++q) {
            const double v = q < p.nrhs ? rhs_poly<P>(p, q, r, e) : 0.0;
            X[r * NRHS + q] = static_cast<T>(v);
            if constexpr (MIXED) b64[r * NRHS + q] = v;
        }
    }
    // padding rows: zero right-hand sides
    for (int r = n + lg; r < NTP; r += G) {
#pragma unroll
        for (int q = 0; q < NRHS; ++q) {
            X[r * NRHS + q] = T(0);
            if constexpr (MIXED) b64[r * NRHS + q] = 0.0;
        }
    }
    // the zero polynomial block, the padding columns of the real rows and the
    // identity padding rows, each as a flat sequence over the lanes
    for (int f = lg; f < NP * NP; f += G) S[(f / NP) * LDS + C::scol(f % NP)] = T(0);
    for (int r = lg; r < n; r += G)
        for (int c = n; c < NTP; ++c) S[r * LDS + C::scol(c)] = T(0);
    for (int f = lg; f < (NTP - n) * NTP; f += G) {
        const int r = n + f / NTP, c = f % NTP;
        S[r * LDS + C::scol(c)] = (r == c) ? T(1) : T(0);
    }
    // prefetch, stage 2: the next stencil's ja row (its bounds have landed);
    // its size goes to nia[2] (0: no next stencil), not held in a register
    if constexpr (PF) {
        int offn = 0, ksn = 0;
        if (sn >= 0) {
            if (p.ia) {
                cp_async_wait_all();
                __syncwarp(gmask);
                offn = nia[0];
                ksn = nia[1] - offn;
            } else {
                offn = (sn - p.row_base) * p.k;
                ksn = p.k;
            }
            for (int j = lg; j < ksn; j += G) cp_async4(nja + j, p.ja + offn + j);
        }
        __syncwarp(gmask);  // every lane has read nia[0..1]
        if (lg == 0) nia[2] = ksn;
    }
    __syncwarp(gmask);

    using V = typename Vec<T>::type;
    T yv[R][NRHS];
    int pst[R];
    T dinv[R];
    int* pivrow = reinterpret_cast<int*>(smem + C::off_piv);
    int info = 0;
    if constexpr (!SMEM) {
    // ---- rows into registers (vector loads)
    constexpr int NV = CW / VEC;  // register tuples per row slot
    V a[R][NV];
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        const int r = lr + GR * sl;
        const V* Sr = reinterpret_cast<const V*>(S + r * LDS + lc * CW);
#pragma unroll
        for (int cb = 0; cb < NV; ++cb) a[sl][cb] = Sr[cb];
#pragma unroll
        for (int q = 0; q < NRHS; ++q) yv[sl][q] = X[r * NRHS + q];
        pst[sl] = kFree;
        dinv[sl] = T(0);
    }

    // ---- elimination with row-implicit partial pivoting
    //
    // A runtime loop over blocks of SB = GC * VEC steps keeps the code small
    // enough for the instruction cache. The steps of a block pivot on the
    // columns held in register tuple 0 (static components); after the block,
    // tuple 0 -- now final: L multipliers of the rows not yet pivoted and U
    // entries of the others -- goes to S (physical row layout), and the
    // remaining tuples shift down by one. The blocks run in NWC width classes:
    // class w updates the NV - w*NV/NWC tuples still active at its start
    // (tuples that died inside the class hold zeros), so the bodies compiled
    // are NWC, not NTP.
    constexpr int SB = GC * VEC;
    static_assert(NTP % SB == 0, "padded size must be a whole number of blocks");
    // Width classes: more classes skip more dead tuples but compile more
    // step bodies (instruction-cache pressure). Measured on B200: rows of 12
    // or more tuples (n = 48; FP32 rows of 16 or 24) run fastest with 2
    // classes, rows of 8 tuples (FP64 n = 32) with 4.
    constexpr int NWC = NV >= 12 ? 2 : (NV >= 4 ? 4 : NV);
    // Pivot search with look-ahead: the keys of step c+1's column are formed
    // and their reduction issued as soon as that column is updated (first),
    // so the reduction runs while the rest of step c's update issues. The
    // pivot is the unused row of largest key (pivot_key: the oracle's rule);
    // used rows send 0.
    uint32_t pm_key = 0;  // reduced key of the next pivot
    T p_inv = T(1);       // reciprocal of this lane's best candidate
    auto keys_begin = [&](int tp, int cp, int lcc) {
        T lbest = T(1);
        uint32_t best = 0;
#pragma unroll
        for (int sl = 0; sl < R; ++sl) {
            const T v = comp(a[sl][tp], cp);
            const uint32_t kk =
                (lc == lcc && pst[sl] == kFree) ? pivot_key(mag32(v), lr + GR * sl) : 0u;
            if (kk > best) {
                best = kk;
                lbest = v;
            }
        }
        pm_key = __reduce_max_sync(gmask, best);
        p_inv = recip_rn(lbest);  // = the oracle's 1 / pivot (both rounded once)
    };
    keys_begin(0, 0, 0);
    auto step_block = [&](auto width, int b) {
        constexpr int W = decltype(width)::value;
#pragma unroll
        for (int j = 0; j < SB; ++j) {
            const int c = b * SB + j;
            const int lcc = j % GC, ctc = j / GC;  // lane-column and component of column c
            T* B = buf + (j & 1) * BW;
            // 1. the pivot found by the look-ahead
            int prow;
            bool zero_pivot;
            prow = 127 - (int)(pm_key & 127u);
            zero_pivot = (pm_key >> 7) <= 1u;
            const T my_inv = p_inv;
            if (zero_pivot && info == 0) info = c + 1;
            const int plr = prow % GR, psl = prow / GR;
            if (lg == 0) pivrow[c] = prow;

            // 2. pivot row to shared memory (owner lane-row), then broadcast
            if (lr == plr) {
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    if (sl == psl) {
                        V* Bv = reinterpret_cast<V*>(B + lc * CW);
#pragma unroll
                        for (int cb = 0; cb < W; ++cb) Bv[cb] = a[sl][cb];
                        if (lc == 0) {
#pragma unroll
                            for (int q = 0; q < NRHS; ++q) B[NTP + q] = yv[sl][q];
                        }
                        if (lc == lcc) B[BW - 1] = my_inv;
                        pst[sl] = c;
                    }
                }
            }
            __syncwarp(gmask);
            const T inv = B[BW - 1];
            if (lr == plr) {
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
                    if (sl == psl) dinv[sl] = inv;
            }
            // 3. multipliers (kept as the L factor) and the update
            T l[R];
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                T av = comp(a[sl][0], ctc);
                if constexpr (GC > 1) av = __shfl_sync(gmask, av, lr * GC + lcc, G);
                l[sl] = (pst[sl] == kFree) ? av * inv : T(0);
                if (lc == lcc && pst[sl] == kFree) comp(a[sl][0], ctc) = l[sl];
            }
            const V* Bv = reinterpret_cast<const V*>(B + lc * CW);
            auto update_tuple = [&](int cb) {
                V u = Bv[cb];
#pragma unroll
                for (int t = 0; t < VEC; ++t) {
                    if (cb == 0 && t < ctc) continue;  // columns already eliminated
                    if (cb == 0 && t == ctc) {
                        if constexpr (GC == 1) continue;
                        if (lc <= lcc) continue;       // column c itself or before it
                    }
#pragma unroll
                    for (int sl = 0; sl < R; ++sl)
                        comp(a[sl][cb], t) = fma(-l[sl], comp(u, t), comp(a[sl][cb], t));
                }
            };
            // the tuple holding the next pivot column first, then its keys
            const int jn = j + 1;
            const int tn = jn < SB ? 0 : 1;  // its tuple (before rotation)
            const bool more = (jn < SB) ? true : (W > 1);
            update_tuple(tn);
            if (tn == 1) update_tuple(0);
            if (more) keys_begin(tn, (jn % SB) / GC, jn % GC);
#pragma unroll
            for (int cb = 1; cb < W; ++cb)
                if (cb != tn) update_tuple(cb);
#pragma unroll
            for (int q = 0; q < NRHS; ++q) {
                const T uq = B[NTP + q];
#pragma unroll
                for (int sl = 0; sl < R; ++sl) yv[sl][q] = fma(-l[sl], uq, yv[sl][q]);
            }
        }
        // tuple 0 is final: to S at its tuple position, then shift down
#pragma unroll
        for (int sl = 0; sl < R; ++sl) {
            reinterpret_cast<V*>(S + (lr + GR * sl) * LDS + lc * CW)[b] = a[sl][0];
#pragma unroll
            for (int cb = 0; cb + 1 < W; ++cb) a[sl][cb] = a[sl][cb + 1];
            a[sl][W - 1] = V{};
        }
    };
    {
        int b = 0;
        auto run_class = [&](auto wc) {
            constexpr int w = decltype(wc)::value;
            constexpr int W = NV - (w * NV) / NWC;  // active tuples at the class start
            constexpr int bend = ((w + 1) * NV) / NWC;
#pragma unroll 1
            for (; b < bend; ++b) step_block(std::integral_constant<int, W>{}, b);
        };
        run_class(std::integral_constant<int, 0>{});
        if constexpr (NWC > 1) run_class(std::integral_constant<int, 1>{});
        if constexpr (NWC > 2) run_class(std::integral_constant<int, 2>{});
        if constexpr (NWC > 3) run_class(std::integral_constant<int, 3>{});
    }
    __syncwarp(gmask);

    } else {
        eliminate_smem<T, GR, GC, NTP, NRHS, C>(S, X, buf, pivrow, yv, pst, dinv, info, lr, lc, lg, gmask);
    }

    // Column-oriented back substitution from S into X[c][q], a runtime loop:
    // the owner lane of step c's pivot row forms x_c = y * (1/pivot) and
    // broadcasts it by shuffle; rows pivoted before c update with S(r, c).
    // The pivot row and the column of S of step c - 1 are loaded during step
    // c, so only the select -> shuffle -> fma chain is serial.
    auto back_substitute = [&](T (&yy)[R][NRHS]) {
        int pr = pivrow[NTP - 1];
        T un[R];
#pragma unroll
        for (int sl = 0; sl < R; ++sl) un[sl] = S[(lr + GR * sl) * LDS + C::scol(NTP - 1)];
#pragma unroll 1
        for (int c = NTP - 1; c >= 0; --c) {
            const int osl = pr / GR, olane = (pr % GR) * GC;
            T uc[R];
#pragma unroll
            for (int sl = 0; sl < R; ++sl) uc[sl] = un[sl];
            const int cn = c > 0 ? c - 1 : 0;
            pr = pivrow[cn];
            const int scn = C::scol(cn);
#pragma unroll
            for (int sl = 0; sl < R; ++sl) un[sl] = S[(lr + GR * sl) * LDS + scn];
            T xq[NRHS];
            T dv = dinv[0];
#pragma unroll
            for (int sl = 1; sl < R; ++sl) dv = (osl == sl) ? dinv[sl] : dv;
#pragma unroll
            for (int q = 0; q < NRHS; ++q) {
                T v = yy[0][q];
#pragma unroll
                for (int sl = 1; sl < R; ++sl) v = (osl == sl) ? yy[sl][q] : v;
                xq[q] = __shfl_sync(gmask, v * dv, olane, G);
            }
            if (lg == 0) {
#pragma unroll
                for (int q = 0; q < NRHS; ++q) X[c * NRHS + q] = xq[q];
            }
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                const T m = (pst[sl] < c) ? uc[sl] : T(0);
#pragma unroll
                for (int q = 0; q < NRHS; ++q) yy[sl][q] = fma(-m, xq[q], yy[sl][q]);
            }
        }
        __syncwarp(gmask);
    };
    // prefetch, stage 3: the next stencil's neighbour coordinates into cx/cy
    // (each lane gathers the slots j it fetched ja for, so no exchange)
    if (const int ksn = PF ? nia[2] : 0; ksn > 0) {
        cp_async_wait_all();
        for (int j = lg; j < ksn; j += G) {
            const int nb = nja[j];
            cp_async8(cx + j, p.x + nb);
            cp_async8(cy + j, p.y + nb);
        }
    }
    back_substitute(yv);

    const int nrhs = p.nrhs;
    if constexpr (!MIXED) {
        // ---- scatter, src/rbf_operators.h:368-375
        const bool bad = info != 0;
        for (int q = 0; q < nrhs; ++q) {
            double* dst = out_column(p, q) + off;
            const int sh = -op_order(p.col_op[q]) * e;
            for (int j = lg; j < ks; j += G) {
                const double v = static_cast<double>(X[(NP + j) * NRHS + q]);
                dst[j] = bad ? __longlong_as_double(0x7ff8000000000000ll) : scalbn(v, sh);
            }
        }
        if (lg == 0 && p.info) p.info[s - p.row_base] = info;
    } else {
        // ---- FP64 iterative refinement
        for (int i = lg; i < NTP * NRHS; i += G) x64[i] = static_cast<double>(X[i]);
        __syncwarp(gmask);
        int sweeps = 0;
        bool converged = false, failed = (info != 0);
        float prev = 3.4e38f;
        while (!converged && !failed) {
            if (sweeps >= p.max_sweeps) {
                failed = true;
                break;
            }
            ++sweeps;
            // residual r = b - M x (FP64), rows split over the lanes, into X (T)
            for (int r = lg; r < NTP; r += G) {
                double acc[NRHS];
#pragma unroll
                for (int q = 0; q < NRHS; ++q) acc[q] = b64[r * NRHS + q];
                if (r < NP) {
                    for (int j = 0; j < ks; ++j) {
                        const double mv = pm[j * NP + r];
#pragma unroll
                        for (int q = 0; q < NRHS; ++q)
                            acc[q] = fma(-mv, x64[(NP + j) * NRHS + q], acc[q]);
                    }
                } else if (r < n) {
                    const int i = r - NP;
#pragma unroll
                    for (int m = 0; m < NP; ++m) {
                        const double mv = pm[i * NP + m];
#pragma unroll
                        for (int q = 0; q < NRHS; ++q) acc[q] = fma(-mv, x64[m * NRHS + q], acc[q]);
                    }
                    // phi(i, j) for j < i: column i of the packed upper triangle,
                    // tri(j, i) advancing by ks - j - 2; for j > i: row i, contiguous
                    int t = i - 1;  // tri(0, i)
                    for (int j = 0; j < i; ++j) {
                        const double fv = phi[t];
                        t += ks - j - 2;
#pragma unroll
                        for (int q = 0; q < NRHS; ++q)
                            acc[q] = fma(-fv, x64[(NP + j) * NRHS + q], acc[q]);
                    }
                    const double* prow_i = phi + (i < ks - 1 ? tri(i, i + 1, ks) : 0);
                    for (int j = i + 1; j < ks; ++j) {
                        const double fv = prow_i[j - i - 1];
#pragma unroll
                        for (int q = 0; q < NRHS; ++q)
                            acc[q] = fma(-fv, x64[(NP + j) * NRHS + q], acc[q]);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < NRHS; ++q) acc[q] = 0.0;
                }
#pragma unroll
                for (int q = 0; q < NRHS; ++q) X[r * NRHS + q] = static_cast<T>(acc[q]);
            }
            __syncwarp(gmask);
            // residual into the row layout, then L (forward) and U (backward)
            T rv[R][NRHS];
#pragma unroll
            for (int sl = 0; sl < R; ++sl)
#pragma unroll
                for (int q = 0; q < NRHS; ++q) rv[sl][q] = X[(lr + GR * sl) * NRHS + q];
            __syncwarp(gmask);
#pragma unroll 1
            for (int t = 0; t < NTP; ++t) {
                const int pr = pivrow[t];
                const int osl = pr / GR, olane = (pr % GR) * GC;
                T zq[NRHS];
#pragma unroll
                for (int q = 0; q < NRHS; ++q) {
                    T v = rv[0][q];
#pragma unroll
                    for (int sl = 1; sl < R; ++sl) v = (osl == sl) ? rv[sl][q] : v;
                    zq[q] = __shfl_sync(gmask, v, olane, G);
                }
                const int st = C::scol(t);
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    const T lv = S[(lr + GR * sl) * LDS + st];
                    const T m = (pst[sl] > t) ? lv : T(0);
#pragma unroll
                    for (int q = 0; q < NRHS; ++q) rv[sl][q] = fma(-m, zq[q], rv[sl][q]);
                }
            }
            back_substitute(rv);
            // x += d; convergence on max|d| / max|x| per right-hand side
            float worst = 0.f;
            for (int q = 0; q < nrhs; ++q) {
                float dmax = 0.f, xmax = 0.f;
                for (int i = lg; i < NTP; i += G) {
                    const double d = static_cast<double>(X[i * NRHS + q]);
                    const double xn = x64[i * NRHS + q] + d;
                    x64[i * NRHS + q] = xn;
                    dmax = fmaxf(dmax, (float)fabs(d));
                    xmax = fmaxf(xmax, (float)fabs(xn));
                }
                dmax = __uint_as_float(__reduce_max_sync(gmask, __float_as_uint(dmax)));
                xmax = __uint_as_float(__reduce_max_sync(gmask, __float_as_uint(xmax)));
                worst = fmaxf(worst, xmax > 0.f ? dmax / xmax : dmax);
            }
            __syncwarp(gmask);
            // The correction of sweep k measures the error before it (tau_k);
            // the error left after it is about tau_k * rho / (1 - rho) with
            // rho = tau_k / tau_(k-1) the observed contraction (about
            // cond(M) * 2^-24). Converged when that prediction is below tol (or
            // the correction itself is at the FP64 floor). A contraction above
            // 0.1 means cond(M) > ~1e6: the prediction is unreliable there and
            // the FP64 rounding floor of the system itself approaches the
            // tolerance, so such a stencil (and a NaN) goes to the FP64 kernel.
            if (!(worst == worst)) {
                failed = true;
            } else {
                const float rho = sweeps >= 2 ? worst / fmaxf(prev, 1e-38f) : 1.0f;
                const float left = rho < 0.1f ? worst * rho / (1.0f - rho) : worst;
                if (left <= (float)p.ir_tol || worst <= 1e-15f) converged = true;
                else if (sweeps >= 2 && rho > 0.1f) failed = true;
            }
            prev = worst;
        }
        if (lg == 0) {
            if (p.sweeps_sum) atomicAdd(p.sweeps_sum, (unsigned long long)sweeps);
            if (p.sweeps_max) atomicMax(p.sweeps_max, sweeps);
        }
        if (failed) {
            if (lg == 0) {
                const int fo = p.list_off_dev ? *p.list_off_dev : 0;
                p.fb_list[fo + atomicAdd(p.fb_count, 1)] = s;
            }
        } else {
            for (int q = 0; q < nrhs; ++q) {
                double* dst = out_column(p, q) + off;
                const int sh = -op_order(p.col_op[q]) * e;
                for (int j = lg; j < ks; j += G) dst[j] = scalbn(x64[(NP + j) * NRHS + q], sh);
            }
            if (lg == 0 && p.info) p.info[s - p.row_base] = 0;
        }
    }
    __syncwarp(gmask);
}

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED, int BLOCK,
          int MINB, bool SMEM = false, bool PF = true>
__global__ void __launch_bounds__(BLOCK, MINB) asm_kernel(AsmParams p) {
    using C = AsmCfg<T, GR, GC, NTP, NRHS, P, Q, MIXED, SMEM>;
    constexpr int G = C::G;
    constexpr int GPB = BLOCK / G;  // groups per CTA
    extern __shared__ __align__(16) char smem_raw[];
    const int gib = threadIdx.x / G;
    const int lg = threadIdx.x % G;
    char* smem = smem_raw + gib * C::bytes;
    const unsigned gmask = group_mask(G);
    const int n = p.nitems_dev ? *p.nitems_dev : p.nitems;
    const int* list = (p.list && p.list_off_dev) ? p.list + *p.list_off_dev : p.list;
    const int ngroups = gridDim.x * GPB;
    auto claim = [&](int next_static) {
        if (!p.work) return next_static;
        int v = 0;
        if (lg == 0) v = atomicAdd(p.work, 1);
        return __shfl_sync(gmask, v, 0, G);
    };
    auto item = [&](int i) { return i < n ? (list ? list[i] : p.item_base + i) : -1; };
    // One call site: the stencil body is inlined once. With PF each call
    // also prefetches the next item's data (claimed one ahead) and the first
    // item is prefetched before the loop, so every call finds its stencil
    // prefetched. The next item number waits in shared memory during the
    // call (no register held across the solve).
    int* next_it = reinterpret_cast<int*>(smem + C::off_nia) + 3;
    int it = claim(blockIdx.x * GPB + gib);
    if constexpr (PF) {
        if (it < n) prefetch_first<C>(p, item(it), smem, lg, gmask);
    }
    while (it < n) {
        const int itn = claim(it + ngroups);
        if (lg == 0) *next_it = itn;
        assemble_one<T, GR, GC, NTP, NRHS, P, Q, MIXED, SMEM, PF>(p, item(it), PF ? item(itn) : -1,
                                                                  smem, lg, gmask);
        it = *next_it;
        __syncwarp(gmask);  // read before the next call overwrites it
    }
}

}  // namespace rbfb
