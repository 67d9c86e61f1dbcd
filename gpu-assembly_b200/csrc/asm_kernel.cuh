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
//   gather   lanes load ja and the neighbour coordinates (FP64), shift to the
//            centre (minimum image in a periodic box) and take the group max
//            of the binary exponents for the power-of-two radius scale;
//   fill     phi for each unordered node pair once, monomials per node, the
//            right-hand sides per row: all FP64, written (rounded to T) into
//            a shared-memory staging matrix S, then vector-loaded into the
//            row registers;
//   factor   per step c (fully unrolled, all register indices static):
//            redux.max over the group on the |a(r,c)| bit patterns of unused
//            rows, redux.min on the row index among the maxima (ties go to
//            the lowest row, as in the oracle); the pivot row's owner lanes
//            write it to a double-buffered shared row, __syncwarp, every lane
//            reads it back (broadcast); l = a(r,c) * (1/pivot) for unused rows
//            (0 otherwise); a(r,j) = fma(-l, u(j), a(r,j)) for j > c and for
//            the right-hand sides; l is kept in a(r,c) (the L factor);
//   solve    the factors go back to S, the registers die; column-oriented
//            back substitution from S: x_c = y(p_c) * (1/pivot_c), then
//            y(r) = fma(-u(r,c), x_c, y(r)) for rows pivoted before c;
//   refine   (MIXED: factor in FP32) residual b - M x in FP64 from the FP64
//            phi cache and monomials in shared memory, correction through
//            the FP32 factors in S, x += d in FP64, until
//            max|d| <= tol * max|x| per right-hand side; a stencil that
//            stalls or runs out of sweeps is queued for the FP64 kernel;
//   scatter  weights of the k node unknowns, rescaled by 2^(-order*e), to
//            values[q][row offset + j] (coalesced over j).
#pragma once

#include <cstdint>

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
    double Lx, Ly;  // periods (<= 0: open axis)
    int scale;
    int nrhs;
    int col_op[kMaxRhs];  // RBFB_OP_* of every right-hand-side column
    int col_ic[kMaxRhs];  // interpolation point index of OP_INTERP columns
    const double* xc;
    const double* yc;
    double* values[kMaxRhs];
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

__device__ __forceinline__ unsigned group_mask(int G) {
    if (G == 32) return 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
}

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED>
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
    static constexpr int VEC = 16 / sizeof(T);
    static_assert(CW % VEC == 0, "register columns must tile the vector width");
    static constexpr int BW = ((NTP + NRHS + VEC - 1) / VEC) * VEC;  // pivot row buffer
    static constexpr int LDS = NTP;                                   // S row stride
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
    static constexpr int bytes = off_b64 + (MIXED ? al16(8 * NTP * NRHS) : 0);
    // S position of column c (de-interleaved by lane-column)
    static __device__ __forceinline__ int scol(int c) { return (c % GC) * CW + c / GC; }
};

// Packed index of the pair (i, j), i < j, of a k-node stencil.
__device__ __forceinline__ int tri(int i, int j, int k) {
    return i * (2 * k - i - 1) / 2 + (j - i - 1);
}
__device__ __forceinline__ double phi_at(const double* phi, int i, int j, int k) {
    return i == j ? 0.0 : (i < j ? phi[tri(i, j, k)] : phi[tri(j, i, k)]);
}

// Right-hand side q for node row (xi, yi) and for polynomial row m, FP64.
template <int P, int Q>
__device__ __forceinline__ double rhs_node(const AsmParams& p, int q, double xi, double yi, int e) {
    const int op = p.col_op[q];
    if (op == kOpInterp) {
        const double xe = scalbn(p.xc[p.col_ic[q]], -e);
        const double ye = scalbn(p.yc[p.col_ic[q]], -e);
        return phs64<Q>(dist2(dsub(xe, xi), dsub(ye, yi)));
    }
    return phs_op_origin<Q>(op, xi, yi);
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

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED>
__device__ __forceinline__ void assemble_one(const AsmParams& p, int s, char* smem, int lg,
                                             unsigned gmask) {
    using C = AsmCfg<T, GR, GC, NTP, NRHS, P, Q, MIXED>;
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
    const int off = p.ia ? p.ia[s] : s * p.k;
    const int ks = p.ia ? p.ia[s + 1] - off : p.k;
    const int n = NP + ks;

    // ---- gather + FP64 shift (+ minimum image), src/rbf_operators.h:354-358
    int e;
    {
        double gx[C::KPL], gy[C::KPL];
        int emax = -100000;
        const double x0 = p.x[s], y0 = p.y[s];
#pragma unroll
        for (int t = 0; t < C::KPL; ++t) {
            const int j = lg + t * G;
            gx[t] = 0.0;
            gy[t] = 0.0;
            if (j < ks) {
                const int nb = __ldg(p.ja + off + j);
                gx[t] = min_image(dsub(__ldg(p.x + nb), x0), p.Lx);
                gy[t] = min_image(dsub(__ldg(p.y + nb), y0), p.Ly);
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
    // phi block: each unordered pair once
    for (int i = 0; i < ks - 1; ++i) {
        const double xi = cx[i], yi = cy[i];
        for (int j = i + 1 + lg; j < ks; j += G) {
            const double v = phs64<Q>(dist2(dsub(cx[j], xi), dsub(cy[j], yi)));
            S[(NP + i) * LDS + C::scol(NP + j)] = static_cast<T>(v);
            S[(NP + j) * LDS + C::scol(NP + i)] = static_cast<T>(v);
            if constexpr (MIXED) phi[tri(i, j, ks)] = v;
        }
    }
    // everything else, one row per lane
    for (int r = lg; r < NTP; r += G) {
        T* Sr = S + r * LDS;
        if (r < NP) {
            // P^T row: zero block, node columns written by the node rows below
            for (int c = 0; c < NP; ++c) Sr[C::scol(c)] = T(0);
            for (int c = n; c < NTP; ++c) Sr[C::scol(c)] = T(0);
#pragma unroll
            for (int q = 0; q < NRHS; ++q) {
                const double v = q < p.nrhs ? rhs_poly<P>(p, q, r, e) : 0.0;
                X[r * NRHS + q] = static_cast<T>(v);
                if constexpr (MIXED) b64[r * NRHS + q] = v;
            }
        } else if (r < n) {
            const int i = r - NP;
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
            for (int c = n; c < NTP; ++c) Sr[C::scol(c)] = T(0);
#pragma unroll
            for (int q = 0; q < NRHS; ++q) {
                const double v = q < p.nrhs ? rhs_node<P, Q>(p, q, xi, yi, e) : 0.0;
                X[r * NRHS + q] = static_cast<T>(v);
                if constexpr (MIXED) b64[r * NRHS + q] = v;
            }
        } else {
            for (int c = 0; c < NTP; ++c) Sr[C::scol(c)] = (c == r) ? T(1) : T(0);
#pragma unroll
            for (int q = 0; q < NRHS; ++q) {
                X[r * NRHS + q] = T(0);
                if constexpr (MIXED) b64[r * NRHS + q] = 0.0;
            }
        }
    }
    __syncwarp(gmask);

    // ---- rows into registers (vector loads)
    T a[R][CW];
    T yv[R][NRHS];
    int pst[R];
    T dinv[R];
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        const int r = lr + GR * sl;
        const T* Sr = S + r * LDS + lc * CW;
#pragma unroll
        for (int cl = 0; cl < CW; cl += VEC) {
            if constexpr (VEC == 4) {
                const float4 v = *reinterpret_cast<const float4*>(Sr + cl);
                a[sl][cl] = v.x; a[sl][cl + 1] = v.y; a[sl][cl + 2] = v.z; a[sl][cl + 3] = v.w;
            } else {
                const double2 v = *reinterpret_cast<const double2*>(Sr + cl);
                a[sl][cl] = v.x; a[sl][cl + 1] = v.y;
            }
        }
#pragma unroll
        for (int q = 0; q < NRHS; ++q) yv[sl][q] = X[r * NRHS + q];
        pst[sl] = kFree;
        dinv[sl] = T(0);
    }

    // ---- elimination with row-implicit partial pivoting
    int info = 0;
#pragma unroll
    for (int c = 0; c < NTP; ++c) {
        const int lcc = c % GC, clc = c / GC;
        T* B = buf + (c & 1) * BW;
        // 1. pivot search
        int prow;
        bool zero_pivot;
        if constexpr (sizeof(T) == 4) {
            uint32_t best = 0;
            if (lc == lcc) {
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    const uint32_t kk =
                        (pst[sl] == kFree) ? __float_as_uint(fabsf(a[sl][clc])) + 1u : 0u;
                    best = max(best, kk);
                }
            }
            const uint32_t m = __reduce_max_sync(gmask, best);
            uint32_t cand = 0xffffffffu;
            if (lc == lcc) {
#pragma unroll
                for (int sl = R - 1; sl >= 0; --sl) {
                    const uint32_t kk =
                        (pst[sl] == kFree) ? __float_as_uint(fabsf(a[sl][clc])) + 1u : 0u;
                    if (kk == m) cand = (uint32_t)(lr + GR * sl);
                }
            }
            prow = (int)__reduce_min_sync(gmask, cand);
            zero_pivot = (m <= 1u);
        } else {
            unsigned long long best = 0;
            if (lc == lcc) {
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    const unsigned long long kk =
                        (pst[sl] == kFree)
                            ? (unsigned long long)__double_as_longlong(fabs((double)a[sl][clc])) + 1ull
                            : 0ull;
                    best = best > kk ? best : kk;
                }
            }
            const uint32_t mh = __reduce_max_sync(gmask, (uint32_t)(best >> 32));
            const uint32_t ml =
                __reduce_max_sync(gmask, ((uint32_t)(best >> 32) == mh) ? (uint32_t)best : 0u);
            const unsigned long long m = ((unsigned long long)mh << 32) | ml;
            uint32_t cand = 0xffffffffu;
            if (lc == lcc) {
#pragma unroll
                for (int sl = R - 1; sl >= 0; --sl) {
                    const unsigned long long kk =
                        (pst[sl] == kFree)
                            ? (unsigned long long)__double_as_longlong(fabs((double)a[sl][clc])) + 1ull
                            : 0ull;
                    if (kk == m) cand = (uint32_t)(lr + GR * sl);
                }
            }
            prow = (int)__reduce_min_sync(gmask, cand);
            zero_pivot = (m <= 1ull);
        }
        if (zero_pivot && info == 0) info = c + 1;
        const int plr = prow % GR, psl = prow / GR;

        // 2. pivot row to shared memory (owner lane-row), then broadcast
        if (lr == plr) {
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                if (sl == psl) {
#pragma unroll
                    for (int cl = (clc / VEC) * VEC; cl < CW; cl += VEC) {
                        if constexpr (VEC == 4) {
                            *reinterpret_cast<float4*>(B + lc * CW + cl) = make_float4(
                                a[sl][cl], a[sl][cl + 1], a[sl][cl + 2], a[sl][cl + 3]);
                        } else {
                            *reinterpret_cast<double2*>(B + lc * CW + cl) =
                                make_double2(a[sl][cl], a[sl][cl + 1]);
                        }
                    }
                    if (lc == 0) {
#pragma unroll
                        for (int q = 0; q < NRHS; ++q) B[NTP + q] = yv[sl][q];
                    }
                    pst[sl] = c;
                }
            }
        }
        __syncwarp(gmask);
        const T inv = T(1) / B[lcc * CW + clc];
        if (lr == plr) {
#pragma unroll
            for (int sl = 0; sl < R; ++sl)
                if (sl == psl) dinv[sl] = inv;
        }
        // 3. multipliers (kept as the L factor) and the update
        T l[R];
#pragma unroll
        for (int sl = 0; sl < R; ++sl) {
            T av = a[sl][clc];
            if constexpr (GC > 1) av = __shfl_sync(gmask, av, lr * GC + lcc, G);
            l[sl] = (pst[sl] == kFree) ? av * inv : T(0);
            if (lc == lcc && pst[sl] == kFree) a[sl][clc] = l[sl];
        }
#pragma unroll
        for (int cb = (clc / VEC) * VEC; cb < CW; cb += VEC) {
            T u[VEC];
            if constexpr (VEC == 4) {
                const float4 v4 = *reinterpret_cast<const float4*>(B + lc * CW + cb);
                u[0] = v4.x; u[1] = v4.y; u[2] = v4.z; u[3] = v4.w;
            } else {
                const double2 v2 = *reinterpret_cast<const double2*>(B + lc * CW + cb);
                u[0] = v2.x; u[1] = v2.y;
            }
#pragma unroll
            for (int t = 0; t < VEC; ++t) {
                const int cl = cb + t;
                if (cl < clc) continue;
                if (cl == clc) {
                    if constexpr (GC == 1) continue;
                    if (lc <= lcc) continue;
                }
#pragma unroll
                for (int sl = 0; sl < R; ++sl) a[sl][cl] = fma(-l[sl], u[t], a[sl][cl]);
            }
        }
#pragma unroll
        for (int q = 0; q < NRHS; ++q) {
            const T uq = B[NTP + q];
#pragma unroll
            for (int sl = 0; sl < R; ++sl) yv[sl][q] = fma(-l[sl], uq, yv[sl][q]);
        }
    }

    // ---- factors back to S (physical row layout); the registers die here
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        T* Sr = S + (lr + GR * sl) * LDS + lc * CW;
#pragma unroll
        for (int cl = 0; cl < CW; cl += VEC) {
            if constexpr (VEC == 4) {
                *reinterpret_cast<float4*>(Sr + cl) =
                    make_float4(a[sl][cl], a[sl][cl + 1], a[sl][cl + 2], a[sl][cl + 3]);
            } else {
                *reinterpret_cast<double2*>(Sr + cl) = make_double2(a[sl][cl], a[sl][cl + 1]);
            }
        }
    }
    __syncwarp(gmask);

    // column-oriented back substitution from S into X[c][q]
    auto back_substitute = [&](T (&yy)[R][NRHS]) {
#pragma unroll 1
        for (int c = NTP - 1; c >= 0; --c) {
#pragma unroll
            for (int sl = 0; sl < R; ++sl)
                if (pst[sl] == c && lc == 0) {
#pragma unroll
                    for (int q = 0; q < NRHS; ++q) X[c * NRHS + q] = yy[sl][q] * dinv[sl];
                }
            __syncwarp(gmask);
            T xq[NRHS];
#pragma unroll
            for (int q = 0; q < NRHS; ++q) xq[q] = X[c * NRHS + q];
            const int sc = C::scol(c);
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                const T u = S[(lr + GR * sl) * LDS + sc];
                const T m = (pst[sl] < c) ? u : T(0);
#pragma unroll
                for (int q = 0; q < NRHS; ++q) yy[sl][q] = fma(-m, xq[q], yy[sl][q]);
            }
        }
        __syncwarp(gmask);
    };
    back_substitute(yv);

    const int nrhs = p.nrhs;
    if constexpr (!MIXED) {
        // ---- scatter, src/rbf_operators.h:368-375
        const bool bad = info != 0;
        for (int q = 0; q < nrhs; ++q) {
            double* dst = p.values[q] + off;
            const int sh = -op_order(p.col_op[q]) * e;
            for (int j = lg; j < ks; j += G) {
                const double v = static_cast<double>(X[(NP + j) * NRHS + q]);
                dst[j] = bad ? __longlong_as_double(0x7ff8000000000000ll) : scalbn(v, sh);
            }
        }
        if (lg == 0 && p.info) p.info[s] = info;
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
                    for (int j = 0; j < ks; ++j) {
                        const double fv = phi_at(phi, i, j, ks);
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
                T* Z = buf + (t & 1) * BW;
#pragma unroll
                for (int sl = 0; sl < R; ++sl)
                    if (pst[sl] == t && lc == 0) {
#pragma unroll
                        for (int q = 0; q < NRHS; ++q) Z[q] = rv[sl][q];
                    }
                __syncwarp(gmask);
                T zq[NRHS];
#pragma unroll
                for (int q = 0; q < NRHS; ++q) zq[q] = Z[q];
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
            if (!(worst == worst)) failed = true;  // NaN
            else if (worst <= (float)p.ir_tol) converged = true;
            else if (sweeps >= 2 && worst > 0.5f * prev) failed = true;  // stalled
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
                double* dst = p.values[q] + off;
                const int sh = -op_order(p.col_op[q]) * e;
                for (int j = lg; j < ks; j += G) dst[j] = scalbn(x64[(NP + j) * NRHS + q], sh);
            }
            if (lg == 0 && p.info) p.info[s] = 0;
        }
    }
    __syncwarp(gmask);
}

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED, int BLOCK,
          int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) asm_kernel(AsmParams p) {
    using C = AsmCfg<T, GR, GC, NTP, NRHS, P, Q, MIXED>;
    constexpr int G = C::G;
    constexpr int GPB = BLOCK / G;  // groups per CTA
    extern __shared__ __align__(16) char smem_raw[];
    const int gib = threadIdx.x / G;
    const int lg = threadIdx.x % G;
    char* smem = smem_raw + gib * C::bytes;
    const unsigned gmask = group_mask(G);
    const int n = p.nitems_dev ? *p.nitems_dev : p.nitems;
    const int* list = (p.list && p.list_off_dev) ? p.list + *p.list_off_dev : p.list;
    if (p.work) {
        for (;;) {
            int it = 0;
            if (lg == 0) it = atomicAdd(p.work, 1);
            it = __shfl_sync(gmask, it, 0, G);
            if (it >= n) break;
            const int s = list ? list[it] : p.item_base + it;
            assemble_one<T, GR, GC, NTP, NRHS, P, Q, MIXED>(p, s, smem, lg, gmask);
        }
    } else {
        const int ngroups = gridDim.x * GPB;
        for (int it = blockIdx.x * GPB + gib; it < n; it += ngroups) {
            const int s = list ? list[it] : p.item_base + it;
            assemble_one<T, GR, GC, NTP, NRHS, P, Q, MIXED>(p, s, smem, lg, gmask);
        }
    }
}

}  // namespace rbfb
