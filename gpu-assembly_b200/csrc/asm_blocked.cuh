// asm_blocked.cuh -- batched RBF-FD assembly on sm_100a with the saddle-point
// system held in shared memory and factored by a blocked right-looking
// Gaussian elimination with row-implicit partial pivoting.
//
// Replaces assemble_interp_weights<Config> (src/rbf_operators.h:292-376),
// whose solve is cuSolverDx gesv_partial_pivot with one stencil per CTA.
//
// A group of G lanes owns one stencil: a warp (G = 32) or a half warp (G =
// 16, two stencils per warp, each step's shuffles and reductions over the
// half's lanes only, so the per-step instruction overhead is paid once for
// two stencils). A CTA holds BLOCK / G groups and the grid is persistent. The system is not padded: n = npoly(P) + k_s unknowns for the
// stencil's own k_s, any n <= NMAX. It is stored row-major in S (row =
// equation, column = unknown) with the NRHS right-hand sides as columns
// n .. n+NRHS-1, polynomial block first: equations [P^T rows (NP), node rows
// (k_s)], unknowns [lambda (NP), w (k_s)]. Rows are never swapped: piv[c] is
// the row that became the pivot row at step c, alive[r] is cleared then.
//
// The elimination runs in panels of PB columns. For panel [c0, c0+PB):
//   1. the rows not yet pivoted are listed in ascending order (act[]); lane
//      l takes list positions l, l+G, ... and loads their PB panel columns
//      into registers;
//   2. PB steps on the panel columns only. Step c: pivot = the unused row of
//      largest key (a 32-bit key: the magnitude word of a(r,c) without its 7
//      lowest bits, plus one, with 127 - list position in those bits, so ties
//      go to the lowest row -- the oracle's rule), found by one warp
//      group reduction whose operands were formed at the end of the previous step;
//      the pivot row's owner writes its whole panel row to S (final: L
//      multipliers left of c, the pivot, U right of it) and 1 / pivot (rounded
//      once, the oracle's reciprocal); every other unused row takes
//      l = a(r,c) * (1 / pivot) and a(r,j) = fma(-l, u(j), a(r,j)) for the
//      panel columns j > c;
//   3. rows still unused write their panel columns (now the L multipliers)
//      back to S;
//   4. the panel's pivot rows over the trailing columns (right-hand sides
//      included): row p_t takes the updates of steps t' < t, in order;
//   5. every unused row over the trailing columns: the PB updates of the
//      panel, in order, multipliers from registers, pivot-row values read
//      once per column pair and broadcast to the group.
// Every matrix and right-hand-side element receives exactly the fused
// multiply-adds of the unblocked elimination, in the same order, so the FP64
// result is bit-identical to the oracle's.
//
// Back substitution is column oriented, as the oracle's: lane l holds the
// transformed right-hand sides of the rows pivoted at steps l, l+G, ...;
// for c = n-1 .. 0 the owner of step c forms x_c = y * (1 / pivot_c) and
// broadcasts it by shuffle, and the rows pivoted before c update with
// u(row, c).
#pragma once

#include <cstdint>

#include "asm_kernel.cuh"

namespace rbfb {

// Layout of one stencil's working set for systems of up to NMAX unknowns
// with up to KMAX neighbours (shared memory, or a global scratch region).
template <typename T, int NMAX, int NRHS, int KMAX_, int PB, int G_ = 32, bool XBUF = true>
struct BlkLayout {
    static constexpr int G = G_;  // lanes per stencil: a warp, or half of one
    static constexpr int KMAX = KMAX_;
    static constexpr int R = (NMAX + G - 1) / G;  // list positions per lane
    static constexpr int VE = 16 / (int)sizeof(T);  // elements per 16-byte vector
    static_assert(PB % VE == 0, "panels are whole vectors");
    static_assert(NMAX <= 128, "pivot keys carry the list position in 7 bits");
    static_assert(G == 32 || G == 16, "a stencil takes a warp or a half warp");
    static_assert(R <= 4, "the substitutions walk at most four step segments");
    static constexpr int WMAX = NMAX + NRHS;  // columns: unknowns + right-hand sides
    // Row stride in vectors: odd, so the 32 rows a warp reads down one column
    // fall in different bank groups (4 wavefronts for 32 vectors).
    static constexpr int LV0 = (WMAX + VE - 1) / VE;
    static constexpr int LDSV = (LV0 % 2) ? LV0 : LV0 + 1;
    static constexpr int LDS = LDSV * VE;
    static_assert(((NMAX + PB - 1) / PB) * PB <= LDS, "a row holds every panel's columns");
    static constexpr int al16(int b) { return (b + 15) & ~15; }
    static constexpr int off_cx = 0;
    static constexpr int off_cy = off_cx + al16(8 * KMAX);
    static constexpr int off_s = off_cy + al16(8 * KMAX);
    static constexpr int off_x = off_s + al16(NMAX * LDS * (int)sizeof(T));
    // the solution X (the refined form's sweeps read it; the FP64 form keeps
    // it in registers and has no X)
    static constexpr int off_end = off_x + (XBUF ? al16(NMAX * NRHS * (int)sizeof(T)) : 0);
    // The elimination's bookkeeping (the list of unused rows, their flags,
    // the pivot order) and the next stencil's prefetched ja row. In the FP64
    // form they share the neighbour-coordinate slots, which are idle from
    // the end of the fill until the next stencil's coordinates are fetched
    // (after the pivot order has been read by the back substitution); the
    // refined form, whose sweeps read the pivot order again, keeps them apart.
    static constexpr int BOOK = al16(4 * NMAX) + al16(NMAX) + al16(4 * NMAX) + al16(4 * KMAX);
    static constexpr bool SHARE = !XBUF && BOOK <= off_s;
    static constexpr int off_act = SHARE ? off_cx : off_end;
    static constexpr int off_alive = off_act + al16(4 * NMAX);
    static constexpr int off_piv = off_alive + al16(NMAX);
    static constexpr int off_nja = off_piv + al16(4 * NMAX);
    // next stencil's centre (x, y) and CSR bounds ia[s], ia[s + 1] (+ size,
    // next item)
    static constexpr int off_nxy = SHARE ? off_end : off_nja + al16(4 * KMAX);
    static constexpr int off_nia = off_nxy + 16;
    // 1 / pivot of every step, written by the step's owner and read by all
    // lanes (a shared-memory broadcast measured faster than a shuffle in the
    // uneven kernel) and by the back substitution
    static constexpr int off_pinv = off_nia + 16;
    static constexpr int bytes = off_pinv + al16(NMAX * (int)sizeof(T));
};

template <typename T, int NMAX, int NRHS, int P, int Q, bool MIXED, int PB, int G_ = 32>
struct BlkCfg : BlkLayout<T, NMAX, NRHS, NMAX - npoly(P), PB, G_, MIXED> {
    using L = BlkLayout<T, NMAX, NRHS, NMAX - npoly(P), PB, G_, MIXED>;
    static_assert(MIXED ? sizeof(T) == 4 : sizeof(T) == 8,
                  "FP64 factors for the plain form, FP32 factors for the refined one");
    static constexpr int NP = npoly(P);
    // FP64 copies the refinement reads (MIXED only): phi (packed strict upper
    // triangle of the node block), the monomials of the nodes, the solution
    // and the right-hand sides
    static constexpr int NPAIR = L::KMAX * (L::KMAX - 1) / 2;
    static constexpr int off_phi = L::bytes;
    static constexpr int off_pm = off_phi + (MIXED ? L::al16(8 * NPAIR) : 0);
    static constexpr int off_x64 = off_pm + (MIXED ? L::al16(8 * L::KMAX * NP) : 0);
    static constexpr int off_b64 = off_x64 + (MIXED ? L::al16(8 * NMAX * NRHS) : 0);
    static constexpr int bytes = off_b64 + (MIXED ? L::al16(8 * NMAX * NRHS) : 0);
};

// 16-byte vector moves between shared memory and register arrays.
__device__ __forceinline__ void ldv(const double* s, double* d) {
    const double2 v = *reinterpret_cast<const double2*>(s);
    d[0] = v.x;
    d[1] = v.y;
}
__device__ __forceinline__ void ldv(const float* s, float* d) {
    const float4 v = *reinterpret_cast<const float4*>(s);
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
    d[3] = v.w;
}
__device__ __forceinline__ void stv(double* s, const double* d) {
    *reinterpret_cast<double2*>(s) = make_double2(d[0], d[1]);
}
__device__ __forceinline__ void stv(float* s, const float* d) {
    *reinterpret_cast<float4*>(s) = make_float4(d[0], d[1], d[2], d[3]);
}

// The word a pivot key is made from: the high 32 bits of a binary64 value
// (sign, exponent, 20 leading mantissa bits), all 32 bits of a binary32 one.
__device__ __forceinline__ uint32_t hiword(double v) {
    return (uint32_t)((unsigned long long)__double_as_longlong(v) >> 32);
}
__device__ __forceinline__ uint32_t hiword(float v) { return __float_as_uint(v); }

// c0, c1 -= m * (b0, b1): one packed FP32 fused multiply-add of sm_100a
// (fma.rn.f32x2; each component rounded once, as fmaf).
__device__ __forceinline__ void fnma2(float m, float b0, float b1, float& c0, float& c1) {
    unsigned long long mm, bb, cc, d;
    const float nm = -m;
    asm("mov.b64 %0, {%1, %1};" : "=l"(mm) : "f"(nm));
    asm("mov.b64 %0, {%1, %2};" : "=l"(bb) : "f"(b0), "f"(b1));
    asm("mov.b64 %0, {%1, %2};" : "=l"(cc) : "f"(c0), "f"(c1));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(mm), "l"(bb), "l"(cc));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(c0), "=f"(c1) : "l"(d));
}

// c[j] = fma(-m, b[j], c[j]) for j0 <= j < END: FP64 one fused multiply-add
// each; FP32 in aligned pairs through fnma2.
template <int END>
__device__ __forceinline__ void fnma_range(double m, const double* b, double* c, int j0) {
#pragma unroll
    for (int j = j0; j < END; ++j) c[j] = fma(-m, b[j], c[j]);
}
template <int END>
__device__ __forceinline__ void fnma_range(float m, const float* b, float* c, int j0) {
    int j = j0;
    if (j & 1) {
        if (j < END) c[j] = fmaf(-m, b[j], c[j]);
        ++j;
    }
#pragma unroll
    for (; j + 1 < END; j += 2) fnma2(m, b[j], b[j + 1], c[j], c[j + 1]);
    if (j < END) c[j] = fmaf(-m, b[j], c[j]);
}

// ---- the phases of one stencil, shared by the fixed-shape and the uneven
// kernels. A stencil's working set (S, X, pinv, piv, act, alive, cx, cy) is
// in shared memory, or -- for the uneven kernel's large stencils -- in a
// global scratch region of the same layout.

// Gather + FP64 shift to the centre (x0, y0) (+ minimum image), and the
// power-of-two radius scale (src/rbf_operators.h:354-358): cx/cy receive the
// shifted, scaled coordinates of the ks neighbours (with PF they hold the
// raw prefetched ones on entry). Returns the scale exponent e.
template <int KMAX, bool PF, int G = 32>
__device__ __forceinline__ int gather_scale(const AsmParams& p, int off, int ks, double x0,
                                            double y0, double* cx, double* cy, int lane) {
    constexpr int KPL = (KMAX + G - 1) / G;
    double gx[KPL], gy[KPL];
    int emax = -100000;
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        const int j = lane + t * G;
        gx[t] = 0.0;
        gy[t] = 0.0;
        if (j < ks) {
            double xn, yn;
            if constexpr (PF) {
                xn = cx[j];
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
    int e = __reduce_max_sync(group_mask(G), emax);
    e = (p.scale && e > -100000) ? e : 0;
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        const int j = lane + t * G;
        if (j < ks) {
            cx[j] = scalbn(gx[t], -e);
            cy[j] = scalbn(gy[t], -e);
        }
    }
    __syncwarp(group_mask(G));
    return e;
}

// The augmented system in S (row stride LDS): phi block (each unordered pair
// once, a flat walk over the lanes), monomial rows and columns, zero
// polynomial block, right-hand sides as columns n .. n+NRHS-1 (fill_matrix /
// fill_rhs, src/rbf_operators.h:116-185).
// With phi != nullptr (the refined form) the FP64 values are also kept: phi
// (pair (i, j), i < j, at its number in row-major order of the strict upper
// triangle), pm[i*NP + m] (monomials of node i) and b64[r*NRHS + q].
template <typename T, int LDS, int NRHS, int P, int Q, int G = 32>
__device__ __forceinline__ void fill_system(const AsmParams& p, T* S, const double* cx,
                                            const double* cy, int ks, int e, int lane,
                                            double* phi = nullptr, double* pm = nullptr,
                                            double* b64 = nullptr) {
    constexpr int NP = npoly(P);
    const int n = NP + ks;
    {
        const int npair = ks * (ks - 1) / 2;
        int i = 0, j = 1 + lane;
        while (i < ks - 1 && j >= ks) {
            j += i + 2 - ks;
            ++i;
        }
        for (int t = lane; t < npair; t += G) {
            const double v64 = phs64<Q>(dist2(dsub(cx[j], cx[i]), dsub(cy[j], cy[i])));
            const T v = static_cast<T>(v64);
            S[(NP + i) * LDS + NP + j] = v;
            S[(NP + j) * LDS + NP + i] = v;
            if (phi) phi[t] = v64;
            j += G;
            while (i < ks - 1 && j >= ks) {
                j += i + 2 - ks;
                ++i;
            }
        }
    }
    for (int i = lane; i < ks; i += G) {
        const int r = NP + i;
        T* Sr = S + r * LDS;
        const double xi = cx[i], yi = cy[i];
        double mon[NP];
        monomials<P>(xi, yi, mon);
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            Sr[m] = static_cast<T>(mon[m]);
            S[m * LDS + r] = static_cast<T>(mon[m]);
            if (pm) pm[i * NP + m] = mon[m];
        }
        Sr[r] = T(0);
        double rv[NRHS];
        rhs_node<P, Q, NRHS>(p, xi, yi, e, rv);
#pragma unroll
        for (int q = 0; q < NRHS; ++q) {
            Sr[n + q] = static_cast<T>(rv[q]);
            if (b64) b64[r * NRHS + q] = rv[q];
        }
    }
    for (int f = lane; f < NP * NP; f += G) S[(f / NP) * LDS + f % NP] = T(0);
    for (int r = lane; r < NP; r += G) {
#pragma unroll
        for (int q = 0; q < NRHS; ++q) {
            const double v = q < p.nrhs ? rhs_poly<P>(p, q, r, e) : 0.0;
            S[r * LDS + n + q] = static_cast<T>(v);
            if (b64) b64[r * NRHS + q] = v;
        }
    }
}

// Blocked right-looking elimination of the n x n system in S with its NRHS
// right-hand-side columns (panels of PB; R list positions per lane, R*32 >=
// n). Returns info: 0, or c + 1 for the first zero pivot.
template <typename T, int R, int LDS, int NRHS, int PB, int G = 32>
__device__ __forceinline__ int eliminate_blocked(T* S, T* pinv, int* piv, int* act,
                                                 unsigned char* alive, int n, int lane) {
    constexpr int VE = 16 / (int)sizeof(T);
    const unsigned FULL = group_mask(G);  // the group's lanes
    const int gbase = (threadIdx.x & 31) & ~(G - 1);
    const int W = n + NRHS;  // columns in use
    int info = 0;
    for (int r = lane; r < n; r += G) alive[r] = 1;
    __syncwarp(group_mask(G));
#pragma unroll 1
    for (int c0 = 0; c0 < n; c0 += PB) {
        // 1. the unused rows, ascending, and this lane's panel rows
        int m = 0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int r = lane + G * j;
            const bool a = r < n && alive[r];
            const unsigned b = (__ballot_sync(FULL, a) & FULL) >> gbase;
            if (a) act[m + __popc(b & ((1u << lane) - 1u))] = r;
            m += __popc(b);
        }
        __syncwarp(group_mask(G));
        T a[R][PB];
        int arow[R];
        uint32_t kmask[R], kcon[R];
#pragma unroll
        for (int sl = 0; sl < R; ++sl) {
            const int pos = lane + G * sl;
            const bool v = pos < m;
            arow[sl] = v ? act[pos] : 0;
            kmask[sl] = v ? 0x7fffff80u : 0u;
            kcon[sl] = v ? 255u - (uint32_t)pos : 0u;
            const T* src = S + arow[sl] * LDS + c0;
#pragma unroll
            for (int v4 = 0; v4 < PB; v4 += VE) ldv(src + v4, &a[sl][v4]);
        }
        const int tend = min(PB, n - c0);  // steps in this panel
        // look-ahead operands of the pivot search of the panel's first column:
        // this lane's best key and its candidate value
        uint32_t pkey;
        T pbv;
        auto keys = [&](int t) {
            uint32_t best = 0;
            T bv = T(1);
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                const uint32_t kk = (hiword(a[sl][t]) & kmask[sl]) + kcon[sl];
                if (kk > best) {
                    best = kk;
                    bv = a[sl][t];
                }
            }
            pkey = best;
            pbv = bv;
        };
        keys(0);
        // the reduction of step t is issued as soon as column t is updated
        // (at the end of step t - 1), ahead of the rest of that update
        uint32_t mk_next = __reduce_max_sync(FULL, pkey);
        // 2. the panel's steps
#pragma unroll
        for (int t = 0; t < PB; ++t) {
            if (t < tend) {
                const int c = c0 + t;
                const uint32_t mk = mk_next;
                // the oracle's 1 / pivot, if this lane owns the pivot
                const T pinvl = recip_rn(pbv);
                if (mk < 256u && info == 0) info = c + 1;  // zero pivot column
                const int pos = 127 - (int)(mk & 127u);
                const int owner = pos & (G - 1), osl = pos / G;
                if (lane == owner) {
#pragma unroll
                    for (int sl = 0; sl < R; ++sl) {
                        if (sl == osl) {
                            T* dst = S + arow[sl] * LDS + c0;
#pragma unroll
                            for (int v4 = 0; v4 < PB; v4 += VE) stv(dst + v4, &a[sl][v4]);
                            piv[c] = arow[sl];
                            alive[arow[sl]] = 0;
                            kmask[sl] = 0u;
                            kcon[sl] = 0u;
                        }
                    }
                    pinv[c] = pinvl;
                }
                __syncwarp(group_mask(G));
                const T inv = pinv[c];
                const T* U = S + piv[c] * LDS + c0;
                // multipliers of the unused rows (0 for the others)
                T l[R];
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    l[sl] = kmask[sl] ? a[sl][t] * inv : T(0);
                    a[sl][t] = l[sl];
                }
                // the panel columns right of c: column c + 1 first, then the
                // next pivot search, then the rest
                if (t + 1 < PB) {
                    T u[PB];
#pragma unroll
                    for (int v4 = ((t + 1) / VE) * VE; v4 < PB; v4 += VE) ldv(U + v4, &u[v4]);
#pragma unroll
                    for (int sl = 0; sl < R; ++sl) a[sl][t + 1] = fma(-l[sl], u[t + 1], a[sl][t + 1]);
                    if (t + 1 < tend) {
                        keys(t + 1);
                        mk_next = __reduce_max_sync(FULL, pkey);
                    }
#pragma unroll
                    for (int sl = 0; sl < R; ++sl) fnma_range<PB>(l[sl], u, a[sl], t + 2);
                }
            }
        }
        // 3. rows still unused: their L multipliers back to S
#pragma unroll
        for (int sl = 0; sl < R; ++sl) {
            if (kmask[sl]) {
                T* dst = S + arow[sl] * LDS + c0;
#pragma unroll
                for (int v4 = 0; v4 < PB; v4 += VE) stv(dst + v4, &a[sl][v4]);
            }
        }
        __syncwarp(group_mask(G));
        const int jt = c0 + PB;  // first trailing column
        if (jt >= W) break;
        const int nv = (W - jt + VE - 1) / VE;  // trailing column vectors
        int prw[PB];
#pragma unroll
        for (int t = 0; t < PB; ++t) prw[t] = piv[c0 + (t < tend ? t : 0)];
        // 4. the panel's pivot rows over the trailing columns
        for (int v = lane; v < nv; v += G) {
            const int col = jt + v * VE;
            T u[PB][VE];
#pragma unroll
            for (int t = 0; t < PB; ++t) {
                if (t < tend) {
                    ldv(S + prw[t] * LDS + col, u[t]);
#pragma unroll
                    for (int tp = 0; tp < t; ++tp) {
                        const T lv = S[prw[t] * LDS + c0 + tp];
                        fnma_range<VE>(lv, u[tp], u[t], 0);
                    }
                    stv(S + prw[t] * LDS + col, u[t]);
                }
            }
        }
        __syncwarp(group_mask(G));
        // 5. the unused rows over the trailing columns (all lanes walk the same
        // columns: the pivot-row values are broadcast loads)
        if (m > tend) {
            bool any[R];
#pragma unroll
            for (int sl = 0; sl < R; ++sl) any[sl] = __any_sync(FULL, kmask[sl] != 0u);
            // two column vectors per iteration: independent FMA chains
#pragma unroll 2
            for (int v = 0; v < nv; ++v) {
                const int col = jt + v * VE;
                T u[PB][VE];
#pragma unroll
                for (int t = 0; t < PB; ++t) ldv(S + prw[t] * LDS + col, u[t]);
#pragma unroll
                for (int sl = 0; sl < R; ++sl) {
                    if (any[sl]) {
                        T* cp = S + arow[sl] * LDS + col;
                        T cv[VE];
                        ldv(cp, cv);
#pragma unroll
                        for (int t = 0; t < PB; ++t) fnma_range<VE>(a[sl][t], u[t], cv, 0);
                        if (kmask[sl]) stv(cp, cv);
                    }
                }
            }
            __syncwarp(group_mask(G));
        }
    }
    return info;
}

// Column-oriented back substitution (the oracle's order): lane l holds the
// transformed right-hand sides of the rows pivoted at steps l, l + G, ...;
// for c = n-1 .. 0 the owner of step c forms x_c = y * (1 / pivot_c) and
// broadcasts it by shuffle, and the rows pivoted before c update with
// u(row, c). The owner keeps x_c: xs[sl][q] of lane l is component
// l + G*sl. With TOX, X[c*NRHS + q] also receives x_c. Each lane reads
// 1 / pivot of its own steps up front, and `after_loads` runs once the pivot
// order has been read (it may reuse the bookkeeping slots). Steps below `cstop` are not
// taken: x_c depends only on the x of later steps, so a caller that needs
// the unknowns cstop .. n-1 alone (the weights, after the polynomial
// multipliers) gets them unchanged.
struct NoHook {
    __device__ void operator()() const {}
};
template <typename T, int R, int LDS, int NRHS, int G = 32, bool TOX = true, class Hook = NoHook>
__device__ __forceinline__ void back_substitute_blk(const T* S, const int* piv, const T* pinv,
                                                    T* X, int n,
                                                    int lane, T (&xs)[R][NRHS],
                                                    Hook after_loads = Hook{}, int cstop = 0) {
    const unsigned FULL = group_mask(G);
    T y[R][NRHS];
#pragma unroll
    for (int sl = 0; sl < R; ++sl)
#pragma unroll
        for (int q = 0; q < NRHS; ++q) xs[sl][q] = T(0);
    int prow_t[R];
    T dvown[R];  // 1 / pivot of this lane's steps
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        const int t = lane + G * sl;
        prow_t[sl] = t < n ? piv[t] : 0;
#pragma unroll
        for (int q = 0; q < NRHS; ++q) y[sl][q] = t < n ? S[prow_t[sl] * LDS + n + q] : T(0);
        dvown[sl] = t < n ? pinv[t] : T(0);
    }
    __syncwarp(group_mask(G));
    after_loads();
    // Steps in segments of G from the last: in segment OS the owner of step c
    // holds it in slot OS (static), the slots below OS hold steps all before
    // c (updated unconditionally), the slots above OS steps all after it.
    // The column of S of step c - 1 is loaded during step c, so only the
    // multiply -> shuffle -> fma chain is serial.
    auto segment = [&](auto os_c) {
        constexpr int OS = decltype(os_c)::value;
        const int ctop = min(n, G * (OS + 1)) - 1;
        const int cend = max(G * OS, cstop);  // last step of the segment
        if (ctop < cend) return;
        T un[OS + 1];
#pragma unroll
        for (int sl = 0; sl <= OS; ++sl) un[sl] = S[prow_t[sl] * LDS + ctop];
#pragma unroll 1
        for (int c = ctop; c >= cend; --c) {
            T uc[OS + 1];
#pragma unroll
            for (int sl = 0; sl <= OS; ++sl) uc[sl] = un[sl];
            if (c > cend) {
#pragma unroll
                for (int sl = 0; sl <= OS; ++sl) un[sl] = S[prow_t[sl] * LDS + c - 1];
            }
            T xq[NRHS];
            const bool own = lane == c - G * OS;
#pragma unroll
            for (int q = 0; q < NRHS; ++q) {
                const T v = y[OS][q] * dvown[OS];  // the owner's value is x_c
                xq[q] = __shfl_sync(FULL, v, c - G * OS, G);
                if (own) xs[OS][q] = v;
            }
            if (TOX && lane == 0) {
#pragma unroll
                for (int q = 0; q < NRHS; ++q) X[c * NRHS + q] = xq[q];
            }
#pragma unroll
            for (int sl = 0; sl <= OS; ++sl) {
                const T u = (sl == OS && lane + G * sl >= c) ? T(0) : uc[sl];
                fnma_range<NRHS>(u, xq, y[sl], 0);
            }
        }
    };
    if constexpr (R > 3) segment(std::integral_constant<int, 3>{});
    if constexpr (R > 2) segment(std::integral_constant<int, 2>{});
    if constexpr (R > 1) segment(std::integral_constant<int, 1>{});
    segment(std::integral_constant<int, 0>{});
    __syncwarp(group_mask(G));
}

// Forward substitution with the unit lower factor kept in S (the refined
// form): the right-hand sides in S's columns n .. n+NRHS-1, in row order, are
// replaced by L^-1 P b in the layout the elimination leaves them (row piv[t]
// holds component t). Lane l holds the components of steps l, l + G, ...;
// for c = 0 .. n-1 the owner of step c broadcasts it by shuffle and the rows
// pivoted after c update with their multiplier l(row, c) = S(row, c).
template <typename T, int R, int LDS, int NRHS, int G = 32>
__device__ __forceinline__ void forward_substitute_blk(T* S, const int* piv, int n, int lane) {
    const unsigned FULL = group_mask(G);
    T y[R][NRHS];
    int prow_t[R];
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        const int t = lane + G * sl;
        prow_t[sl] = t < n ? piv[t] : 0;
#pragma unroll
        for (int q = 0; q < NRHS; ++q) y[sl][q] = t < n ? S[prow_t[sl] * LDS + n + q] : T(0);
    }
    // segments of G steps from the first: in segment OS the owner of step c
    // holds it in slot OS, the slots above OS hold steps all after c
    auto segment = [&](auto os_c) {
        constexpr int OS = decltype(os_c)::value;
#pragma unroll 1
        for (int c = G * OS; c < min(n, G * (OS + 1)); ++c) {
            T z[NRHS];
#pragma unroll
            for (int q = 0; q < NRHS; ++q) z[q] = __shfl_sync(FULL, y[OS][q], c - G * OS, G);
#pragma unroll
            for (int sl = OS; sl < R; ++sl) {
                T l = S[prow_t[sl] * LDS + c];
                if (sl == OS) l = (lane + G * sl > c) ? l : T(0);
                fnma_range<NRHS>(l, z, y[sl], 0);
            }
        }
    };
    segment(std::integral_constant<int, 0>{});
    if constexpr (R > 1) segment(std::integral_constant<int, 1>{});
    if constexpr (R > 2) segment(std::integral_constant<int, 2>{});
    if constexpr (R > 3) segment(std::integral_constant<int, 3>{});
#pragma unroll
    for (int sl = 0; sl < R; ++sl) {
        if (lane + G * sl < n) {
#pragma unroll
            for (int q = 0; q < NRHS; ++q) S[prow_t[sl] * LDS + n + q] = y[sl][q];
        }
    }
    __syncwarp(group_mask(G));
}

// Packed index of the pair (i, j), i < j, of a k-node stencil.
__device__ __forceinline__ int tri_idx(int i, int j, int k) {
    return i * (2 * k - i - 1) / 2 + (j - i - 1);
}

// FP64 residual b - M x of the refined form, from the FP64 copies, rounded to
// T into S's right-hand-side columns (row order).
template <typename T, int LDS, int NRHS, int NP, int G = 32>
__device__ __forceinline__ void residual_blk(T* S, const double* phi, const double* pm,
                                             const double* x64, const double* b64, int ks,
                                             int lane) {
    const int n = NP + ks;
    for (int r = lane; r < n; r += G) {
        double acc[NRHS];
#pragma unroll
        for (int q = 0; q < NRHS; ++q) acc[q] = b64[r * NRHS + q];
        if (r < NP) {
            for (int j = 0; j < ks; ++j) {
                const double mv = pm[j * NP + r];
#pragma unroll
                for (int q = 0; q < NRHS; ++q) acc[q] = fma(-mv, x64[(NP + j) * NRHS + q], acc[q]);
            }
        } else {
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
                for (int q = 0; q < NRHS; ++q) acc[q] = fma(-fv, x64[(NP + j) * NRHS + q], acc[q]);
            }
            const double* prow_i = phi + (i < ks - 1 ? tri_idx(i, i + 1, ks) : 0);
            for (int j = i + 1; j < ks; ++j) {
                const double fv = prow_i[j - i - 1];
#pragma unroll
                for (int q = 0; q < NRHS; ++q) acc[q] = fma(-fv, x64[(NP + j) * NRHS + q], acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < NRHS; ++q) S[r * LDS + n + q] = static_cast<T>(acc[q]);
    }
    __syncwarp(group_mask(G));
}

// Scatter of the k node weights (unknowns NP .. NP+ks-1), rescaled,
// src/rbf_operators.h:368-375; NaN for a singular stencil; info. The
// solution comes from the lanes' registers (xs of back_substitute_blk):
// lane l writes the weights of unknowns l + G*sl.
template <typename T, int R, int NRHS, int G = 32>
__device__ __forceinline__ void scatter_regs(const AsmParams& p, const T (&xs)[R][NRHS], int np,
                                             int ks, int off, int e, int info, int s, int lane) {
    const bool bad = info != 0;
#pragma unroll
    for (int q = 0; q < NRHS; ++q) {
        if (q < p.nrhs) {
            double* dst = out_column(p, q) + off;
            const int sh = -op_order(p.col_op[q]) * e;
#pragma unroll
            for (int sl = 0; sl < R; ++sl) {
                const int j = lane + G * sl - np;
                if (j >= 0 && j < ks)
                    dst[j] = bad ? __longlong_as_double(0x7ff8000000000000ll)
                                 : scalbn(static_cast<double>(xs[sl][q]), sh);
            }
        }
    }
    if (lane == 0 && p.info) p.info[s - p.row_base] = info;
    __syncwarp(group_mask(G));
}

template <typename T, int NMAX, int NRHS, int P, int Q, bool MIXED, int PB, bool PF, int GW = 32>
__device__ __forceinline__ void assemble_blk(const AsmParams& p, int s, int sn, char* smem,
                                             int lane) {
    using C = BlkCfg<T, NMAX, NRHS, P, Q, MIXED, PB, GW>;
    constexpr int G = C::G, NP = C::NP, R = C::R, LDS = C::LDS;
    double* cx = reinterpret_cast<double*>(smem + C::off_cx);
    double* cy = reinterpret_cast<double*>(smem + C::off_cy);
    T* S = reinterpret_cast<T*>(smem + C::off_s);
    T* X = MIXED ? reinterpret_cast<T*>(smem + C::off_x) : nullptr;
    int* piv = reinterpret_cast<int*>(smem + C::off_piv);
    int* act = reinterpret_cast<int*>(smem + C::off_act);
    unsigned char* alive = reinterpret_cast<unsigned char*>(smem + C::off_alive);
    int* nja = reinterpret_cast<int*>(smem + C::off_nja);
    double* nxy = reinterpret_cast<double*>(smem + C::off_nxy);
    int* nia = reinterpret_cast<int*>(smem + C::off_nia);
    double* phi = MIXED ? reinterpret_cast<double*>(smem + C::off_phi) : nullptr;
    double* pm = MIXED ? reinterpret_cast<double*>(smem + C::off_pm) : nullptr;
    double* x64 = MIXED ? reinterpret_cast<double*>(smem + C::off_x64) : nullptr;
    double* b64 = MIXED ? reinterpret_cast<double*>(smem + C::off_b64) : nullptr;

    // With PF, stencil s was prefetched (by the previous call of this warp, or
    // by prefetch_first): its neighbour coordinates wait in cx/cy (raw), its
    // centre in nxy, its CSR bounds in nia. Without PF everything comes from
    // global memory.
    int off, ks;
    double x0, y0;
    if constexpr (PF) {
        cp_async_wait_all();
        __syncwarp(group_mask(G));
        x0 = nxy[0];
        y0 = nxy[1];
        off = p.ia ? nia[0] : (s - p.row_base) * p.k;
        ks = p.ia ? nia[1] - off : p.k;
        __syncwarp(group_mask(G));  // read before the slots are refilled below
    } else {
        x0 = p.x[s];
        y0 = p.y[s];
        off = p.ia ? p.ia[s] : (s - p.row_base) * p.k;
        ks = p.ia ? p.ia[s + 1] - off : p.k;
    }
    const int n = NP + ks;
    if (PF && sn >= 0 && lane == 0) {  // prefetch stage 1: next centre and CSR bounds
        cp_async8(nxy, p.x + sn);
        cp_async8(nxy + 1, p.y + sn);
        if (p.ia) {
            cp_async4(nia, p.ia + sn);
            cp_async4(nia + 1, p.ia + sn + 1);
        }
    }
    const int e = gather_scale<C::KMAX, PF, G>(p, off, ks, x0, y0, cx, cy, lane);
    fill_system<T, LDS, NRHS, P, Q, G>(p, S, cx, cy, ks, e, lane, phi, pm, b64);
    // the coordinate slots are read: with C::SHARE the bookkeeping and the
    // next ja row may now take them
    __syncwarp(group_mask(G));

    // prefetch stage 2: the next stencil's ja row (its bounds have landed)
    if constexpr (PF) {
        int offn = 0, ksn = 0;
        if (sn >= 0) {
            if (p.ia) {
                cp_async_wait_all();
                __syncwarp(group_mask(G));
                offn = nia[0];
                ksn = nia[1] - offn;
            } else {
                offn = (sn - p.row_base) * p.k;
                ksn = p.k;
            }
            for (int j = lane; j < ksn; j += G) cp_async4(nja + j, p.ja + offn + j);
        }
        __syncwarp(group_mask(G));
        if (lane == 0) nia[2] = ksn;
    }
    __syncwarp(group_mask(G));

    T* pinv = reinterpret_cast<T*>(smem + C::off_pinv);
    const int info = eliminate_blocked<T, R, LDS, NRHS, PB, G>(S, pinv, piv, act, alive, n, lane);

    // prefetch stage 3: the next stencil's neighbour coordinates into cx/cy,
    // once the back substitution has read the pivot order: every lane reads
    // its ja slots first, then the copies may land on the shared slots
    auto stage3 = [&]() {
        if constexpr (PF) {
            constexpr int KPL = (C::KMAX + G - 1) / G;
            const int ksn = nia[2];
            if (ksn > 0) {
                cp_async_wait_all();
                int nb[KPL];
#pragma unroll
                for (int t = 0; t < KPL; ++t) {
                    const int j = lane + G * t;
                    nb[t] = j < ksn ? nja[j] : 0;
                }
                __syncwarp(group_mask(G));
#pragma unroll
                for (int t = 0; t < KPL; ++t) {
                    const int j = lane + G * t;
                    if (j < ksn) {
                        cp_async8(cx + j, p.x + nb[t]);
                        cp_async8(cy + j, p.y + nb[t]);
                    }
                }
            }
        }
    };
    T xs[R][NRHS];
    // the FP64 form needs the weights alone (unknowns NP .. n-1); the refined
    // form's residual needs every unknown
    back_substitute_blk<T, R, LDS, NRHS, G, MIXED>(S, piv, pinv, X, n, lane, xs, stage3,
                                                   MIXED ? 0 : NP);
    if constexpr (!MIXED) {
        scatter_regs<T, R, NRHS, G>(p, xs, NP, ks, off, e, info, s, lane);
    } else {
        // ---- FP64 iterative refinement with the FP32 factors
        for (int i = lane; i < n * NRHS; i += G) x64[i] = static_cast<double>(X[i]);
        __syncwarp(group_mask(G));
        int sweeps = 0;
        bool converged = false, failed = (info != 0);
        float prev = 3.4e38f;
        while (!converged && !failed) {
            if (sweeps >= p.max_sweeps) {
                failed = true;
                break;
            }
            ++sweeps;
            residual_blk<T, LDS, NRHS, NP, G>(S, phi, pm, x64, b64, ks, lane);
            forward_substitute_blk<T, R, LDS, NRHS, G>(S, piv, n, lane);
            back_substitute_blk<T, R, LDS, NRHS, G, true>(S, piv, pinv, X, n, lane, xs);
            // x += d; convergence on max|d| / max|x| per right-hand side
            float worst = 0.f;
            for (int q = 0; q < p.nrhs; ++q) {
                float dmax = 0.f, xmax = 0.f;
                for (int i = lane; i < n; i += G) {
                    const double d = static_cast<double>(X[i * NRHS + q]);
                    const double xn = x64[i * NRHS + q] + d;
                    x64[i * NRHS + q] = xn;
                    dmax = fmaxf(dmax, (float)fabs(d));
                    xmax = fmaxf(xmax, (float)fabs(xn));
                }
                dmax = __uint_as_float(__reduce_max_sync(group_mask(G), __float_as_uint(dmax)));
                xmax = __uint_as_float(__reduce_max_sync(group_mask(G), __float_as_uint(xmax)));
                worst = fmaxf(worst, xmax > 0.f ? dmax / xmax : dmax);
            }
            __syncwarp(group_mask(G));
            // The correction of sweep k measures the error before it (tau_k);
            // the error left after it is about tau_k * rho / (1 - rho) with
            // rho = tau_k / tau_(k-1) the observed contraction (about
            // cond(M) * 2^-24). Converged when that prediction is below tol
            // (or the correction itself is at the FP64 floor). A contraction
            // above 0.1 means cond(M) > ~1e6: the prediction is unreliable
            // there and the FP64 rounding floor of the system itself nears the
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
        if (lane == 0) {
            if (p.sweeps_sum) atomicAdd(p.sweeps_sum, (unsigned long long)sweeps);
            if (p.sweeps_max) atomicMax(p.sweeps_max, sweeps);
        }
        if (failed) {
            if (lane == 0) {
                const int fo = p.list_off_dev ? *p.list_off_dev : 0;
                p.fb_list[fo + atomicAdd(p.fb_count, 1)] = s;
            }
        } else {
            for (int q = 0; q < p.nrhs; ++q) {
                double* dst = out_column(p, q) + off;
                const int sh = -op_order(p.col_op[q]) * e;
                for (int j = lane; j < ks; j += G) dst[j] = scalbn(x64[(NP + j) * NRHS + q], sh);
            }
            if (lane == 0 && p.info) p.info[s - p.row_base] = 0;
        }
        __syncwarp(group_mask(G));
    }
}

// The prefetch of a group's first stencil, done up front: centre and CSR
// bounds, then the ja row, then the neighbour coordinates into cx/cy (every
// lane reads its ja slots before any copy may land on shared slots).
template <class C>
__device__ __forceinline__ void prefetch_first_blk(const AsmParams& p, int s, char* smem,
                                                   int lane) {
    constexpr int G = C::G, KPL = (C::KMAX + G - 1) / G;
    double* cx = reinterpret_cast<double*>(smem + C::off_cx);
    double* cy = reinterpret_cast<double*>(smem + C::off_cy);
    int* nja = reinterpret_cast<int*>(smem + C::off_nja);
    double* nxy = reinterpret_cast<double*>(smem + C::off_nxy);
    int* nia = reinterpret_cast<int*>(smem + C::off_nia);
    if (lane == 0) {
        cp_async8(nxy, p.x + s);
        cp_async8(nxy + 1, p.y + s);
        if (p.ia) {
            cp_async4(nia, p.ia + s);
            cp_async4(nia + 1, p.ia + s + 1);
        }
    }
    cp_async_wait_all();
    __syncwarp(group_mask(G));
    const int off = p.ia ? nia[0] : (s - p.row_base) * p.k;
    const int ks = p.ia ? nia[1] - off : p.k;
    for (int j = lane; j < ks; j += G) cp_async4(nja + j, p.ja + off + j);
    cp_async_wait_all();
    int nb[KPL];
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        const int j = lane + G * t;
        nb[t] = j < ks ? nja[j] : 0;
    }
    __syncwarp(group_mask(G));
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        const int j = lane + G * t;
        if (j < ks) {
            cp_async8(cx + j, p.x + nb[t]);
            cp_async8(cy + j, p.y + nb[t]);
        }
    }
}

template <typename T, int NMAX, int NRHS, int P, int Q, bool MIXED, int BLOCK, int MINB, int PB,
          bool PF, int GW = 32>
__global__ void __launch_bounds__(BLOCK, MINB) blk_kernel(AsmParams p) {
    using C = BlkCfg<T, NMAX, NRHS, P, Q, MIXED, PB, GW>;
    constexpr int G = C::G;
    const unsigned gmask = group_mask(G);
    constexpr int GPB = BLOCK / G;  // warps (stencils in flight) per CTA
    extern __shared__ __align__(16) char smem_raw[];
    const int gib = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    char* smem = smem_raw + gib * C::bytes;
    const int n = p.nitems_dev ? *p.nitems_dev : p.nitems;
    const int* list = (p.list && p.list_off_dev) ? p.list + *p.list_off_dev : p.list;
    const int ngroups = gridDim.x * GPB;
    auto claim = [&](int next_static) {
        if (!p.work) return next_static;
        int v = 0;
        if (lane == 0) v = atomicAdd(p.work, 1);
        return __shfl_sync(gmask, v, 0, G);
    };
    auto item = [&](int i) { return i < n ? (list ? list[i] : p.item_base + i) : -1; };
    // One call site: the stencil body is inlined once. With PF each call
    // also prefetches the next item's data (claimed one ahead).
    int* next_it = reinterpret_cast<int*>(smem + C::off_nia) + 3;
    int it = claim(blockIdx.x * GPB + gib);
    if constexpr (PF) {
        if (it < n) prefetch_first_blk<C>(p, item(it), smem, lane);
    }
    while (it < n) {
        const int itn = claim(it + ngroups);
        if (lane == 0) *next_it = itn;
        assemble_blk<T, NMAX, NRHS, P, Q, MIXED, PB, PF, GW>(p, item(it), PF ? item(itn) : -1, smem,
                                                             lane);
        it = *next_it;
        __syncwarp(group_mask(G));
    }
}

// ---- one persistent launch for an uneven batch ------------------------------
//
// Ragged stencils in CSR form, each with its own size k_s = ia[s+1] - ia[s],
// degree P_s (degree[s], or P0 for all) and PHS exponent Q_s = phs, or
// 2 P_s - 1 when phs = 0: the reference's one-grid-over-all-stencils launch
// (src/rbf_operators.h:197-200,340) for stencils of any mix of shapes. Warps
// claim stencils from one device work counter. A system of up to NS unknowns
// is solved in the warp's shared-memory slot; a larger one (up to NG) in the
// warp's region of a global scratch buffer, which stays in L2. Supported:
// P_s in 1..4 and Q_s in {3, 5, 7, 9}; a stencil outside that (or above NG
// unknowns, or with no neighbour) sets *err and is skipped.

// Runtime-Q dispatch of the fill (the elimination does not depend on P or Q).
template <typename T, int LDS, int NRHS, int P>
__device__ __forceinline__ void fill_system_q(const AsmParams& p, int Q, T* S, const double* cx,
                                              const double* cy, int ks, int e, int lane) {
    switch (Q) {
        case 3: fill_system<T, LDS, NRHS, P, 3>(p, S, cx, cy, ks, e, lane); break;
        case 5: fill_system<T, LDS, NRHS, P, 5>(p, S, cx, cy, ks, e, lane); break;
        case 7: fill_system<T, LDS, NRHS, P, 7>(p, S, cx, cy, ks, e, lane); break;
        default: fill_system<T, LDS, NRHS, P, 9>(p, S, cx, cy, ks, e, lane); break;
    }
}

// One stencil in the working set `base` (layout L): gather, fill, eliminate,
// back-substitute, scatter.
template <typename T, class L, int NRHS, int PB>
__device__ __forceinline__ void assemble_any(const AsmParams& p, int s, int off, int ks, int P,
                                             int Q, char* base, int lane) {
    constexpr int LDS = L::LDS, G = L::G;
    double* cx = reinterpret_cast<double*>(base + L::off_cx);
    double* cy = reinterpret_cast<double*>(base + L::off_cy);
    T* S = reinterpret_cast<T*>(base + L::off_s);
    int* piv = reinterpret_cast<int*>(base + L::off_piv);
    int* act = reinterpret_cast<int*>(base + L::off_act);
    unsigned char* alive = reinterpret_cast<unsigned char*>(base + L::off_alive);
    const int np = npoly(P), n = np + ks;
    const int e = gather_scale<L::KMAX, false>(p, off, ks, p.x[s], p.y[s], cx, cy, lane);
    switch (P) {
        case 1: fill_system_q<T, LDS, NRHS, 1>(p, Q, S, cx, cy, ks, e, lane); break;
        case 2: fill_system_q<T, LDS, NRHS, 2>(p, Q, S, cx, cy, ks, e, lane); break;
        case 3: fill_system_q<T, LDS, NRHS, 3>(p, Q, S, cx, cy, ks, e, lane); break;
        default: fill_system_q<T, LDS, NRHS, 4>(p, Q, S, cx, cy, ks, e, lane); break;
    }
    __syncwarp(group_mask(G));
    T* pinv = reinterpret_cast<T*>(base + L::off_pinv);
    const int info = eliminate_blocked<T, L::R, LDS, NRHS, PB>(S, pinv, piv, act, alive, n, lane);
    T xs[L::R][NRHS];
    back_substitute_blk<T, L::R, LDS, NRHS, G, false>(S, piv, pinv, nullptr, n, lane, xs, NoHook{}, np);
    scatter_regs<T, L::R, NRHS, G>(p, xs, np, ks, off, e, info, s, lane);
}

template <typename T, int NS, int NG, int NRHS, int PB>
struct CsrCfg {
    using SmemL = BlkLayout<T, NS, NRHS, NS, PB, 32, false>;  // shared-memory slot
    using GlobL = BlkLayout<T, NG, NRHS, NG, PB, 32, false>;  // global scratch region
    static constexpr size_t gbytes = (static_cast<size_t>(GlobL::bytes) + 255) & ~size_t(255);
};

template <typename T, int NS, int NG, int NRHS, int BLOCK, int PB, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB)
    blk_csr_kernel(AsmParams p, const int8_t* degree, int P0, int phs, char* gscratch, int* err) {
    using C = CsrCfg<T, NS, NG, NRHS, PB>;
    constexpr int G = 32, GPB = BLOCK / G;
    extern __shared__ __align__(16) char smem_raw[];
    const int gib = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    char* slot = smem_raw + gib * C::SmemL::bytes;
    char* gslot = gscratch + (static_cast<size_t>(blockIdx.x) * GPB + gib) * C::gbytes;
    const int nitems = p.nitems_dev ? *p.nitems_dev : p.nitems;
    const int* list = (p.list && p.list_off_dev) ? p.list + *p.list_off_dev : p.list;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(p.work, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        const int s = list ? list[it] : p.item_base + it;
        const int off = p.ia[s], ks = p.ia[s + 1] - off;
        const int P = degree ? degree[s] : P0;
        const int Q = phs ? phs : 2 * P - 1;
        const int n = ks + npoly(P);
        const bool ok = P >= 1 && P <= 4 && (Q == 3 || Q == 5 || Q == 7 || Q == 9) && ks >= 1 &&
                        n <= NG;
        if (!ok) {
            if (lane == 0) atomicExch(err, 1);
            continue;
        }
        if (n <= NS)
            assemble_any<T, typename C::SmemL, NRHS, PB>(p, s, off, ks, P, Q, slot, lane);
        else
            assemble_any<T, typename C::GlobL, NRHS, PB>(p, s, off, ks, P, Q, gslot, lane);
    }
}

}  // namespace rbfb
