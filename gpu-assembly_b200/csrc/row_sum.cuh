// row_sum.cuh -- one operator row applied to a vector: the sum over the
// row's stored entries q in [q, e) of values[q] * x(ja[q]), in row order, by
// fused multiply-adds from zero (the order the CPU oracle restates).
//
// Each thread walks its own row, so the loads of consecutive lanes fall in
// different rows: the walk takes eight entries at a time, loading the
// eight weights and columns before the eight gathers and the eight gathers
// before the eight fused multiply-adds (eight gathers in flight instead of
// one). With 16-byte aligned arrays (vec) the row is first walked entry by
// entry up to a multiple of 4 entries, and each group of eight then loads
// its columns as two 16-byte vectors and its weights as four: six load
// instructions instead of sixteen. The sums are the same either way.
#pragma once

#include <cstdint>

namespace rbfb {

inline bool rows_vectorizable(const void* ja, const void* values) {
    return ((reinterpret_cast<uintptr_t>(ja) | reinterpret_cast<uintptr_t>(values)) & 15) == 0;
}

template <class X>
__device__ __forceinline__ double row_sum(const int* __restrict__ ja,
                                          const double* __restrict__ values, long long q,
                                          long long e, bool vec, X x) {
    double acc = 0.0;
    if (vec) {
        for (; q < e && (q & 3); ++q) acc = fma(__ldg(values + q), x(__ldg(ja + q)), acc);
        for (; q + 8 <= e; q += 8) {
            const int4 j0 = __ldg(reinterpret_cast<const int4*>(ja + q));
            const int4 j1 = __ldg(reinterpret_cast<const int4*>(ja + q + 4));
            double2 v[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) v[i] = __ldg(reinterpret_cast<const double2*>(values + q) + i);
            const int j[8] = {j0.x, j0.y, j0.z, j0.w, j1.x, j1.y, j1.z, j1.w};
            double w[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) w[i] = x(j[i]);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                acc = fma(v[i].x, w[2 * i], acc);
                acc = fma(v[i].y, w[2 * i + 1], acc);
            }
        }
    } else {
        for (; q + 8 <= e; q += 8) {
            int j[8];
            double v[8], w[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) j[i] = __ldg(ja + q + i);
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = __ldg(values + q + i);
#pragma unroll
            for (int i = 0; i < 8; ++i) w[i] = x(j[i]);
#pragma unroll
            for (int i = 0; i < 8; ++i) acc = fma(v[i], w[i], acc);
        }
    }
    for (; q < e; ++q) acc = fma(__ldg(values + q), x(__ldg(ja + q)), acc);
    return acc;
}

}  // namespace rbfb
