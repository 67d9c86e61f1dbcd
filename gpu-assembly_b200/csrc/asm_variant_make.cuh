// asm_variant_make.cuh -- defines one compiled shape of the assembly kernel
// (RBFB_DEFINE_VARIANT) and the Variant record the runtime launches it by.
#pragma once

#include <cuda_runtime.h>

#include "asm_blocked.cuh"
#include "asm_kernel.cuh"
#include "asm_variants.h"

namespace rbfb {

template <typename T, int GR, int GC, int NTP, int NRHS, int P, int Q, bool MIXED, int BLOCK,
          int MINB, bool SMEM, bool PF>
Variant make_variant(const char* name) {
    using C = AsmCfg<T, GR, GC, NTP, NRHS, P, Q, MIXED, SMEM>;
    Variant v{};
    v.name = name;
    v.kernel =
        reinterpret_cast<const void*>(&asm_kernel<T, GR, GC, NTP, NRHS, P, Q, MIXED, BLOCK, MINB, SMEM, PF>);
    v.launch = [](dim3 grid, int block, size_t smem, cudaStream_t st, const AsmParams& p) {
        asm_kernel<T, GR, GC, NTP, NRHS, P, Q, MIXED, BLOCK, MINB, SMEM, PF><<<grid, block, smem, st>>>(p);
    };
    v.mixed = MIXED;
    v.P = P;
    v.Q = Q;
    v.ntp = NTP;
    v.nrhs = NRHS;
    v.group = C::G;
    v.block = BLOCK;
    v.smem_group = C::bytes;
    v.smem_block = C::bytes * (BLOCK / C::G);
    return v;
}

template <typename T, int NMAX, int NRHS, int P, int Q, bool MIXED, int BLOCK, int MINB, int PB,
          bool PF, int GW = 32>
Variant make_blk_variant(const char* name) {
    using C = BlkCfg<T, NMAX, NRHS, P, Q, MIXED, PB, GW>;
    Variant v{};
    v.name = name;
    v.kernel = reinterpret_cast<const void*>(
        &blk_kernel<T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF, GW>);
    v.launch = [](dim3 grid, int block, size_t smem, cudaStream_t st, const AsmParams& p) {
        blk_kernel<T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF, GW><<<grid, block, smem, st>>>(p);
    };
    v.mixed = MIXED;
    v.P = P;
    v.Q = Q;
    v.ntp = NMAX;
    v.nrhs = NRHS;
    v.group = C::G;
    v.block = BLOCK;
    v.smem_group = C::bytes;
    v.smem_block = C::bytes * (BLOCK / C::G);
    return v;
}

}  // namespace rbfb

#define RBFB_DEFINE_BLK_VARIANT(name, T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF)          \
    namespace rbfb {                                                                           \
    Variant variant_##name() {                                                                 \
        return make_blk_variant<T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF>(#name);       \
    }                                                                                          \
    }

// the same with half-warp groups: two stencils per warp
#define RBFB_DEFINE_BLK16_VARIANT(name, T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF)        \
    namespace rbfb {                                                                           \
    Variant variant_##name() {                                                                 \
        return make_blk_variant<T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF, 16>(#name);   \
    }                                                                                          \
    }

#define RBFB_DEFINE_VARIANT(name, T, GR, GC, NTP, NRHS, P, Q, MIXED, BLOCK, MINB, SMEM, PF)    \
    namespace rbfb {                                                                           \
    Variant variant_##name() {                                                                 \
        return make_variant<T, GR, GC, NTP, NRHS, P, Q, MIXED, BLOCK, MINB, SMEM, PF>(#name);  \
    }                                                                                          \
    }
