// asm_variants.h -- launch metadata of the compiled assembly kernel shapes.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace rbfb {

struct AsmParams;

struct Variant {
    const char* name;
    const void* kernel;  // for occupancy queries and attributes
    void (*launch)(dim3 grid, int block, size_t smem, cudaStream_t st, const AsmParams& p);
    bool mixed;
    int P, Q;
    int ntp;         // padded system size (stencil size + polynomial terms <= ntp)
    int nrhs;        // right-hand-side columns compiled in
    int group;       // lanes per stencil
    int block;       // threads per CTA
    int smem_group;  // shared memory per stencil in flight, bytes
    int smem_block;  // dynamic shared memory per CTA, bytes
};

const std::vector<Variant>& variants();

}  // namespace rbfb
