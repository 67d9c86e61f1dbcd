// spmv.cu -- applying an assembled operator: out = A u over the fixed-width
// CSR (ja, values) of the assembly, then the boundary fix out[b] = u[b] for the
// listed boundary rows. The reference sketches exactly this step after its
// assembly (A.spmv(x, y) and the parallel_for over boundary nodes,
// src/main.cpp:57-66), with neither piece implemented.
//
// One thread per row, summing its k products in row order with fused
// multiply-adds from zero: acc = fma(values[s*k+j], u[ja[s*k+j]], acc),
// j = 0..k-1 (row_sum.cuh). The order is pinned so the result is
// reproducible (the CPU oracle does the same).
#include <cuda_runtime.h>

#include <algorithm>

#include "row_sum.cuh"
#include "runtime.h"

namespace rbfb {

__global__ void spmv_fixed_kernel(int n, int k, const int* __restrict__ ja,
                                  const double* __restrict__ values, const double* __restrict__ u,
                                  double* __restrict__ out, bool vec) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const long long q = static_cast<long long>(s) * k;
        out[s] = row_sum(ja, values, q, q + k, vec, [u](int j) { return __ldg(u + j); });
    }
}

__global__ void boundary_fix_kernel(int nb, const int* __restrict__ bnd,
                                    const double* __restrict__ u, double* __restrict__ out) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        out[bnd[b]] = u[bnd[b]];
}

}  // namespace rbfb

extern "C" int rbfb_spmv(int n, int k, const int* ja, const double* values, const double* u,
                         double* out, const int* bnd, int nbnd, void* stream) {
    if (n < 0 || k < 1 || nbnd < 0 || (n > 0 && (!ja || !values || !u || !out)) ||
        (nbnd > 0 && !bnd))
        return RBFB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n > 0) {
        const int blocks = std::min((n + 255) / 256, 148 * 16);
        rbfb::spmv_fixed_kernel<<<blocks, 256, 0, st>>>(n, k, ja, values, u, out,
                                                        rbfb::rows_vectorizable(ja, values));
    }
    if (nbnd > 0) {
        const int blocks = std::min((nbnd + 255) / 256, 148 * 4);
        rbfb::boundary_fix_kernel<<<blocks, 256, 0, st>>>(nbnd, bnd, u, out);
    }
    return cudaGetLastError() == cudaSuccess ? RBFB_OK : RBFB_ECUDA;
}
