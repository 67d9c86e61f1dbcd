// ref_lbm.cu -- host launchers for the reference's own D2Q9 kernels
// (feq_kernel, macros_kernel, bgk_kernel_split: src/lbm/d2q9_kernels.cu and
// its header), for both instantiations.
//
// TEST INFRASTRUCTURE. ref_lbm_run.cu includes this file, which includes the
// reference's d2q9_kernels.cu where it lies (nothing of it is copied here;
// one translation unit, so the kernel templates and their launches meet);
// oracle/Makefile compiles that into oracle/_ref/ref_lbm_run with
// --fmad=false, so that every product and sum is rounded as the source
// writes it. It pins the library's LBM kernels to the reference's own, bit
// for bit. The launchers take device pointers, launch through
// cudaLaunchKernel, check the launch and synchronise; they allocate nothing.
// They return 0, or -1 (launch error) / -2 (run error), and ref_lbm_error()
// names the CUDA error of the last failure.
#include <cuda_runtime.h>

#include "d2q9_kernels.cu"

namespace {
cudaError_t last_err = cudaSuccess;
inline int grid(int n) { return (n + 255) / 256; }

// One launch of kernel `k` over n nodes (256 threads a block) with the given
// arguments, by address: the <<< >>> form of these explicitly instantiated
// kernel templates failed here at launch with "invalid device function",
// while a launch through cudaLaunchKernel with the same address runs.
template <typename... A>
int launch(const void* k, int n, A... a) {
    void* args[] = {static_cast<void*>(&a)...};
    last_err = cudaLaunchKernel(k, dim3(grid(n)), dim3(256), args, 0, nullptr);
    if (last_err != cudaSuccess) return -1;
    last_err = cudaDeviceSynchronize();
    return last_err == cudaSuccess ? 0 : -2;
}
}  // namespace

extern "C" {

const char* ref_lbm_error() { return cudaGetErrorString(last_err); }

// precision 0: double arrays, 1: float arrays
int ref_lbm_feq(int n, int precision, const void* rho, const void* ux, const void* uy, void* pdf) {
    if (n <= 0) return 0;
    if (precision == 0)
        return launch(reinterpret_cast<const void*>(&feq_kernel<double>), n, n,
                      static_cast<const double*>(rho), static_cast<const double*>(ux),
                      static_cast<const double*>(uy), static_cast<double*>(pdf));
    return launch(reinterpret_cast<const void*>(&feq_kernel<float>), n, n,
                  static_cast<const float*>(rho), static_cast<const float*>(ux),
                  static_cast<const float*>(uy), static_cast<float*>(pdf));
}

int ref_lbm_macros(int n, int precision, const void* pdf, void* rho, void* ux, void* uy) {
    if (n <= 0) return 0;
    if (precision == 0)
        return launch(reinterpret_cast<const void*>(&macros_kernel<double>), n, n,
                      static_cast<const double*>(pdf), static_cast<double*>(rho),
                      static_cast<double*>(ux), static_cast<double*>(uy));
    return launch(reinterpret_cast<const void*>(&macros_kernel<float>), n, n,
                  static_cast<const float*>(pdf), static_cast<float*>(rho),
                  static_cast<float*>(ux), static_cast<float*>(uy));
}

int ref_lbm_bgk_split(int n, int precision, double omega, void* pdf, void* rho, void* ux, void* uy,
                      void* indp) {
    if (n <= 0) return 0;
    if (precision == 0)
        return launch(reinterpret_cast<const void*>(&bgk_kernel_split<double>), n, n, omega,
                      static_cast<double*>(pdf), static_cast<double*>(rho),
                      static_cast<double*>(ux), static_cast<double*>(uy),
                      static_cast<double*>(indp));
    return launch(reinterpret_cast<const void*>(&bgk_kernel_split<float>), n, n,
                  static_cast<float>(omega), static_cast<float*>(pdf), static_cast<float*>(rho),
                  static_cast<float*>(ux), static_cast<float*>(uy), static_cast<float*>(indp));
}

}  // extern "C"
