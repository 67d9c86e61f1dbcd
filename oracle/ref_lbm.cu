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
// for bit. The launchers take device pointers, check the launch and
// synchronise; they allocate nothing. They return 0, or -1 (launch error) /
// -2 (run error), and ref_lbm_error() names the CUDA error of the last failure.
#include <cuda_runtime.h>

#include "d2q9_kernels.cu"

namespace {
cudaError_t last_err = cudaSuccess;
inline int grid(int n) { return (n + 255) / 256; }
inline int done() {
    last_err = cudaGetLastError();
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
        feq_kernel<double><<<grid(n), 256>>>(n, static_cast<const double*>(rho),
                                             static_cast<const double*>(ux),
                                             static_cast<const double*>(uy),
                                             static_cast<double*>(pdf));
    else
        feq_kernel<float><<<grid(n), 256>>>(n, static_cast<const float*>(rho),
                                            static_cast<const float*>(ux),
                                            static_cast<const float*>(uy), static_cast<float*>(pdf));
    return done();
}

int ref_lbm_macros(int n, int precision, const void* pdf, void* rho, void* ux, void* uy) {
    if (n <= 0) return 0;
    if (precision == 0)
        macros_kernel<double><<<grid(n), 256>>>(n, static_cast<const double*>(pdf),
                                                static_cast<double*>(rho),
                                                static_cast<double*>(ux),
                                                static_cast<double*>(uy));
    else
        macros_kernel<float><<<grid(n), 256>>>(n, static_cast<const float*>(pdf),
                                               static_cast<float*>(rho), static_cast<float*>(ux),
                                               static_cast<float*>(uy));
    return done();
}

int ref_lbm_bgk_split(int n, int precision, double omega, void* pdf, void* rho, void* ux, void* uy,
                      void* indp) {
    if (n <= 0) return 0;
    if (precision == 0)
        bgk_kernel_split<double><<<grid(n), 256>>>(n, omega, static_cast<double*>(pdf),
                                                   static_cast<double*>(rho),
                                                   static_cast<double*>(ux),
                                                   static_cast<double*>(uy),
                                                   static_cast<double*>(indp));
    else
        bgk_kernel_split<float><<<grid(n), 256>>>(n, static_cast<float>(omega),
                                                  static_cast<float*>(pdf),
                                                  static_cast<float*>(rho),
                                                  static_cast<float*>(ux), static_cast<float*>(uy),
                                                  static_cast<float*>(indp));
    return done();
}

}  // extern "C"
