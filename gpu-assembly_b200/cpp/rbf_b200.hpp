// rbf_b200.hpp -- C++ host interface mirroring the reference's operator
// interface for the assembly path, over the C ABI of include/rbf_b200.h.
//
// Names, argument meaning and error behaviour follow the reference:
//
//   rbf_b200::NodeSet<T, I>::stencils(k)       rbf::NodeSet::stencils (src/rbf_nodeset.h:155-181):
//                                              ja(k, n) in Fortran order, self first, sorted by
//                                              distance; k < 1 or k > n prints an error and exits
//   rbf_b200::spatial::knn_stencils(...)       rbf::spatial::KdTree::knn_stencils in a periodic
//                                              box (src/rbf_spatial.h:178-183)
//   rbf_b200::interp_config<N,NRHS,P,Q,ARCH,T> rbf_operators::interp_config (src/rbf_operators.h:
//                                              187-290): N, NRHS, P, Q as there; ARCH is accepted
//                                              and ignored (one target, sm_100a)
//   rbf_b200::assemble_interp_weights<Config>  the kernel of src/rbf_operators.h:320-376, as a host
//                                              call with the same arguments, all device pointers:
//                                              A is the device-resident table of NRHS device
//                                              pointers the reference kernel dereferences
//   rbf_b200::laplace_config / assemble_laplace_weights
//                                              the Laplacian assembly src/main.cpp:15-16,44-45
//                                              sketches (never implemented there)
//   rbf_b200::StencilOperator                  mv_op of src/main.cpp:57-66 (A.spmv, then the
//                                              boundary fix) and, as solve(), the solve that
//                                              src/main.cpp:68 leaves empty (BiCGSTAB)
//
// T = double assembles in FP64; rbf_b200::Precision lets a caller ask for
// the FP32-factorisation + FP64-refinement form instead (weights are FP64
// either way).
#ifndef RBF_B200_HPP
#define RBF_B200_HPP

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "rbf_b200.h"

namespace rbf_b200 {

enum class Precision { fp64 = RBFB_FP64, fp32_refined = RBFB_FP32_IR };

// The library context of the calling thread (created on first use).
inline rbfb_ctx* context(int device = 0) {
    thread_local rbfb_ctx* ctx = nullptr;
    thread_local struct Guard {
        rbfb_ctx** p;
        ~Guard() {
            if (*p) rbfb_destroy(*p);
        }
    } guard{&ctx};
    if (!ctx && rbfb_create(&ctx, device) != RBFB_OK)
        throw std::runtime_error("rbf_b200: cannot create a context on device " +
                                 std::to_string(device));
    return ctx;
}

inline void check(int status, const char* what) {
    if (status < 0) {
        throw std::runtime_error(std::string("rbf_b200: ") + what + ": " +
                                 rbfb_status_string(status) + " (" +
                                 rbfb_last_error(context()) + ")");
    }
}

// Device buffer with RAII, for the staging inside the host conveniences.
template <typename V>
struct DeviceArray {
    V* p = nullptr;
    explicit DeviceArray(size_t n) {
        if (n && cudaMalloc(&p, n * sizeof(V)) != cudaSuccess)
            throw std::runtime_error("rbf_b200: cudaMalloc failed");
    }
    ~DeviceArray() { cudaFree(p); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
};

// Node set with the reference's stencils(k): x, y on the host (as there).
template <typename T = double, typename I = int32_t>
class NodeSet {
    static_assert(std::is_same_v<T, double>, "the B200 search works on double coordinates");
    static_assert(std::is_same_v<I, int32_t>, "stencil indices are int32");

public:
    std::vector<T> x, y;
    std::vector<int> flag;

    NodeSet(std::vector<T> x_, std::vector<T> y_, std::vector<int> flag_)
        : x(std::move(x_)), y(std::move(y_)), flag(std::move(flag_)) {}

    size_t num_points() const { return x.size(); }

    // ja(k, n), Fortran order: the k nearest neighbours of node s at ja[s*k],
    // sorted by distance, ja[s*k] == s (src/rbf_nodeset.h:155-181).
    std::vector<I> stencils(int k) const {
        const auto n = static_cast<I>(x.size());
        if (k < 1 || static_cast<size_t>(k) > x.size()) {
            std::cerr << "error: NodeSet::stencils: k=" << k << " with " << n << " nodes\n";
            std::exit(1);
        }
        DeviceArray<double> xd(x.size()), yd(y.size());
        DeviceArray<int> ja(x.size() * k);
        cudaMemcpy(xd.p, x.data(), x.size() * sizeof(double), cudaMemcpyHostToDevice);
        cudaMemcpy(yd.p, y.data(), y.size() * sizeof(double), cudaMemcpyHostToDevice);
        check(rbfb_knn_stencils(context(), static_cast<int>(n), xd.p, yd.p, k, nullptr, ja.p,
                                nullptr),
              "NodeSet::stencils");
        std::vector<I> out(x.size() * k);
        cudaMemcpy(out.data(), ja.p, out.size() * sizeof(int), cudaMemcpyDeviceToHost);
        return out;
    }
};

namespace spatial {
// KdTree(points, PeriodicBox{{Lx, Ly}}).knn_stencils(k) of the reference:
// periodic minimum-image k-NN of the cloud's own points, ja(k, n) int32.
inline std::vector<int32_t> knn_stencils(const std::vector<double>& x,
                                         const std::vector<double>& y, double Lx, double Ly,
                                         int k) {
    const int n = static_cast<int>(x.size());
    if (k < 1 || k > n) {
        std::fprintf(stderr, "rbf::spatial: KdTree::query: k outside [1, number of points]\n");
        std::exit(1);
    }
    DeviceArray<double> xd(n), yd(n);
    DeviceArray<int> ja(static_cast<size_t>(n) * k);
    cudaMemcpy(xd.p, x.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(yd.p, y.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    const double period[2] = {Lx, Ly};
    check(rbfb_knn_stencils(context(), n, xd.p, yd.p, k, period, ja.p, nullptr), "knn_stencils");
    std::vector<int32_t> out(static_cast<size_t>(n) * k);
    cudaMemcpy(out.data(), ja.p, out.size() * sizeof(int), cudaMemcpyDeviceToHost);
    return out;
}
}  // namespace spatial

constexpr int npoly(int P) { return (P + 1) * (P + 2) / 2; }

// The reference's interp_config<N, NRHS, P, Q, ARCH, T>: stencil size N,
// NRHS interpolation points, degree P, PHS exponent Q.
template <int N_, int NRHS_, int P_, int Q_ = 3, unsigned ARCH_ = 1000, typename T_ = double,
          Precision PREC_ = Precision::fp64>
struct interp_config {
    using value_type = T_;
    static constexpr int N = N_, NRHS = NRHS_, P = P_, Q = Q_;
    static constexpr unsigned ARCH = ARCH_;
    static constexpr int npoly = rbf_b200::npoly(P);
    static constexpr int nt = N + npoly;
    static constexpr Precision precision = PREC_;
    static_assert(std::is_same_v<T_, double>, "weights are assembled and returned in FP64");
    static_assert(NRHS >= 1 && NRHS <= RBFB_MAX_RHS, "1..RBFB_MAX_RHS right-hand sides");
};

// The reference's kernel assemble_interp_weights<Config> as a host call:
// nstencils stencils of N neighbours (ja: device, row s at ja[s*N]), weights
// of interpolation point j (xc[j], yc[j], stencil-local frame, device arrays)
// into A[j][s*N + k], per-stencil status into info (device, 0 = ok). A is,
// as in the reference (src/rbf_operators.h:324,370-375), a DEVICE array of
// NRHS device pointers, read by the kernel. Asynchronous on `stream`.
template <class Config>
void assemble_interp_weights(int nstencils, const typename Config::value_type* x,
                             const typename Config::value_type* y, const int* ja,
                             typename Config::value_type* const* A,
                             const typename Config::value_type* xc,
                             const typename Config::value_type* yc, int* info,
                             cudaStream_t stream = nullptr) {
    rbfb_desc d{};
    d.degree = Config::P;
    d.phs = Config::Q;
    d.ops = RBFB_OP_INTERP;
    d.precision = static_cast<int>(Config::precision);
    d.scale = 1;
    d.nc = Config::NRHS;
    d.xc = xc;
    d.yc = yc;
    check(rbfb_assemble_dtab(context(), &d, nstencils, x, y, Config::N, ja, A, info, nullptr,
                             stream),
          "assemble_interp_weights");
}

// The Laplacian assembly src/main.cpp:15-16 names: laplace_config<N, P, Q,
// ARCH, T> and assemble_laplace_weights<Config>(npoints, x, y, ja, A_tab,
// info), one right-hand side (the Laplacian at the stencil centre); A_tab is
// a device table of one device pointer, passed as ptr(A_tab) there
// (src/main.cpp:44-45).
template <int N_, int P_, int Q_ = 3, unsigned ARCH_ = 1000, typename T_ = double,
          Precision PREC_ = Precision::fp64>
struct laplace_config : interp_config<N_, 1, P_, Q_, ARCH_, T_, PREC_> {};

template <class Config>
void assemble_laplace_weights(int npoints, const typename Config::value_type* x,
                              const typename Config::value_type* y, const int* ja,
                              typename Config::value_type* const* A_tab, int* info,
                              cudaStream_t stream = nullptr) {
    rbfb_desc d{};
    d.degree = Config::P;
    d.phs = Config::Q;
    d.ops = RBFB_OP_LAPLACE;
    d.precision = static_cast<int>(Config::precision);
    d.scale = 1;
    check(rbfb_assemble_dtab(context(), &d, npoints, x, y, Config::N, ja, A_tab, info, nullptr,
                             stream),
          "assemble_laplace_weights");
}

// The assembled operator with identity rows at the boundary nodes, on device
// arrays: operator() is mv_op (y = A x, then y[bnd] = x[bnd]); solve() runs
// BiCGSTAB for A u = f from the guess in u to ||f - A u|| <= tol ||f|| and
// returns the iterations taken, throwing on argument or CUDA errors and,
// unless allow_unconverged, when maxit runs out or the method breaks down.
// ia == nullptr selects fixed-width rows of k (the reference's layout,
// src/rbf_operators.h:307-313); operator() needs that layout.
struct StencilOperator {
    int n = 0;
    int k = 0;
    const int* ja = nullptr;
    const double* values = nullptr;
    const int* bnd = nullptr;
    int nbnd = 0;
    const int* ia = nullptr;

    void operator()(const double* x, double* y, cudaStream_t stream = nullptr) const {
        if (ia) throw std::runtime_error("rbf_b200: mv_op needs fixed-width rows");
        check(rbfb_spmv(n, k, ja, values, x, y, bnd, nbnd, stream), "mv_op");
    }

    int solve(const double* f, double* u, double tol = 1e-10, int maxit = 10000,
              double* relres = nullptr, bool allow_unconverged = false,
              cudaStream_t stream = nullptr) const {
        int iters = 0;
        double rel = 0.0;
        const int st = rbfb_solve_bicgstab(context(), n, k, ia, ja, values, bnd, nbnd, f, u, tol,
                                           maxit, &iters, &rel, stream);
        if (relres) *relres = rel;
        if (st == RBFB_ENOCONV || st == RBFB_EBREAKDOWN) {
            if (!allow_unconverged) check(st, "solve");
        } else {
            check(st, "solve");
        }
        return iters;
    }
};

}  // namespace rbf_b200

#endif  // RBF_B200_HPP
