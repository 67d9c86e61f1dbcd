// ref_knn.cpp -- a C entry point over the reference's own stencil searches.
//
// TEST INFRASTRUCTURE. Compiled by oracle/Makefile from the reference
// sources where they lie (nothing of them is copied here) into
// oracle/_ref/libref_knn.so. Only tests/ and the CPU legs of bench.py load
// it: it is the k-NN oracle and the reference's CPU baseline.
//
//   ref_nodeset_stencils  rbf::NodeSet<double,int32_t>::stencils(k), the
//                         nanoflann open-plane search (src/rbf_nodeset.h:162-181)
//   ref_kdtree_stencils   rbf::spatial::KdTree::knn_stencils(k), the ckdtree
//                         search, periodic when both periods are positive
//                         (src/rbf_spatial.h:178-183, src/rbf_spatial.cpp:251-260)
//
// Both reference functions exit the process on bad input, so the checks
// they make are repeated here first and reported as -1 instead.

#include <cstdint>
#include <vector>

#include "rbf_nodeset.h"
#include "rbf_spatial.h"

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

void ref_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int ref_nodeset_stencils(int n, const double* x, const double* y, int k, int* ja) {
    if (n < 1 || k < 1 || k > n) return -1;
    rbf::NodeSet<double, std::int32_t> ns(std::vector<double>(x, x + n),
                                          std::vector<double>(y, y + n), std::vector<int>(n, 0));
    const auto st = ns.stencils(k);
    for (size_t i = 0; i < st.size(); ++i) ja[i] = st[i];
    return 0;
}

int ref_kdtree_stencils(int n, const double* x, const double* y, int k, double Lx, double Ly,
                        int* ja) {
    if (n < 1 || k < 1 || k > n) return -1;
    const bool periodic = Lx > 0 && Ly > 0;
    if ((Lx > 0) != (Ly > 0)) return -1;
    std::vector<double> xv(x, x + n), yv(y, y + n);
    const auto pts = rbf::spatial::interleave(xv, yv);
    std::vector<std::int32_t> st;
    if (periodic) {
        const rbf::spatial::PeriodicBox<double, 2> box{{Lx, Ly}};
        rbf::spatial::KdTree tree(pts, box);
        st = tree.knn_stencils(k);
    } else {
        rbf::spatial::KdTree tree(pts, 2);
        st = tree.knn_stencils(k);
    }
    for (size_t i = 0; i < st.size(); ++i) ja[i] = st[i];
    return 0;
}

}  // extern "C"
