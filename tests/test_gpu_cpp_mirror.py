"""The C++ host interface (cpp/rbf_b200.hpp) run on the GPU, as a reference
caller would use it: NodeSet::stencils(k), then assemble_laplace_weights and
assemble_interp_weights with the operator table A in DEVICE memory
(src/rbf_operators.h:324,370-375; src/main.cpp:44-45), then the mv_op of
src/main.cpp:57-66. A small C++ program is compiled against the header and
the library, run, and its outputs are checked against the oracle: stencils
index for index, FP64 weights bit for bit, the operator application to the
oracle's row sums.
"""
import subprocess

import numpy as np
import pytest

import oracle as O
import rbf_b200
from conftest import ROOT
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu

CALLER = r'''
#include "rbf_b200.hpp"
#include <cstdio>
#include <vector>

using Lap = rbf_b200::laplace_config<21, 2, 3>;
using Interp = rbf_b200::interp_config<21, 2, 2, 3>;

template <typename V>
static std::vector<V> slurp(const char* path, size_t n) {
    std::vector<V> v(n);
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fread(v.data(), sizeof(V), n, f) != n) std::exit(3);
    std::fclose(f);
    return v;
}
template <typename V>
static void dump(const char* path, const V* p, size_t n) {
    FILE* f = std::fopen(path, "wb");
    if (!f || std::fwrite(p, sizeof(V), n, f) != n) std::exit(4);
    std::fclose(f);
}
template <typename V>
static V* dev(const V* h, size_t n) {
    V* d = nullptr;
    if (cudaMalloc(&d, n * sizeof(V)) != cudaSuccess) std::exit(5);
    if (h) cudaMemcpy(d, h, n * sizeof(V), cudaMemcpyHostToDevice);
    return d;
}

int main(int argc, char** argv) {
    const int n = std::atoi(argv[1]);
    const std::string dir = argv[2];
    auto x = slurp<double>((dir + "/x.bin").c_str(), n);
    auto y = slurp<double>((dir + "/y.bin").c_str(), n);
    rbf_b200::NodeSet<> ns(x, y, std::vector<int>(n, 0));
    const std::vector<int> ja = ns.stencils(Lap::N);
    const size_t nnz = static_cast<size_t>(n) * Lap::N;
    double* xd = dev(x.data(), n);
    double* yd = dev(y.data(), n);
    int* jad = dev(ja.data(), nnz);
    int* info = dev<int>(nullptr, n);
    // the operator tables live in device memory, as the reference's A
    double* lap = dev<double>(nullptr, nnz);
    double** lap_tab = dev(&lap, 1);
    rbf_b200::assemble_laplace_weights<Lap>(n, xd, yd, jad, lap_tab, info);
    double* w[2] = {dev<double>(nullptr, nnz), dev<double>(nullptr, nnz)};
    double** w_tab = dev(w, 2);
    const double xc_h[2] = {0.0, 0.25e-2}, yc_h[2] = {0.0, -0.5e-2};
    double* xc = dev(xc_h, 2);
    double* yc = dev(yc_h, 2);
    rbf_b200::assemble_interp_weights<Interp>(n, xd, yd, jad, w_tab, xc, yc, info);
    // mv_op of the Laplacian, boundary rows 0 and 1 fixed to the input
    std::vector<double> u(n);
    for (int i = 0; i < n; ++i) u[i] = x[i] * x[i] + 3.0 * y[i];
    double* ud = dev(u.data(), n);
    double* vd = dev<double>(nullptr, n);
    const int bnd_h[2] = {0, 1};
    int* bnd = dev(bnd_h, 2);
    rbf_b200::StencilOperator op;
    op.n = n;
    op.k = Lap::N;
    op.ja = jad;
    op.values = lap;
    op.bnd = bnd;
    op.nbnd = 2;
    op(ud, vd);
    if (cudaDeviceSynchronize() != cudaSuccess) return 6;
    std::vector<double> hv(nnz);
    std::vector<int> hi(n);
    dump((dir + "/ja.bin").c_str(), ja.data(), nnz);
    cudaMemcpy(hv.data(), lap, nnz * sizeof(double), cudaMemcpyDeviceToHost);
    dump((dir + "/lap.bin").c_str(), hv.data(), nnz);
    for (int j = 0; j < 2; ++j) {
        cudaMemcpy(hv.data(), w[j], nnz * sizeof(double), cudaMemcpyDeviceToHost);
        dump((dir + "/w" + std::to_string(j) + ".bin").c_str(), hv.data(), nnz);
    }
    cudaMemcpy(hi.data(), info, n * sizeof(int), cudaMemcpyDeviceToHost);
    dump((dir + "/info.bin").c_str(), hi.data(), n);
    cudaMemcpy(u.data(), vd, n * sizeof(double), cudaMemcpyDeviceToHost);
    dump((dir + "/mv.bin").c_str(), u.data(), n);
    std::puts("ok");
    return 0;
}
'''


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    d = tmp_path_factory.mktemp("cpp_mirror")
    src = d / "caller.cpp"
    src.write_text(CALLER)
    exe = d / "caller"
    libdir = rbf_b200.LIB_PATH.parent
    cmd = ["g++", "-std=c++17", "-O1", str(src), "-o", str(exe),
           f"-I{ROOT / 'include'}", f"-I{ROOT / 'gpu-assembly_b200' / 'cpp'}",
           "-I/usr/local/cuda/include", f"-L{libdir}", "-lrbf_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_mirror_runs_and_matches_the_oracle(torch_cuda, caller, tmp_path):
    c = NS.config_small()
    x, y = c["x"], c["y"]
    n, k = x.size, 21
    x.astype(np.float64).tofile(tmp_path / "x.bin")
    y.astype(np.float64).tofile(tmp_path / "y.bin")
    r = subprocess.run([str(caller), str(n), str(tmp_path)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
    ja = np.fromfile(tmp_path / "ja.bin", np.int32)
    np.testing.assert_array_equal(ja, O.knn_brute(x, y, k))
    np.testing.assert_array_equal(np.fromfile(tmp_path / "info.bin", np.int32), 0)
    lap = np.fromfile(tmp_path / "lap.bin")
    Wl, _ = O.assemble(x, y, ja, k, 2, 3, ops=O.OP_LAPLACE)
    np.testing.assert_array_equal(lap, Wl[0])
    xc, yc = np.array([0.0, 0.25e-2]), np.array([0.0, -0.5e-2])
    Wi, _ = O.assemble(x, y, ja, k, 2, 3, ops=O.OP_INTERP, xc=xc, yc=yc)
    for j in range(2):
        np.testing.assert_array_equal(np.fromfile(tmp_path / f"w{j}.bin"), Wi[j])
    # interpolation at the centre reproduces the node value: weight 1 on self
    np.testing.assert_allclose(Wi[0].reshape(n, k)[:, 0], 1.0, atol=1e-10)
    mv = np.fromfile(tmp_path / "mv.bin")
    u = x * x + 3.0 * y
    want = O.spmv(ja, lap, u, k, bnd=np.array([0, 1], np.int32))
    np.testing.assert_array_equal(mv, want)
