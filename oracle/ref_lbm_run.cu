// ref_lbm_run.cu -- command-line runner of the reference's own D2Q9 kernels
// through the launchers of ref_lbm.cu, for the GPU tests: a process of its
// own, so the reference's kernels and CUDA runtime share nothing with the
// process that checks them.
//
// TEST INFRASTRUCTURE, built by oracle/Makefile into oracle/_ref/ref_lbm_run.
//
//   ref_lbm_run DIR N PREC OMEGA
//
// reads DIR/{rho,ux,uy,pert}.bin (raw, N or 9N values of double when PREC is
// 0, float when 1), runs feq_kernel, then bgk_kernel_split on pert, then
// macros_kernel on the post-collision populations, and writes DIR/{feq,post,
// rho,ux,uy,indp,rho2,ux2,uy2}.bin. Prints "ok", or the failing step and its
// CUDA error and exits 1.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "ref_lbm.cu"

namespace {

std::vector<char> slurp(const std::string& path, size_t bytes) {
    std::vector<char> v(bytes);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), 1, bytes, f) != bytes) {
        std::fprintf(stderr, "cannot read %s\n", path.c_str());
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

void dump(const std::string& path, const void* dev, size_t bytes) {
    std::vector<char> h(bytes);
    cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(h.data(), 1, bytes, f) != bytes) std::exit(3);
    std::fclose(f);
}

void* upload(const std::vector<char>& h) {
    void* d = nullptr;
    if (cudaMalloc(&d, h.size()) != cudaSuccess) std::exit(4);
    cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice);
    return d;
}

void check(int rc, const char* what) {
    if (rc != 0) {
        std::printf("%s: %d %s\n", what, rc, ref_lbm_error());
        std::exit(1);
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 5) return 5;
    const std::string dir = argv[1];
    const int n = std::atoi(argv[2]);
    const int prec = std::atoi(argv[3]);
    const double omega = std::atof(argv[4]);
    const size_t es = prec == 0 ? sizeof(double) : sizeof(float);
    const size_t b1 = es * n, b9 = 9 * b1;
    void* rho = upload(slurp(dir + "/rho.bin", b1));
    void* ux = upload(slurp(dir + "/ux.bin", b1));
    void* uy = upload(slurp(dir + "/uy.bin", b1));
    void* pdf = upload(std::vector<char>(b9));
    check(ref_lbm_feq(n, prec, rho, ux, uy, pdf), "feq_kernel");
    dump(dir + "/feq.bin", pdf, b9);
    void* pert = upload(slurp(dir + "/pert.bin", b9));
    void* r = upload(std::vector<char>(b1));
    void* u = upload(std::vector<char>(b1));
    void* v = upload(std::vector<char>(b1));
    void* ip = upload(std::vector<char>(b1));
    check(ref_lbm_bgk_split(n, prec, omega, pert, r, u, v, ip), "bgk_kernel_split");
    dump(dir + "/post.bin", pert, b9);
    dump(dir + "/rho.bin", r, b1);
    dump(dir + "/ux.bin", u, b1);
    dump(dir + "/uy.bin", v, b1);
    dump(dir + "/indp.bin", ip, b1);
    check(ref_lbm_macros(n, prec, pert, r, u, v), "macros_kernel");
    dump(dir + "/rho2.bin", r, b1);
    dump(dir + "/ux2.bin", u, b1);
    dump(dir + "/uy2.bin", v, b1);
    std::puts("ok");
    return 0;
}
