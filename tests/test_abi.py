"""The C ABI boundary, without a GPU: the library loads, exports every entry
point include/rbf_b200.h declares, the Python binding covers all of them,
and argument errors come back as status codes (no kernel is launched)."""
import ctypes as C
import re
import subprocess

import pytest

import rbf_b200
from conftest import ROOT

HEADER = ROOT / "include" / "rbf_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    c_part = text.split("#ifdef __CUDACC__")[0]
    names = re.findall(r"^\s*(?:const\s+)?[a-z_][\w\s\*]*?\b(rbfb_\w+)\s*\(", c_part, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_abi():
    names = declared_functions()
    for must in ("rbfb_create", "rbfb_knn_stencils", "rbfb_assemble", "rbfb_assemble_csr",
                 "rbfb_assemble_host", "rbfb_fill_matrices", "rbfb_store_to_csr",
                 "rbfb_solve_dp", "rbfb_autotune", "rbfb_server_submit"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = rbf_b200.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    # the reference's kernel symbol, same name (src/rbf_operators.cpp:7)
    out = subprocess.run(["nm", "-D", str(rbf_b200.LIB_PATH)], capture_output=True, text=True).stdout
    assert re.search(r"\bT solve_dp\b", out)


def test_binding_covers_the_header():
    assert set(declared_functions()) == set(rbf_b200.exported_symbols())


def test_status_strings():
    assert rbf_b200.status_string(0) == "ok"
    assert "invalid" in rbf_b200.status_string(rbf_b200.EINVAL)
    assert "kernel" in rbf_b200.status_string(rbf_b200.EUNSUPPORTED)


def test_argument_errors_without_a_device():
    L = rbf_b200.lib()
    assert L.rbfb_create(None, 0) == rbf_b200.EINVAL
    assert L.rbfb_destroy(None) == 0
    assert L.rbfb_assemble(None, None, 0, None, None, 1, None, None, None, None, None) == rbf_b200.EINVAL
    assert L.rbfb_knn_stencils(None, 0, None, None, 1, None, None, None) == rbf_b200.EINVAL
    assert L.rbfb_solve_dp(None, None, None, None, None) == rbf_b200.EINVAL
    assert L.rbfb_store_to_csr(-1, None, None, None, None, None) == rbf_b200.EINVAL
    assert L.rbfb_server_submit(None, None, None) == rbf_b200.EINVAL
    assert L.rbfb_server_poll(None, 1, 0, None) == rbf_b200.EINVAL


def test_create_fails_cleanly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert rbf_b200.lib().rbfb_create(C.byref(h), 0) in (rbf_b200.ECUDA, rbf_b200.EINVAL)
    assert not h.value


def test_cpp_mirror_compiles_and_links(tmp_path):
    """A C++ caller of the reference-shaped interface (cpp/rbf_b200.hpp)
    builds against include/rbf_b200.h and links to the library; the program
    is run only to the point of creating a context, which fails cleanly
    without a device."""
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include "rbf_b200.hpp"
#include <cstdio>
using Lap = rbf_b200::laplace_config<21, 2, 3>;
using Interp = rbf_b200::interp_config<35, 4, 3, 5>;
static_assert(Lap::nt == 27 && Interp::nt == 45, "system sizes");
int main() {
    rbfb_ctx* ctx = nullptr;
    int st = rbfb_create(&ctx, 0);
    if (st == RBFB_OK) {
        rbfb_destroy(ctx);
        std::puts("device");
        return 0;
    }
    std::printf("%s\n", rbfb_status_string(st));
    if (false) {   // instantiate the templates
        double* A[4] = {};
        rbf_b200::assemble_laplace_weights<Lap>(0, nullptr, nullptr, nullptr, A, nullptr);
        rbf_b200::assemble_interp_weights<Interp>(0, nullptr, nullptr, nullptr, A, nullptr,
                                                  nullptr, nullptr);
        rbf_b200::NodeSet<> ns({0.0}, {0.0}, {0});
        (void)ns.stencils(1);
        rbf_b200::StencilOperator op;
        op(nullptr, nullptr);
        (void)op.solve(nullptr, nullptr);
    }
    return st == RBFB_ECUDA ? 0 : 1;
}
''')
    exe = tmp_path / "caller"
    libdir = rbf_b200.LIB_PATH.parent
    cmd = ["g++", "-std=c++17", "-O1", str(src), "-o", str(exe),
           f"-I{ROOT / 'include'}", f"-I{ROOT / 'gpu-assembly_b200' / 'cpp'}",
           "-I/usr/local/cuda/include", f"-L{libdir}", "-lrbf_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    import torch
    if torch.cuda.is_available():
        return
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built CUDA library the binding raises: there is no CPU
    path to fall back on."""
    monkeypatch.setattr(rbf_b200, "_lib", None)
    monkeypatch.setattr(rbf_b200, "LIB_PATH", tmp_path / "missing.so")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        rbf_b200.lib()
    with pytest.raises(RuntimeError):
        rbf_b200.Context(0)
