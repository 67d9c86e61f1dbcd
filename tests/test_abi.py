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
