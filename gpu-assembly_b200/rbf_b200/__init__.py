"""Python binding of the C ABI in ``include/rbf_b200.h`` (ctypes).

The library is ``gpu-assembly_b200/lib/librbf_b200.so`` (built by
``rbf_b200.build``). There is no CPU fallback: without the library every
entry point raises. Device arrays are passed as torch CUDA tensors (only
their data pointers and the current stream reach the library) or as raw
integer device pointers.

Reference interfaces mirrored here (paths relative to the reference repo):

* ``Context.knn_stencils``  -- ``NodeSet::stencils(k)`` (src/rbf_nodeset.h:162)
  and ``KdTree::knn_stencils(k)`` (src/rbf_spatial.h:178-183)
* ``Context.assemble``      -- ``assemble_interp_weights<Config>``
  (src/rbf_operators.h:320-376) with the run-time descriptor standing in for
  ``interp_config<N, NRHS, P, Q, ARCH, T>`` (:187-290)
* ``Context.fill_matrices`` -- ``fill_matrix`` / Fortran ``fill_kernel``
* ``store_to_csr``          -- Fortran ``store_to_csr`` (src/rbf_cuda.f90:139-157)
* ``solve_dp``              -- the ``solve_dp`` kernel (src/rbf_operators.cpp:7-11)
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = PKG / "lib" / "librbf_b200.so"

OK, EINVAL, ECUDA, ENOMEM, EUNSUPPORTED, ETIMEOUT, EBUDGET, ENOTFOUND, EBUSY, ETOOBIG = (
    0, -1, -2, -3, -4, -5, -6, -7, -8, -9)
ENOCONV, EBREAKDOWN = -10, -11  # outcomes of rbfb_solve_bicgstab
STATIC_MAX_NODES = 65536  # limit of rbfb_knn_stencils_static
MORTON, HILBERT = 0, 1  # curves of rbfb_curve_keys / rbfb_curve_order
OP_INTERP, OP_LAPLACE, OP_DX, OP_DY, OP_DXX, OP_DYY, OP_DXY = 1, 2, 4, 8, 16, 32, 64
FP64, FP32_IR = 0, 1
MAX_RHS = 8
DEFAULT_OPS = OP_LAPLACE | OP_DX | OP_DY


class RbfError(RuntimeError):
    """A nonzero status from the library."""

    def __init__(self, status, msg=""):
        super().__init__(f"rbf_b200 status {status}: {msg}")
        self.status = status


class Desc(C.Structure):
    """``rbfb_desc``: degree, PHS exponent, operators, precision, scaling,
    refinement limits, periods and interpolation points."""
    _fields_ = [("degree", C.c_int), ("phs", C.c_int), ("ops", C.c_int),
                ("precision", C.c_int), ("scale", C.c_int), ("max_sweeps", C.c_int),
                ("ir_tol", C.c_double), ("period", C.c_double * 2), ("nc", C.c_int),
                ("xc", C.c_void_p), ("yc", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("stencils", C.c_longlong), ("singular", C.c_longlong),
                ("fallback", C.c_longlong), ("sweeps", C.c_longlong),
                ("max_sweeps_used", C.c_int), ("buckets", C.c_int), ("ms", C.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Request(C.Structure):
    _fields_ = [("n", C.c_int), ("x_h", C.c_void_p), ("y_h", C.c_void_p), ("k", C.c_int),
                ("desc", Desc)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("n", C.c_int), ("k", C.c_int), ("nrhs", C.c_int),
                ("singular", C.c_longlong), ("fallback", C.c_longlong),
                ("ja", C.c_void_p), ("values", C.c_void_p * MAX_RHS),
                ("submit_ms", C.c_double), ("start_ms", C.c_double), ("end_ms", C.c_double),
                ("dev_start_ms", C.c_double), ("dev_end_ms", C.c_double)]


_lib = None

# name -> (restype, argtypes); the full C ABI of include/rbf_b200.h
_vp, _i, _d, _ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
_PROTOS = {
    "rbfb_create": (_i, [C.POINTER(_vp), _i]),
    "rbfb_destroy": (_i, [_vp]),
    "rbfb_status_string": (C.c_char_p, [_i]),
    "rbfb_last_error": (C.c_char_p, [_vp]),
    "rbfb_kernel_launches": (_ll, [_vp]),
    "rbfb_knn_stencils": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp, _vp]),
    "rbfb_knn_query": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp, _vp]),
    "rbfb_knn_status": (_i, [_vp, _vp]),
    "rbfb_knn_stencils_static": (_i, [_i, _vp, _vp, _i, _vp, _vp, _vp]),
    "rbfb_knn_static_status": (_i, [_vp]),
    "rbfb_assemble": (_i, [_vp, C.POINTER(Desc), _i, _vp, _vp, _i, _vp, _vp, _vp,
                           C.POINTER(Stats), _vp]),
    "rbfb_assemble_dtab": (_i, [_vp, C.POINTER(Desc), _i, _vp, _vp, _i, _vp, _vp, _vp,
                                C.POINTER(Stats), _vp]),
    "rbfb_assemble_range": (_i, [_vp, C.POINTER(Desc), _i, _i, _i, _vp, _vp, _i, _vp, _vp, _vp,
                                 C.POINTER(Stats), _vp]),
    "rbfb_assemble_csr": (_i, [_vp, C.POINTER(Desc), _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               C.POINTER(Stats), _vp]),
    "rbfb_assemble_host": (_i, [_vp, C.POINTER(Desc), _i, _vp, _vp, _i, _vp, _vp, _vp, _vp,
                                C.POINTER(Stats)]),
    "rbfb_fill_matrices": (_i, [_vp, C.POINTER(Desc), _i, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "rbfb_store_to_csr": (_i, [_i, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_fill_kernel": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "rbfb_fill_rhs": (_i, [_i, _vp, _vp, _i, _vp, _vp, _vp, _i, _vp]),
    "rbfb_store_to_csr_stencil": (_i, [_i, _vp, _vp, _vp, _i, _i, _vp]),
    "rbfb_spmv": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "rbfb_solve_bicgstab": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp, _d, _i,
                                 C.POINTER(_i), C.POINTER(_d), _vp]),
    "rbfb_curve_keys": (_i, [_vp, _i, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "rbfb_curve_order": (_i, [_vp, _i, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp]),
    "rbfb_boundary_last": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "rbfb_renumber_stencils": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_renumber_csr": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_permute": (_i, [_i, _vp, _vp, _vp, _i, _vp]),
    "rbfb_solve_dp": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "rbfb_lbm_feq": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_lbm_macros": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_lbm_bgk": (_i, [_i, _i, _d, _vp, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_lbm_stream_collide": (_i, [_i, _i, _i, _vp, _vp, _d, _vp, _vp, _vp, _vp, _vp, _vp]),
    "rbfb_autotune": (_i, [_vp, C.POINTER(Desc), _i, _vp, _vp, _i, _vp, _vp]),
    "rbfb_variant_name": (C.c_char_p, [_i]),
    "rbfb_select_variant": (_i, [_vp, C.POINTER(Desc), _i, _i, _i]),
    "rbfb_server_create": (_i, [C.POINTER(_vp), _i, C.c_size_t, _i]),
    "rbfb_server_submit": (_i, [_vp, C.POINTER(Request), C.POINTER(_ll)]),
    "rbfb_server_poll": (_i, [_vp, _ll, _i, C.POINTER(Result)]),
    "rbfb_server_fetch": (_i, [_vp, _ll, _vp, _vp]),
    "rbfb_server_release": (_i, [_vp, _ll]),
    "rbfb_server_destroy": (_i, [_vp]),
    "rbfb_server_resident_bytes": (C.c_size_t, [_vp]),
}


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"rbf_b200 CUDA library not built: {LIB_PATH} "
                               "(run python -m rbf_b200.build); there is no CPU fallback")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names of the C ABI this binding expects (include/rbf_b200.h)."""
    return sorted(_PROTOS)


def _ptr(a):
    """Device pointer of a torch tensor, an int, or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    return a.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def status_string(status: int) -> str:
    return lib().rbfb_status_string(status).decode()


def make_desc(degree, phs=0, ops=DEFAULT_OPS, precision=FP64, scale=True, max_sweeps=0,
              ir_tol=0.0, period=None, xc=None, yc=None, nc=0) -> Desc:
    d = Desc()
    d.degree = degree
    d.phs = phs
    d.ops = ops
    d.precision = precision
    d.scale = 1 if scale else 0
    d.max_sweeps = max_sweeps
    d.ir_tol = ir_tol
    d.period[0], d.period[1] = (0.0, 0.0) if period is None else (float(period[0]),
                                                                  float(period[1]))
    d.nc = nc
    d.xc = _ptr(xc)
    d.yc = _ptr(yc)
    return d


def num_rhs(ops: int, nc: int = 0) -> int:
    n = nc if ops & OP_INTERP else 0
    b = OP_LAPLACE
    while b <= OP_DXY:
        n += bool(ops & b)
        b <<= 1
    return n


class Context:
    """``rbfb_ctx``: one per host thread. Holds workspace, the launch table
    and counters. Use as a context manager or call close()."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib().rbfb_create(C.byref(h), device)
        if st != OK:
            raise RbfError(st, "rbfb_create failed")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().rbfb_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st < 0:
            raise RbfError(st, f"{what}: {lib().rbfb_last_error(self.h).decode()}")
        return st

    def launches(self) -> int:
        return int(lib().rbfb_kernel_launches(self.h))

    # ---- stencil search
    def knn_stencils(self, x, y, k, ja, period=None, stream=None):
        """ja (int32 device, n*k) <- k nearest neighbours of every node."""
        n = x.numel() if hasattr(x, "numel") else int(len(x))
        per = None if period is None else (C.c_double * 2)(*period)
        st = lib().rbfb_knn_stencils(self.h, n, _ptr(x), _ptr(y), k, per, _ptr(ja),
                                     _stream(stream))
        return self._check(st, "knn_stencils")

    def knn_status(self, stream=None) -> int:
        return self._check(lib().rbfb_knn_status(self.h, _stream(stream)), "knn_status")

    def knn_query(self, x, y, xq, yq, k, ja, period=None, stream=None):
        n = x.numel()
        per = None if period is None else (C.c_double * 2)(*period)
        st = lib().rbfb_knn_query(self.h, n, _ptr(x), _ptr(y), xq.numel(), _ptr(xq), _ptr(yq),
                                  k, per, _ptr(ja), _stream(stream))
        return self._check(st, "knn_query")

    # ---- solving with an assembled operator
    def solve_bicgstab(self, values, ja, f, u, k=None, ia=None, bnd=None, tol=1e-10,
                       maxit=10000, stream=None):
        """BiCGSTAB for A u = f, A = the stencil operator (fixed width k, or
        CSR rows ia) with identity rows at bnd; u (float64 device) holds the
        initial guess and receives the iterate. Returns (status, iters,
        relres) with status OK, ENOCONV or EBREAKDOWN; raises on errors."""
        n = f.numel()
        it, rel = C.c_int(0), C.c_double(0.0)
        nb = 0 if bnd is None else bnd.numel()
        st = lib().rbfb_solve_bicgstab(self.h, n, 0 if k is None else k, _ptr(ia), _ptr(ja),
                                       _ptr(values), _ptr(bnd), nb, _ptr(f), _ptr(u), tol, maxit,
                                       C.byref(it), C.byref(rel), _stream(stream))
        if st not in (OK, ENOCONV, EBREAKDOWN):
            self._check(st, "solve_bicgstab")
        return st, it.value, rel.value

    # ---- assembly
    def assemble(self, desc: Desc, x, y, k, ja, values, info=None, stats=False, stream=None):
        """values: list of float64 device tensors (n*k each), one per
        right-hand side. Returns a Stats dict when stats=True."""
        n = x.numel()
        tab = (C.c_void_p * len(values))(*[_ptr(v) for v in values])
        s = Stats() if stats else None
        st = lib().rbfb_assemble(self.h, C.byref(desc), n, _ptr(x), _ptr(y), k, _ptr(ja), tab,
                                 _ptr(info), C.byref(s) if s is not None else None,
                                 _stream(stream))
        self._check(st, "assemble")
        return s.as_dict() if s is not None else None

    def assemble_dtab(self, desc: Desc, x, y, k, ja, values_tab, info=None, stats=False,
                      stream=None):
        """rbfb_assemble with the output pointer table in device memory
        (values_tab: an int64 device tensor of nrhs device pointers)."""
        n = x.numel()
        s = Stats() if stats else None
        st = lib().rbfb_assemble_dtab(self.h, C.byref(desc), n, _ptr(x), _ptr(y), k, _ptr(ja),
                                      _ptr(values_tab), _ptr(info),
                                      C.byref(s) if s is not None else None, _stream(stream))
        self._check(st, "assemble_dtab")
        return s.as_dict() if s is not None else None

    def assemble_range(self, desc: Desc, first, count, x, y, k, ja_rows, values_rows,
                       info_rows=None, stats=False, stream=None):
        """Stencils first..first+count-1 of the node set (x, y): ja_rows and
        values_rows hold only those rows."""
        tab = (C.c_void_p * len(values_rows))(*[_ptr(v) for v in values_rows])
        s = Stats() if stats else None
        st = lib().rbfb_assemble_range(self.h, C.byref(desc), first, count, x.numel(), _ptr(x),
                                       _ptr(y), k, _ptr(ja_rows), tab, _ptr(info_rows),
                                       C.byref(s) if s is not None else None, _stream(stream))
        self._check(st, "assemble_range")
        return s.as_dict() if s is not None else None

    def assemble_csr(self, desc: Desc, x, y, ia, ja, values, degree=None, info=None,
                     stats=False, stream=None):
        n = x.numel()
        tab = (C.c_void_p * len(values))(*[_ptr(v) for v in values])
        s = Stats() if stats else None
        st = lib().rbfb_assemble_csr(self.h, C.byref(desc), n, _ptr(x), _ptr(y), _ptr(ia),
                                     _ptr(ja), _ptr(degree), tab, _ptr(info),
                                     C.byref(s) if s is not None else None, _stream(stream))
        self._check(st, "assemble_csr")
        return s.as_dict() if s is not None else None

    def assemble_host(self, desc: Desc, x_h, y_h, k, values_h, ja_h=None, ja_out_h=None,
                      info_h=None, stats=True):
        """End to end from host numpy (or pinned torch CPU) arrays."""
        def hp(a):
            if a is None:
                return None
            if hasattr(a, "data_ptr"):
                return a.data_ptr()
            return a.ctypes.data
        n = len(x_h)
        tab = (C.c_void_p * len(values_h))(*[hp(v) for v in values_h])
        s = Stats()
        st = lib().rbfb_assemble_host(self.h, C.byref(desc), n, hp(x_h), hp(y_h), k, hp(ja_h),
                                      hp(ja_out_h), tab, hp(info_h),
                                      C.byref(s) if stats else None)
        self._check(st, "assemble_host")
        return s.as_dict()

    def fill_matrices(self, desc: Desc, x, y, ia, ja, M, ldm, stream=None):
        st = lib().rbfb_fill_matrices(self.h, C.byref(desc), x.numel(), _ptr(x), _ptr(y),
                                      _ptr(ia), _ptr(ja), _ptr(M), ldm, _stream(stream))
        return self._check(st, "fill_matrices")

    def autotune(self, desc: Desc, x, y, k, ja, values):
        tab = (C.c_void_p * len(values))(*[_ptr(v) for v in values])
        st = lib().rbfb_autotune(self.h, C.byref(desc), x.numel(), _ptr(x), _ptr(y), k,
                                 _ptr(ja), tab)
        return self._check(st, "autotune")

    def select_variant(self, desc: Desc, k, index, blocks_per_sm=0):
        """Pin compiled shape `index` for desc's class of k-node stencils."""
        st = lib().rbfb_select_variant(self.h, C.byref(desc), k, index, blocks_per_sm)
        return self._check(st, "select_variant")

    # ---- node renumbering (permutations in gather form: perm[new] = old)
    def curve_keys(self, x, y, keys, ndiv=16, curve=MORTON, bbox=None, stream=None):
        """int64 device keys <- Morton (curve=MORTON) or Hilbert curve keys."""
        bb = None if bbox is None else (C.c_double * 4)(*bbox)
        st = lib().rbfb_curve_keys(self.h, x.numel(), _ptr(x), _ptr(y), bb, ndiv, curve,
                                   _ptr(keys), _stream(stream))
        return self._check(st, "curve_keys")

    def curve_order(self, x, y, perm, inv=None, keys=None, ndiv=16, curve=MORTON, bbox=None,
                    stream=None):
        """perm (int32 device) <- the nodes in stable curve order."""
        bb = None if bbox is None else (C.c_double * 4)(*bbox)
        st = lib().rbfb_curve_order(self.h, x.numel(), _ptr(x), _ptr(y), bb, ndiv, curve,
                                    _ptr(keys), _ptr(perm), _ptr(inv), _stream(stream))
        return self._check(st, "curve_order")

    def boundary_last(self, flag, perm, inv=None, stream=None):
        st = lib().rbfb_boundary_last(self.h, flag.numel(), _ptr(flag), _ptr(perm), _ptr(inv),
                                      _stream(stream))
        return self._check(st, "boundary_last")

    def renumber_csr(self, ia, ja, perm, inv, ia_out, ja_out, stream=None):
        st = lib().rbfb_renumber_csr(self.h, perm.numel(), _ptr(ia), _ptr(ja), _ptr(perm),
                                     _ptr(inv), _ptr(ia_out), _ptr(ja_out), _stream(stream))
        return self._check(st, "renumber_csr")


def knn_stencils_static(x, y, k, ja, period=None, stream=None):
    """rbfb_knn_stencils_static: the k-NN search without any allocation
    (fixed device scratch, n <= STATIC_MAX_NODES). Raises RbfError."""
    n = x.numel()
    per = None if period is None else (C.c_double * 2)(*period)
    st = lib().rbfb_knn_stencils_static(n, _ptr(x), _ptr(y), k, per, _ptr(ja), _stream(stream))
    if st != OK:
        raise RbfError(st, status_string(st))


def knn_static_status(stream=None) -> int:
    """rbfb_knn_static_status: 0 when the last no-allocation search on the
    current device finished every query, 1 when one gave up. Synchronises."""
    st = lib().rbfb_knn_static_status(_stream(stream))
    if st < 0:
        raise RbfError(st, status_string(st))
    return st


def variant_name(index: int):
    v = lib().rbfb_variant_name(index)
    return None if v is None else v.decode()


def variant_names():
    """Names of every compiled kernel shape, by index."""
    out = []
    while (v := variant_name(len(out))) is not None:
        out.append(v)
    return out


def renumber_stencils(n, k, ja, perm, inv, ja_out, stream=None):
    """ja_out[s*k+j] = inv[ja[perm[s]*k+j]] (out of place)."""
    st = lib().rbfb_renumber_stencils(n, k, _ptr(ja), _ptr(perm), _ptr(inv), _ptr(ja_out),
                                      _stream(stream))
    if st != OK:
        raise RbfError(st, "renumber_stencils")


def permute(perm, src, out, stream=None):
    """out[i] = src[perm[i]] for 4- or 8-byte elements (out of place)."""
    st = lib().rbfb_permute(perm.numel(), _ptr(perm), _ptr(src), _ptr(out), src.element_size(),
                            _stream(stream))
    if st != OK:
        raise RbfError(st, "permute")


def spmv(n, k, ja, values, u, out, bnd=None, stream=None):
    """out = A u over the fixed-width CSR (ja, values); out[bnd] = u[bnd]."""
    nb = 0 if bnd is None else bnd.numel()
    st = lib().rbfb_spmv(n, k, _ptr(ja), _ptr(values), _ptr(u), _ptr(out), _ptr(bnd), nb,
                         _stream(stream))
    if st != OK:
        raise RbfError(st, "spmv")


def store_to_csr(nstencils, ia, wxx, wyy, va, stream=None):
    st = lib().rbfb_store_to_csr(nstencils, _ptr(ia), _ptr(wxx), _ptr(wyy), _ptr(va),
                                 _stream(stream))
    if st != OK:
        raise RbfError(st, "store_to_csr")


def fill_kernel(nstencils, x, y, ia, ja, M, ldm, stream=None):
    """rbfb_fill_kernel: the Fortran fill_kernel (degree 2, r^3, absolute
    coordinates), stencil s's matrix at M[s*ldm*ldm:]."""
    st = lib().rbfb_fill_kernel(nstencils, _ptr(x), _ptr(y), _ptr(ia), _ptr(ja), _ptr(M), ldm,
                                _stream(stream))
    if st != OK:
        raise RbfError(st, "fill_kernel")


def fill_rhs(n, x, y, xc, yc, B, ldb, stream=None):
    """rbfb_fill_rhs: the Fortran fill_rhs (interpolation right-hand sides)."""
    st = lib().rbfb_fill_rhs(n, _ptr(x), _ptr(y), xc.numel(), _ptr(xc), _ptr(yc), _ptr(B), ldb,
                             _stream(stream))
    if st != OK:
        raise RbfError(st, "fill_rhs")


def store_to_csr_stencil(nstencils, ia, va, W, ldw, idx, stream=None):
    """rbfb_store_to_csr_stencil: the Fortran store_to_csr for stencil idx."""
    st = lib().rbfb_store_to_csr_stencil(nstencils, _ptr(ia), _ptr(va), _ptr(W), ldw, idx,
                                         _stream(stream))
    if st != OK:
        raise RbfError(st, "store_to_csr_stencil")


# ---- D2Q9 lattice Boltzmann (src/lbm/d2q9_kernels.cu) ----------------------
LBM_FP64, LBM_FP32 = 0, 1
# lattice velocities c_a, a = 0..8: rest, E, N, W, S, NE, NW, SW, SE
LBM_C = ((0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1))


def _lbm_prec(t):
    import torch
    if t.dtype == torch.float64:
        return LBM_FP64
    if t.dtype == torch.float32:
        return LBM_FP32
    raise TypeError("LBM arrays are float32 or float64")


def lbm_feq(rho, ux, uy, pdf, stream=None):
    """pdf (9n) <- equilibrium populations of rho, ux, uy: feq_kernel."""
    st = lib().rbfb_lbm_feq(rho.numel(), _lbm_prec(rho), _ptr(rho), _ptr(ux), _ptr(uy),
                            _ptr(pdf), _stream(stream))
    if st != OK:
        raise RbfError(st, "lbm_feq")


def lbm_macros(pdf, rho, ux, uy, stream=None):
    """rho, ux, uy <- moments of pdf: macros_kernel."""
    st = lib().rbfb_lbm_macros(rho.numel(), _lbm_prec(rho), _ptr(pdf), _ptr(rho), _ptr(ux),
                               _ptr(uy), _stream(stream))
    if st != OK:
        raise RbfError(st, "lbm_macros")


def lbm_bgk(omega, pdf, rho, ux, uy, indp=None, stream=None):
    """BGK collision in place (bgk_kernel; bgk_kernel_split with indp)."""
    st = lib().rbfb_lbm_bgk(rho.numel(), _lbm_prec(rho), float(omega), _ptr(pdf), _ptr(rho),
                            _ptr(ux), _ptr(uy), _ptr(indp), _stream(stream))
    if st != OK:
        raise RbfError(st, "lbm_bgk")


def lbm_stream_collide(k, ja, W, omega, pdf_in, pdf_out, rho=None, ux=None, uy=None,
                       stream=None):
    """One semi-Lagrangian step: stream pdf_in through the interpolation
    operators W (8*n*k float64, direction a at [(a-1)*n*k:]) and collide into
    pdf_out."""
    n = pdf_in.numel() // 9
    st = lib().rbfb_lbm_stream_collide(n, _lbm_prec(pdf_in), k, _ptr(ja), _ptr(W), float(omega),
                                       _ptr(pdf_in), _ptr(pdf_out), _ptr(rho), _ptr(ux),
                                       _ptr(uy), _stream(stream))
    if st != OK:
        raise RbfError(st, "lbm_stream_collide")


def lbm_departure_points(dt):
    """The 8 departure points -c_a dt (a = 1..8) in a stencil's local frame:
    the interpolation points of the streaming operators."""
    xc = np.array([-c[0] * dt for c in LBM_C[1:]], np.float64)
    yc = np.array([-c[1] * dt for c in LBM_C[1:]], np.float64)
    return xc, yc


def solve_dp(A, ipiv, B, info, stream=None):
    st = lib().rbfb_solve_dp(_ptr(A), _ptr(ipiv), _ptr(B), _ptr(info), _stream(stream))
    if st != OK:
        raise RbfError(st, "solve_dp")


class Server:
    """``rbfb_server``: continuous-batching assembly requests with device-
    resident results, admitted under an HBM budget."""

    def __init__(self, device=0, hbm_budget=40 << 30, max_slots=8):
        h = C.c_void_p()
        st = lib().rbfb_server_create(C.byref(h), device, int(hbm_budget), max_slots)
        if st != OK:
            raise RbfError(st, "server_create")
        self.h = h

    def submit(self, x_h, y_h, k, desc: Desc) -> int:
        x_h = np.ascontiguousarray(x_h, np.float64)
        y_h = np.ascontiguousarray(y_h, np.float64)
        r = Request()
        r.n = x_h.size
        r.x_h = x_h.ctypes.data
        r.y_h = y_h.ctypes.data
        r.k = k
        r.desc = desc
        t = C.c_longlong()
        st = lib().rbfb_server_submit(self.h, C.byref(r), C.byref(t))
        if st != OK:
            raise RbfError(st, "server_submit")
        return t.value

    def poll(self, ticket, wait_ms=-1):
        res = Result()
        st = lib().rbfb_server_poll(self.h, ticket, wait_ms, C.byref(res))
        return st, res

    def fetch(self, ticket, n, k, nrhs, with_ja=False):
        vals = [np.empty(n * k, np.float64) for _ in range(nrhs)]
        tab = (C.c_void_p * nrhs)(*[v.ctypes.data for v in vals])
        ja = np.empty(n * k, np.int32) if with_ja else None
        st = lib().rbfb_server_fetch(self.h, ticket, None if ja is None else ja.ctypes.data, tab)
        if st != OK:
            raise RbfError(st, "server_fetch")
        return vals, ja

    def release(self, ticket):
        return lib().rbfb_server_release(self.h, ticket)

    def resident_bytes(self):
        return int(lib().rbfb_server_resident_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().rbfb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
