"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may
import this module: it is the checker and the CPU baseline, never part of the
product. It loads

* ``oracle/_build/liboracle.so`` -- the CPU restatement of the reference's
  assembly path (``oracle/rbf_oracle.cpp``), and
* ``oracle/_ref/libref_knn.so`` -- the reference's own nanoflann / ckdtree
  stencil searches compiled from the reference sources (``oracle/Makefile``),
* ``oracle/_ref/libref_fill.so`` -- the reference's own ``fill_matrix`` /
  ``fill_rhs`` templates (``src/rbf_operators.h:39-185``) compiled from its
  header against a declarations-only cuSolverDx stand-in.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libref_knn.so"
REF_FILL_SO = HERE / "_ref" / "libref_fill.so"

OP_INTERP, OP_LAPLACE, OP_DX, OP_DY, OP_DXX, OP_DYY, OP_DXY = 1, 2, 4, 8, 16, 32, 64

_lib = None
_ref = None
_ref_fill = None

_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def lib():
    """The oracle library (built by ``make -C oracle``)."""
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        L = C.CDLL(str(ORACLE_SO))
        L.orc_assemble_fixed.restype = C.c_longlong
        L.orc_assemble_fixed.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                         C.c_double, C.c_void_p, C.c_void_p]
        L.orc_assemble_csr.restype = C.c_longlong
        L.orc_assemble_csr.argtypes = [C.c_int, _dp, _dp, _ip, _ip, C.c_void_p, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_solve_stencil.restype = C.c_int
        L.orc_solve_stencil.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                        C.c_double, _dp, C.c_void_p]
        L.orc_fill_matrix.restype = C.c_int
        L.orc_fill_matrix.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, C.c_int, C.c_int,
                                      C.c_double, C.c_double, _dp, C.c_int, C.c_int]
        L.orc_knn_brute.restype = C.c_int
        L.orc_knn_brute.argtypes = [C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_int, C.c_double,
                                    C.c_double, _ip, C.c_void_p]
        L.orc_stencil_d2.restype = None
        L.orc_stencil_d2.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_double, C.c_double, _dp]
        L.orc_num_rhs.restype = C.c_int
        L.orc_num_rhs.argtypes = [C.c_int, C.c_int]
        L.orc_npoly.restype = C.c_int
        L.orc_npoly.argtypes = [C.c_int]
        L.orc_assemble_fixed_ld.restype = C.c_longlong
        L.orc_assemble_fixed_ld.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, C.c_int,
                                            C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                            C.c_void_p]
        L.orc_spmv.restype = None
        L.orc_spmv.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, _dp, C.c_void_p, C.c_int]
        L.orc_solve_grid.restype = C.c_int
        L.orc_solve_grid.argtypes = [C.c_int, C.c_int]
        L.orc_bicgstab.restype = C.c_int
        L.orc_bicgstab.argtypes = [C.c_int, C.c_int, C.c_void_p, _ip, _dp, C.c_void_p, C.c_int,
                                   _dp, _dp, C.c_double, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_curve_keys.restype = C.c_int
        L.orc_curve_keys.argtypes = [C.c_int, _dp, _dp, C.c_void_p, C.c_int, C.c_int,
                                     np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
        L.orc_curve_order.restype = C.c_int
        L.orc_curve_order.argtypes = [C.c_int, _dp, _dp, C.c_void_p, C.c_int, C.c_int, _ip]
        L.orc_boundary_last.restype = None
        L.orc_boundary_last.argtypes = [C.c_int, _ip, _ip]
        L.orc_renumber_stencils.restype = None
        L.orc_renumber_stencils.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip]
        L.orc_renumber_csr.restype = None
        L.orc_renumber_csr.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _ip]
        L.orc_system.restype = C.c_int
        L.orc_system.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, C.c_int, C.c_int,
                                 C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double,
                                 _dp, _dp, _dp]
        for nm in ("orc_lbm_feq", "orc_lbm_macros", "orc_lbm_bgk", "orc_lbm_stream_collide"):
            getattr(L, nm).restype = None
        L.orc_lbm_feq.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4
        L.orc_lbm_macros.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4
        L.orc_lbm_bgk.argtypes = [C.c_int, C.c_int, C.c_double] + [C.c_void_p] * 5
        L.orc_lbm_stream_collide.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _dp, C.c_double,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
        L.orc_phs.restype = C.c_double
        L.orc_phs.argtypes = [C.c_int, C.c_double]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def ref():
    """The reference's own stencil searches, or None when not built here."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        L = C.CDLL(str(REF_SO))
        L.ref_nodeset_stencils.restype = C.c_int
        L.ref_nodeset_stencils.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip]
        L.ref_kdtree_stencils.restype = C.c_int
        L.ref_kdtree_stencils.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, _ip]
        L.ref_set_threads.argtypes = [C.c_int]
        _ref = L
    return _ref


def ref_fill_lib():
    """The reference's own fill templates, or None when not built here."""
    global _ref_fill
    if _ref_fill is None:
        if not REF_FILL_SO.exists():
            return None
        L = C.CDLL(str(REF_FILL_SO))
        L.ref_fill.restype = C.c_int
        L.ref_fill.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp]
        _ref_fill = L
    return _ref_fill


def ref_fill(xs, ys, P, Q, xc=(), yc=()):
    """The reference's fill_matrix and fill_rhs (src/rbf_operators.h:116-185)
    on stencil-local coordinates: (M, B) as numpy (nt, nt) and (nt, nc)
    arrays in the reference's layout (node rows first, then the monomials),
    or None when the library or the (k, P, Q) combination is absent."""
    L = ref_fill_lib()
    if L is None:
        return None
    xs, ys = _f64(xs), _f64(ys)
    xc, yc = _f64(np.asarray(xc, np.float64).ravel()), _f64(np.asarray(yc, np.float64).ravel())
    k = xs.size
    nt = k + npoly(P)
    M = np.zeros(nt * nt)
    B = np.zeros(nt * max(xc.size, 1))
    if L.ref_fill(k, P, Q, xs, ys, xc.size, xc if xc.size else np.zeros(1),
                  yc if yc.size else np.zeros(1), M, B) < 0:
        return None
    return M.reshape(nt, nt).T.copy(), B[:nt * xc.size].reshape(xc.size, nt).T.copy()


def system(s, x, y, idx, P, Q=None, ops=OP_LAPLACE | OP_DX | OP_DY, xc=None, yc=None,
           scale=True, period=None):
    """The oracle's augmented system of stencil s as its elimination receives
    it: (xs, ys, a, e) with the local coordinates, a = row-major n x (n+nrhs)
    (polynomial block first, right-hand sides last) and the scale exponent."""
    x, y, idx = _f64(x), _f64(y), _i32(idx)
    k = idx.size
    Q = 2 * P - 1 if Q is None else Q
    nc = 0 if xc is None else len(xc)
    nrhs = num_rhs(ops, nc)
    n = k + npoly(P)
    xs, ys = np.empty(k), np.empty(k)
    a = np.empty(n * (n + nrhs))
    xcp = None if xc is None else _f64(xc)
    ycp = None if yc is None else _f64(yc)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    e = lib().orc_system(s, x, y, k, idx, P, Q, ops, nc,
                         None if xcp is None else xcp.ctypes.data,
                         None if ycp is None else ycp.ctypes.data, int(bool(scale)), Lx, Ly,
                         xs, ys, a)
    if e == -1000:
        raise ValueError("oracle rejected the arguments")
    return xs, ys, a.reshape(n, n + nrhs), e


def _lbm_p(a):
    return 0 if a.dtype == np.float64 else 1


def lbm_feq(rho, ux, uy):
    """feq_kernel restated: the 9 x n planar equilibrium populations."""
    pdf = np.empty(9 * rho.size, rho.dtype)
    lib().orc_lbm_feq(rho.size, _lbm_p(rho), rho.ctypes.data, ux.ctypes.data, uy.ctypes.data,
                      pdf.ctypes.data)
    return pdf


def lbm_macros(pdf):
    """macros_kernel restated: (rho, ux, uy) of planar populations."""
    n = pdf.size // 9
    rho, ux, uy = (np.empty(n, pdf.dtype) for _ in range(3))
    lib().orc_lbm_macros(n, _lbm_p(pdf), pdf.ctypes.data, rho.ctypes.data, ux.ctypes.data,
                         uy.ctypes.data)
    return rho, ux, uy


def lbm_bgk(pdf, omega):
    """bgk_kernel_split restated on a copy: (pdf, rho, ux, uy, indp)."""
    pdf = np.array(pdf, copy=True)
    n = pdf.size // 9
    rho, ux, uy, indp = (np.empty(n, pdf.dtype) for _ in range(4))
    lib().orc_lbm_bgk(n, _lbm_p(pdf), float(omega), pdf.ctypes.data, rho.ctypes.data,
                      ux.ctypes.data, uy.ctypes.data, indp.ctypes.data)
    return pdf, rho, ux, uy, indp


def lbm_stream_collide(k, ja, W, omega, pdf):
    """One streaming + collision step restated: (pdf_out, rho, ux, uy)."""
    n = pdf.size // 9
    out = np.empty_like(pdf)
    rho, ux, uy = (np.empty(n, pdf.dtype) for _ in range(3))
    lib().orc_lbm_stream_collide(n, _lbm_p(pdf), k, _i32(ja), _f64(W), float(omega),
                                 pdf.ctypes.data, out.ctypes.data, rho.ctypes.data,
                                 ux.ctypes.data, uy.ctypes.data)
    return out, rho, ux, uy


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))
    r = ref()
    if r is not None:
        r.ref_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def npoly(P: int) -> int:
    return (P + 1) * (P + 2) // 2 if P >= 0 else 0


def num_rhs(ops: int, nc: int = 0) -> int:
    return int(lib().orc_num_rhs(ops, nc))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr_table(arrs):
    t = (C.c_void_p * len(arrs))()
    for i, a in enumerate(arrs):
        t[i] = a.ctypes.data
    return t


def assemble(x, y, ja, k, P, Q=None, ops=OP_LAPLACE | OP_DX | OP_DY, xc=None, yc=None,
             scale=True, period=None):
    """FP64 assembly of fixed-width stencils (ja: n*k). Returns (values, info)
    with values of shape (nrhs, n*k)."""
    x, y, ja = _f64(x), _f64(y), _i32(ja)
    n = x.size
    Q = 2 * P - 1 if Q is None else Q
    nc = 0 if xc is None else len(xc)
    xc_a = None if xc is None else _f64(xc)
    yc_a = None if yc is None else _f64(yc)
    nrhs = num_rhs(ops, nc)
    out = [np.empty(n * k, np.float64) for _ in range(nrhs)]
    info = np.zeros(n, np.int32)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    rc = lib().orc_assemble_fixed(n, x, y, k, ja, P, Q, ops, nc,
                                  None if xc_a is None else xc_a.ctypes.data,
                                  None if yc_a is None else yc_a.ctypes.data, int(bool(scale)),
                                  Lx, Ly, _ptr_table(out), info.ctypes.data)
    if rc < 0:
        raise ValueError("oracle rejected the arguments")
    return np.stack(out), info


def assemble_ld(x, y, ja, k, P, Q=None, ops=OP_LAPLACE | OP_DX | OP_DY, scale=True, period=None,
                nstencils=None):
    """The same assembly in x87 long double (64-bit significand): a more
    accurate solution to measure FP64 and refined-FP32 errors against on
    ill-conditioned stencils. Derivative operators only. nstencils restricts
    it to the stencils of the first nodes (ja then holds only their rows)."""
    x, y, ja = _f64(x), _f64(y), _i32(ja)
    n = x.size if nstencils is None else int(nstencils)
    Q = 2 * P - 1 if Q is None else Q
    nrhs = num_rhs(ops, 0)
    out = [np.empty(n * k, np.float64) for _ in range(nrhs)]
    info = np.zeros(n, np.int32)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    rc = lib().orc_assemble_fixed_ld(n, x, y, k, ja, P, Q, ops, int(bool(scale)), Lx, Ly,
                                     _ptr_table(out), info.ctypes.data)
    if rc < 0:
        raise ValueError("oracle rejected the arguments")
    return np.stack(out), info


def assemble_csr(x, y, ia, ja, degree=None, P=2, Q=0, ops=OP_LAPLACE | OP_DX | OP_DY,
                 scale=True, period=None, nstencils=None):
    """FP64 assembly of ragged CSR stencils; degree: per-stencil int8 or None.
    Q = 0 selects Q_s = 2 P_s - 1. Stencil s is centred on node s; by default
    every node has a stencil, nstencils restricts it to the first ones."""
    x, y, ia, ja = _f64(x), _f64(y), _i32(ia), _i32(ja)
    n = x.size if nstencils is None else int(nstencils)
    nrhs = num_rhs(ops, 0)
    out = [np.empty(int(ia[-1]), np.float64) for _ in range(nrhs)]
    info = np.zeros(n, np.int32)
    deg = None if degree is None else np.ascontiguousarray(degree, dtype=np.int8)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    rc = lib().orc_assemble_csr(n, x, y, ia, ja, None if deg is None else deg.ctypes.data, P, Q,
                                ops, 0, None, None, int(bool(scale)), Lx, Ly, _ptr_table(out),
                                info.ctypes.data)
    if rc < 0:
        raise ValueError("oracle rejected the arguments")
    return np.stack(out), info


def solve_stencil(s, x, y, idx, P, Q=None, ops=OP_LAPLACE | OP_DX | OP_DY, scale=True,
                  period=None):
    """Full solution (np polynomial coefficients, then k weights) of one
    stencil in the scaled frame, shape (n, nrhs); plus info."""
    x, y, idx = _f64(x), _f64(y), _i32(idx)
    k = idx.size
    Q = 2 * P - 1 if Q is None else Q
    nrhs = num_rhs(ops, 0)
    n = k + npoly(P)
    sol = np.empty(n * nrhs, np.float64)
    out = [np.empty(k, np.float64) for _ in range(nrhs)]
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    info = lib().orc_solve_stencil(s, x, y, k, idx, P, Q, ops, 0, None, None, int(bool(scale)),
                                   Lx, Ly, sol, _ptr_table(out))
    return sol.reshape(n, nrhs), info


def fill_matrix(s, x, y, idx, P, Q=None, scale=True, period=None, shift=True):
    """The reference-layout saddle-point matrix [A P; P^T 0] of one stencil
    (column-major in the reference; returned as a numpy (n, n) array);
    shift=False fills from the absolute coordinates (the Fortran
    fill_kernel)."""
    x, y, idx = _f64(x), _f64(y), _i32(idx)
    k = idx.size
    Q = 2 * P - 1 if Q is None else Q
    n = k + npoly(P)
    M = np.empty(n * n, np.float64)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    e = lib().orc_fill_matrix(s, x, y, k, idx, P, Q, int(bool(scale)), Lx, Ly, M, n,
                              int(bool(shift)))
    return M.reshape(n, n).T.copy(), e


def knn_brute(x, y, k, xq=None, yq=None, period=None, return_d2=False):
    """Brute-force k-NN ordered by (squared distance, index) in the
    reference's distance arithmetic. O(n) per query."""
    x, y = _f64(x), _f64(y)
    xq = x if xq is None else _f64(xq)
    yq = y if yq is None else _f64(yq)
    nq = xq.size
    ja = np.empty(nq * k, np.int32)
    d2 = np.empty(nq * k, np.float64) if return_d2 else None
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    rc = lib().orc_knn_brute(x.size, x, y, nq, xq, yq, k, Lx, Ly, ja,
                             None if d2 is None else d2.ctypes.data)
    if rc < 0:
        raise ValueError("bad k")
    return (ja, d2) if return_d2 else ja


def stencil_d2(x, y, ja, k, period=None):
    """Squared distances of a stencil table, in the reference's arithmetic."""
    x, y, ja = _f64(x), _f64(y), _i32(ja)
    d2 = np.empty(ja.size, np.float64)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    lib().orc_stencil_d2(x.size, x, y, k, ja, Lx, Ly, d2)
    return d2


def ref_nodeset_stencils(x, y, k):
    """rbf::NodeSet::stencils(k) of the reference (nanoflann, open plane)."""
    r = ref()
    if r is None:
        raise RuntimeError("reference search library not built (oracle/_ref)")
    x, y = _f64(x), _f64(y)
    ja = np.empty(x.size * k, np.int32)
    if r.ref_nodeset_stencils(x.size, x, y, k, ja) != 0:
        raise ValueError("bad k")
    return ja


def ref_kdtree_stencils(x, y, k, period=None):
    """rbf::spatial::KdTree::knn_stencils(k) of the reference (ckdtree)."""
    r = ref()
    if r is None:
        raise RuntimeError("reference search library not built (oracle/_ref)")
    x, y = _f64(x), _f64(y)
    ja = np.empty(x.size * k, np.int32)
    Lx, Ly = (0.0, 0.0) if period is None else (float(period[0]), float(period[1]))
    if r.ref_kdtree_stencils(x.size, x, y, k, Lx, Ly, ja) != 0:
        raise ValueError("bad k")
    return ja


def spmv(ja, values, u, k, bnd=None):
    """out = A u (row-order fused multiply-adds from zero), out[bnd] = u[bnd]."""
    ja, values, u = _i32(ja), _f64(values), _f64(u)
    n = ja.size // k
    out = np.empty(n, np.float64)
    b = None if bnd is None else _i32(bnd)
    lib().orc_spmv(n, k, ja, values, u, out, None if b is None else b.ctypes.data,
                   0 if b is None else b.size)
    return out


def solve_grid(n, sms):
    """Blocks of the CUDA solver's reductions for n rows on `sms` SMs."""
    return lib().orc_solve_grid(n, sms)


def bicgstab(values, ja, f, u0, k=None, ia=None, bnd=None, tol=1e-10, maxit=10000, grid=1):
    """BiCGSTAB with the CUDA solver's summation order for a grid of `grid`
    blocks. Returns (status, u, iters, relres); status 0, -10 (maxit) or
    -11 (breakdown); ValueError on bad arguments."""
    values, ja, f = _f64(values), _i32(ja), _f64(f)
    u = _f64(u0).copy()
    n = f.size
    iaa = None if ia is None else _i32(ia)
    b = None if bnd is None else _i32(bnd)
    it, rel = C.c_int(0), C.c_double(0.0)
    st = lib().orc_bicgstab(n, 0 if k is None else k, None if iaa is None else iaa.ctypes.data,
                            ja, values, None if b is None else b.ctypes.data,
                            0 if b is None else b.size, f, u, tol, maxit, grid, C.byref(it),
                            C.byref(rel))
    if st == -1:
        raise ValueError("bad bicgstab arguments")
    return st, u, it.value, rel.value


MORTON, HILBERT = 0, 1


def curve_keys(x, y, ndiv=16, curve=MORTON, bbox=None):
    """zidx / hidx keys of every point (int64)."""
    x, y = _f64(x), _f64(y)
    keys = np.empty(x.size, np.int64)
    bb = None if bbox is None else (C.c_double * 4)(*bbox)
    if lib().orc_curve_keys(x.size, x, y, bb, ndiv, curve, keys) < 0:
        raise ValueError("bad ndiv or curve")
    return keys


def curve_order(x, y, ndiv=16, curve=MORTON, bbox=None):
    """morton_order / hilbert_order: perm[new] = old (stable)."""
    x, y = _f64(x), _f64(y)
    perm = np.empty(x.size, np.int32)
    bb = None if bbox is None else (C.c_double * 4)(*bbox)
    if lib().orc_curve_order(x.size, x, y, bb, ndiv, curve, perm) < 0:
        raise ValueError("bad ndiv or curve")
    return perm


def boundary_last(flag):
    flag = _i32(flag)
    perm = np.empty(flag.size, np.int32)
    lib().orc_boundary_last(flag.size, flag, perm)
    return perm


def renumber_stencils(ja, k, perm):
    ja, perm = _i32(ja), _i32(perm)
    out = np.empty_like(ja)
    lib().orc_renumber_stencils(perm.size, k, ja, perm, out)
    return out


def renumber_csr(ia, ja, perm):
    ia, ja, perm = _i32(ia), _i32(ja), _i32(perm)
    ia_out = np.empty_like(ia)
    ja_out = np.empty_like(ja)
    lib().orc_renumber_csr(perm.size, ia, ja, perm, ia_out, ja_out)
    return ia_out, ja_out


def max_rel_err(w, w_ref, k):
    """Per stencil and right-hand side, ||w - w_ref||_inf / ||w_ref||_inf;
    returns the maximum over stencils for every right-hand side."""
    w = np.asarray(w).reshape(w.shape[0], -1, k)
    w_ref = np.asarray(w_ref).reshape(w_ref.shape[0], -1, k)
    num = np.abs(w - w_ref).max(axis=2)
    den = np.abs(w_ref).max(axis=2)
    den = np.where(den > 0, den, 1.0)
    return (num / den).max(axis=1)


if os.environ.get("RBFB_ORACLE_THREADS"):
    set_threads(int(os.environ["RBFB_ORACLE_THREADS"]))
