"""The Fortran-module and solve_dp counterparts against the oracle/LAPACK."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as O
import rbf_b200 as R
from conftest import golden

pytestmark = pytest.mark.gpu


def test_solve_dp_matches_lapack(torch_cuda):
    T = torch_cuda
    rng = np.random.default_rng(3)
    A = rng.standard_normal((15, 15))
    B = rng.standard_normal((15, 9))
    Ad = T.as_tensor(A.T.copy().ravel()).cuda()  # column-major
    Bd = T.as_tensor(B.T.copy().ravel()).cuda()
    ipiv = T.zeros(15, dtype=T.int32, device="cuda")
    info = T.zeros(1, dtype=T.int32, device="cuda")
    R.solve_dp(Ad, ipiv, Bd, info)
    T.cuda.synchronize()
    assert int(info.item()) == 0
    X = Bd.cpu().numpy().reshape(9, 15).T
    np.testing.assert_allclose(X, np.linalg.solve(A, B), rtol=1e-10, atol=1e-12)
    lu, piv = sl.lu_factor(A)
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv + 1)
    np.testing.assert_allclose(Ad.cpu().numpy().reshape(15, 15).T, lu, rtol=1e-12, atol=1e-13)


def test_solve_dp_singular(torch_cuda):
    T = torch_cuda
    A = np.eye(15)
    A[4, 4] = 0.0
    Ad = T.as_tensor(A.T.copy().ravel()).cuda()
    Bd = T.ones(15 * 9, dtype=T.float64, device="cuda")
    ipiv = T.zeros(15, dtype=T.int32, device="cuda")
    info = T.zeros(1, dtype=T.int32, device="cuda")
    R.solve_dp(Ad, ipiv, Bd, info)
    T.cuda.synchronize()
    assert int(info.item()) == 5


def test_fill_matrices_match_oracle(ctx, torch_cuda):
    T = torch_cuda
    g = golden("square69_k21")
    k, P = 21, 2
    n = 200
    ia = np.arange(n + 1, dtype=np.int32) * k
    ja = g["ja_nanoflann"][: n * k]
    ldm = 32
    M = T.zeros(n * ldm * ldm, dtype=T.float64, device="cuda")
    d = R.make_desc(P)
    x = T.as_tensor(g["x"]).cuda()
    y = T.as_tensor(g["y"]).cuda()
    # only the first n stencils: x, y stay complete (neighbours index them);
    # the device arrays are held in names so they live through the launch
    iad = T.as_tensor(ia).cuda()
    jad = T.as_tensor(ja).cuda()
    st = R.lib().rbfb_fill_matrices(ctx.h, d, n, x.data_ptr(), y.data_ptr(), iad.data_ptr(),
                                    jad.data_ptr(), M.data_ptr(), ldm, None)
    assert st == 0
    T.cuda.synchronize()
    Mh = M.cpu().numpy().reshape(n, ldm, ldm)
    for s in (0, 17, 199):
        Mo, e = O.fill_matrix(s, g["x"], g["y"], ja[s * k:(s + 1) * k].copy(), P)
        np.testing.assert_array_equal(Mh[s].T[: k + 6, : k + 6], Mo)


def test_store_to_csr(torch_cuda):
    T = torch_cuda
    ia = T.as_tensor(np.array([0, 3, 7, 12], np.int32)).cuda()
    a = T.arange(12, dtype=T.float64, device="cuda")
    b = T.full((12,), 0.5, dtype=T.float64, device="cuda")
    va = T.zeros(12, dtype=T.float64, device="cuda")
    R.store_to_csr(3, ia, a, b, va)
    T.cuda.synchronize()
    np.testing.assert_array_equal(va.cpu().numpy(), np.arange(12) + 0.5)


def test_fortran_fill_kernel_absolute(torch_cuda):
    """rbfb_fill_kernel, the Fortran fill_kernel: degree 2, r^3, from the
    absolute coordinates, against the oracle's fill in that mode and, where
    built, the reference's own fill_matrix on the same coordinates."""
    T = torch_cuda
    g = golden("square69_k21")
    k, n, ldm = 21, 64, 28
    ja = g["ja_nanoflann"][: n * k].copy()
    ia = np.arange(n + 1, dtype=np.int32) * k
    M = T.full((n * ldm * ldm,), -7.0, dtype=T.float64, device="cuda")
    x = T.as_tensor(g["x"]).cuda()
    y = T.as_tensor(g["y"]).cuda()
    iad, jad = T.as_tensor(ia).cuda(), T.as_tensor(ja).cuda()
    R.fill_kernel(n, x, y, iad, jad, M, ldm)
    T.cuda.synchronize()
    Mh = M.cpu().numpy().reshape(n, ldm, ldm)
    for s in (0, 5, 63):
        idx = ja[s * k:(s + 1) * k]
        Mo, e = O.fill_matrix(s, g["x"], g["y"], idx, 2, 3, scale=False, shift=False)
        assert e == 0
        np.testing.assert_array_equal(Mh[s].T[: k + 6, : k + 6], Mo)
        ref = O.ref_fill(g["x"][idx], g["y"][idx], 2, 3)
        if ref is not None:
            np.testing.assert_array_equal(Mo, ref[0])


def test_fortran_fill_rhs(torch_cuda):
    """rbfb_fill_rhs, the Fortran fill_rhs, against the reference's own
    fill_rhs (where built) and a plain restatement."""
    T = torch_cuda
    rng = np.random.default_rng(9)
    n, nc, ldb = 21, 3, 30
    xs, ys = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    xc, yc = rng.uniform(-0.2, 0.2, nc), rng.uniform(-0.2, 0.2, nc)
    B = T.full((ldb * nc,), -7.0, dtype=T.float64, device="cuda")
    R.fill_rhs(n, T.as_tensor(xs).cuda(), T.as_tensor(ys).cuda(), T.as_tensor(xc).cuda(),
               T.as_tensor(yc).cuda(), B, ldb)
    T.cuda.synchronize()
    Bh = B.cpu().numpy().reshape(nc, ldb).T
    for j in range(nc):
        r2 = (xc[j] - xs) * (xc[j] - xs) + (yc[j] - ys) * (yc[j] - ys)
        np.testing.assert_array_equal(Bh[:n, j], r2 * np.sqrt(r2))
        want = [1.0, xc[j], yc[j], xc[j] * xc[j], xc[j] * yc[j], yc[j] * yc[j]]
        np.testing.assert_array_equal(Bh[n:n + 6, j], want)
    np.testing.assert_array_equal(Bh[n + 6:, :], -7.0)  # rows past the system untouched
    ref = O.ref_fill(xs, ys, 2, 3, xc, yc)
    if ref is not None:
        np.testing.assert_array_equal(Bh[:n + 6, :], ref[1])


def test_fortran_store_to_csr_stencil(torch_cuda):
    T = torch_cuda
    ia = T.as_tensor(np.array([0, 3, 7, 12], np.int32)).cuda()
    ldw = 6
    W = T.as_tensor(np.arange(2 * ldw, dtype=np.float64)).cuda()  # W(:,1) = 0..5, W(:,2) = 6..11
    va = T.zeros(12, dtype=T.float64, device="cuda")
    R.store_to_csr_stencil(3, ia, va, W, ldw, 1)
    T.cuda.synchronize()
    want = np.zeros(12)
    want[3:7] = np.arange(4) + np.arange(6, 10)
    np.testing.assert_array_equal(va.cpu().numpy(), want)
    with pytest.raises(R.RbfError):
        R.store_to_csr_stencil(3, ia, va, W, ldw, 3)
