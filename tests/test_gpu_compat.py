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
