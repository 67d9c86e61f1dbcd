"""Mathematical checks of the CPU oracle (the weights have no reference
fixture: the reference's solver, cuSolverDx, is closed and absent).

* polynomial reproduction: sum_j w_j p(x_j - x_s) = (L p)(0) for every
  monomial of degree <= P, the defining property of PHS + polynomial RBF-FD;
* LU cross-check against scipy/LAPACK getrf/getrs on the reference-layout
  matrix [A P; P^T 0] (fill_matrix, src/rbf_operators.h:116-154);
* scale covariance: power-of-two radius scaling leaves the weights unchanged;
* operator consistency: d2/dx2 + d2/dy2 = Laplacian; interpolation at a node
  reproduces the unit vector;
* singular stencils: coincident nodes give info != 0 and NaN weights.
"""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as O
from conftest import golden
from rbf_b200 import nodesets as NS


def monomial_checks(x, y, ja, k, W, P, ops):
    n = x.size
    J = ja.reshape(n, k)
    dx = x[J] - x[:, None]
    dy = y[J] - y[:, None]
    h = np.abs(np.stack([dx, dy])).max(axis=(0, 2))[:, None]
    out = {}
    for q, op in enumerate(ops):
        w = W[q].reshape(n, k)
        worst = 0.0
        for d in range(P + 1):
            for j in range(d + 1):
                a, b = d - j, j
                p = dx ** a * dy ** b
                target = {O.OP_LAPLACE: 2.0 if (a, b) in ((2, 0), (0, 2)) else 0.0,
                          O.OP_DX: 1.0 if (a, b) == (1, 0) else 0.0,
                          O.OP_DY: 1.0 if (a, b) == (0, 1) else 0.0}[op]
                order = 2 if op == O.OP_LAPLACE else 1
                # relative to the weight scale |w| h^(a+b) ~ h^(a+b-order)
                scale = (np.abs(w) * np.abs(p)).sum(axis=1) + np.abs(target) * 0 + 1e-300
                err = np.abs((w * p).sum(axis=1) - target) / np.maximum(scale, h[:, 0] ** (a + b - order))
                worst = max(worst, float(err.max()))
        out[op] = worst
    return out


@pytest.mark.parametrize("src,key", [("square69_k21", "ja_nanoflann"), ("shu_square_4786", "ja_nanoflann")])
def test_polynomial_reproduction(src, key):
    g = golden(src)
    ops = [O.OP_LAPLACE, O.OP_DX, O.OP_DY]
    W, info = O.assemble(g["x"], g["y"], g[key], 21, 2)
    assert (info == 0).all()
    errs = monomial_checks(g["x"], g["y"], g[key], 21, W, 2, ops)
    assert max(errs.values()) < 1e-12, errs


def test_periodic_polynomial_reproduction():
    g = golden("periodic64_k35")
    W, info = O.assemble(g["x"], g["y"], g["ja_ckdtree"], 35, 3, period=(1.0, 1.0))
    assert (info == 0).all()
    # minimum-image displacements
    n, k = g["x"].size, 35
    J = g["ja_ckdtree"].reshape(n, k)
    dx = g["x"][J] - g["x"][:, None]
    dy = g["y"][J] - g["y"][:, None]
    dx -= np.rint(dx)
    dy -= np.rint(dy)
    L, Dx = W[0].reshape(n, k), W[1].reshape(n, k)
    for a, b in [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2), (3, 0), (2, 1), (0, 3)]:
        p = dx ** a * dy ** b
        t_l = 2.0 if (a, b) in ((2, 0), (0, 2)) else 0.0
        t_x = 1.0 if (a, b) == (1, 0) else 0.0
        sc = (np.abs(L) * np.abs(p)).sum(1) + 1.0
        assert (np.abs((L * p).sum(1) - t_l) / sc).max() < 1e-11
        sc = (np.abs(Dx) * np.abs(p)).sum(1) + 1.0
        assert (np.abs((Dx * p).sum(1) - t_x) / sc).max() < 1e-11


def test_lu_against_lapack():
    g = golden("shu_square_4786")
    k, P = 21, 2
    J = g["ja_nanoflann"].reshape(-1, k)
    np_ = O.npoly(P)
    worst = 0.0
    for s in range(0, J.shape[0], 61):
        M, e = O.fill_matrix(s, g["x"], g["y"], J[s].copy(), P)
        sol, info = O.solve_stencil(s, g["x"], g["y"], J[s].copy(), P)
        assert info == 0
        # the oracle orders unknowns polynomial first; LAPACK solves the
        # reference layout [w; lambda] with the same right-hand sides
        z = np.concatenate([sol[np_:], sol[:np_]])
        b = M @ z
        z2 = sl.lu_solve(sl.lu_factor(M), b)
        worst = max(worst, float(np.abs(z2 - z).max() / np.abs(z).max()))
    assert worst < 1e-12


def test_fill_matrix_structure():
    g = golden("square69_k21")
    k, P = 21, 2
    J = g["ja_nanoflann"].reshape(-1, k)
    M, e = O.fill_matrix(100, g["x"], g["y"], J[100].copy(), P)
    n = k + O.npoly(P)
    assert M.shape == (n, n)
    np.testing.assert_array_equal(M, M.T)               # symmetric
    np.testing.assert_array_equal(np.diag(M)[:k], 0.0)  # phi(0) = 0
    np.testing.assert_array_equal(M[k:, k:], 0.0)       # zero block
    np.testing.assert_array_equal(M[:k, k], 1.0)        # constant monomial
    # centre first, shifted to the origin
    assert M[0, k + 1] == 0.0 and M[0, k + 2] == 0.0
    assert 0.5 <= np.abs(M[:k, k + 1:k + 3]).max() < 1.0  # scaled into (-1, 1)


def test_scale_covariance():
    c = NS.config_small()
    ja = golden("square69_k21")["ja_nanoflann"]
    W1, _ = O.assemble(c["x"], c["y"], ja, 21, 2, scale=True)
    W0, _ = O.assemble(c["x"], c["y"], ja, 21, 2, scale=False)
    assert O.max_rel_err(W1, W0, 21).max() < 1e-11


def test_second_derivatives_sum_to_laplacian():
    g = golden("square69_k21")
    ops = O.OP_LAPLACE | O.OP_DXX | O.OP_DYY | O.OP_DXY
    W, info = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2, ops=ops)
    assert W.shape[0] == 4
    assert O.max_rel_err(W[1][None] + W[2][None], W[0][None], 21).max() < 1e-12


def test_interpolation_rhs_reproduces_node_values():
    g = golden("square69_k21")
    J = g["ja_nanoflann"].reshape(-1, 21)
    s = 500
    # interpolation points at two stencil nodes (local frame): weights = unit vectors
    xc = np.array([g["x"][J[s, 3]] - g["x"][s], 0.0])
    yc = np.array([g["y"][J[s, 3]] - g["y"][s], 0.0])
    W, info = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2, ops=O.OP_INTERP, xc=xc, yc=yc)
    w0 = W[0].reshape(-1, 21)[s]
    w1 = W[1].reshape(-1, 21)[s]
    e3 = np.zeros(21); e3[3] = 1.0
    e0 = np.zeros(21); e0[0] = 1.0
    assert np.abs(w0 - e3).max() < 1e-12
    assert np.abs(w1 - e0).max() < 1e-12


def test_singular_stencil_reports_info_and_nan():
    c = NS.config_small()
    x, y = c["x"].copy(), c["y"].copy()
    ja = golden("square69_k21")["ja_nanoflann"].copy().reshape(-1, 21)
    # stencil 7 gets a duplicated neighbour: two identical rows, singular matrix
    ja[7, 5] = ja[7, 4]
    W, info = O.assemble(x, y, ja.ravel(), 21, 2)
    assert info[7] != 0 and (np.delete(info, 7) == 0).all()
    assert np.isnan(W[:, 7 * 21:8 * 21]).all()


def test_collinear_stencil_is_singular():
    # all nodes of a stencil on one line: the degree-2 polynomial block is rank deficient
    n = 40
    x = np.linspace(0.0, 1.0, n)
    y = np.zeros(n)
    ja = O.knn_brute(x, y, 10)
    W, info = O.assemble(x, y, ja, 10, 2)
    assert (info != 0).all()


def test_long_double_agrees_on_well_conditioned_stencils():
    # the x87 long double solve (64-bit significand) and the FP64 oracle agree
    # to ~cond * 2^-53 on the degree-2 workload (cond ~ 4e3 scaled)
    g = golden("square69_k21")
    W, _ = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2)
    Wl, _ = O.assemble_ld(g["x"], g["y"], g["ja_nanoflann"], 21, 2)
    assert O.max_rel_err(W, Wl, 21).max() < 1e-12
