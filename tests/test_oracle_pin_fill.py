"""The oracle's saddle-point system against the reference's own fill code.

The reference's PHS<Q>, PolyBasis<P>, fill_matrix<N,P,Q> and
fill_rhs<N,P,NRHS,Q> (src/rbf_operators.h:39-185) are plain host/device
templates. oracle/Makefile compiles them from the reference header where it
lies (oracle/ref_fill.cu, with a declarations-only stand-in for the closed
cuSolverDx header) into oracle/_ref/libref_fill.so. Here the oracle's system
-- the matrix and interpolation right-hand sides its elimination receives --
must equal the reference's bit for bit, after the relabelling the oracle
documents (polynomial block first). With the GPU fill and the FP64 weights
bit-identical to the oracle (tests/test_gpu_*), the weights chain is then
pinned to the reference from the coordinates through the fill; only the
project's elimination stands between it and the weights.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.skipif(O.ref_fill_lib() is None,
                                reason="reference fill not built (needs the reference checkout)")


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


def _cases():
    g = golden("shu_square_4786")
    yield "shu_square_4786", g["x"], g["y"], g["ja_nanoflann"], 21, 2, 3, None
    g = golden("periodic64_k35")
    yield "periodic64_k35", g["x"], g["y"], g["ja_ckdtree"], 35, 3, 5, tuple(g["box"])
    c = NS.config_small()
    ja = O.knn_brute(c["x"], c["y"], 28)
    yield "square69_k28", c["x"], c["y"], ja, 28, 3, 5, None
    x, y, _ = NS.jittered_grid(40, 0.3, seed=11, periodic=True)
    ja = O.knn_brute(x, y, 64, period=(1.0, 1.0))
    yield "periodic40_k64", x, y, ja, 64, 4, 7, (1.0, 1.0)


@pytest.mark.parametrize("scale", [True, False])
@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_system_matches_reference_fill(case, scale):
    name, x, y, ja, k, P, Q, period = case
    np_ = O.npoly(P)
    n = k + np_
    # relabelling: reference row/unknown i (nodes first, then monomials) is
    # the oracle's perm[i] (monomials first, then nodes)
    perm = np.concatenate([np.arange(np_, n), np.arange(np_)])
    rng = np.random.default_rng(3)
    pts = rng.uniform(-0.5, 0.5, size=(2, 3)) * 0.05  # interpolation points, local frame
    stencils = rng.choice(x.size, 24, replace=False)
    for s in stencils:
        idx = ja[s * k:(s + 1) * k]
        xs, ys, a, e = O.system(int(s), x, y, idx, P, Q, ops=O.OP_INTERP, xc=pts[0], yc=pts[1],
                                scale=scale, period=period)
        # the reference fills from the same local coordinates; its
        # interpolation points are the oracle's after the same exact scaling
        M, B = O.ref_fill(xs, ys, P, Q, np.ldexp(pts[0], -e), np.ldexp(pts[1], -e))
        np.testing.assert_array_equal(_bits(a[np.ix_(perm, perm)]), _bits(M),
                                      err_msg=f"{name} stencil {s}: matrix")
        np.testing.assert_array_equal(_bits(a[perm, n:]), _bits(B),
                                      err_msg=f"{name} stencil {s}: right-hand sides")


def test_reference_fill_layout():
    """The reference's matrix is the documented [A P; P^T 0]: symmetric, zero
    diagonal in A, zero polynomial block, first monomial 1."""
    x, y, _ = NS.jittered_grid(16, 0.3, seed=5)
    ja = O.knn_brute(x, y, 21)
    xs, ys, _, _ = O.system(0, x, y, ja[:21], 2, 3, ops=O.OP_INTERP, xc=[0.0], yc=[0.0])
    M, B = O.ref_fill(xs, ys, 2, 3, [0.0], [0.0])
    assert M.shape == (27, 27) and B.shape == (27, 1)
    np.testing.assert_array_equal(M, M.T)
    np.testing.assert_array_equal(np.diag(M)[:21], 0.0)
    np.testing.assert_array_equal(M[21:, 21:], 0.0)
    np.testing.assert_array_equal(M[:21, 21], 1.0)
    # at the centre (node 0) the interpolation right-hand side is column 0
    np.testing.assert_array_equal(B[:, 0], M[:, 0])
