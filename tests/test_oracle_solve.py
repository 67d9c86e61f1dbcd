"""The CPU restatement of the BiCGSTAB solve on an assembled operator
(the step after the reference's mv_op, src/main.cpp:57-68), checked against
an independent direct sparse solve (scipy's SuperLU) and a manufactured
Poisson solution, plus its edge cases. The GPU solver is compared with this
restatement bit for bit in test_gpu_solve.py."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O
from rbf_b200 import nodesets as NS


def u_exact(x, y):
    return np.exp(x) * np.sin(2.0 * y) + x * x


def lap_exact(x, y):
    return -3.0 * np.exp(x) * np.sin(2.0 * y) + 2.0


def poisson_disk(n=2000, nb=160, k=21, P=2, seed=3):
    """Dirichlet Poisson problem on the unit disk: the RBF-FD Laplacian on
    all rows, identity rows at the boundary nodes."""
    x, y, flag = NS.unit_disk(n, nb=nb, seed=seed)
    ja = O.knn_brute(x, y, k)
    W, info = O.assemble(x, y, ja, k, P, ops=O.OP_LAPLACE)
    assert not info.any()
    bnd = np.flatnonzero(flag).astype(np.int32)
    f = lap_exact(x, y)
    f[bnd] = u_exact(x[bnd], y[bnd])
    return dict(x=x, y=y, k=k, ja=ja, L=W[0], bnd=bnd, f=f, n=n)


def as_sparse(pr):
    n, k = pr["n"], pr["k"]
    rows = np.repeat(np.arange(n), k)
    vals = pr["L"].copy()
    isb = np.zeros(n, bool)
    isb[pr["bnd"]] = True
    vals[isb[rows]] = 0.0
    A = sp.csr_matrix((vals, (rows, pr["ja"])), shape=(n, n)).tolil()
    for b in pr["bnd"]:
        A[b, b] = 1.0
    return A.tocsr()


@pytest.fixture(scope="module")
def pr():
    return poisson_disk()


@pytest.mark.parametrize("grid", [1, 7])
def test_bicgstab_matches_direct_solve(pr, grid):
    st, u, it, rel = O.bicgstab(pr["L"], pr["ja"], pr["f"], np.zeros(pr["n"]), k=pr["k"],
                                bnd=pr["bnd"], tol=1e-12, maxit=5000, grid=grid)
    assert st == 0 and 0 < it < 5000 and rel <= 1e-12
    # the recursive residual it stopped on agrees with the true one
    Au = O.spmv(pr["ja"], pr["L"], u, pr["k"], pr["bnd"])
    assert np.linalg.norm(pr["f"] - Au) <= 1e-11 * np.linalg.norm(pr["f"])
    ud = spla.spsolve(as_sparse(pr), pr["f"])
    assert np.abs(u - ud).max() <= 1e-9 * np.abs(ud).max()


def test_manufactured_solution(pr):
    st, u, it, rel = O.bicgstab(pr["L"], pr["ja"], pr["f"], np.zeros(pr["n"]), k=pr["k"],
                                bnd=pr["bnd"], tol=1e-12, maxit=5000)
    assert st == 0
    err = np.abs(u - u_exact(pr["x"], pr["y"])).max()
    assert err < 2e-3, err


def test_ragged_rows_equal_fixed_width(pr):
    n, k = pr["n"], pr["k"]
    ia = np.arange(0, (n + 1) * k, k, dtype=np.int32)
    a = O.bicgstab(pr["L"], pr["ja"], pr["f"], np.zeros(n), k=k, bnd=pr["bnd"], tol=1e-10, grid=3)
    b = O.bicgstab(pr["L"], pr["ja"], pr["f"], np.zeros(n), ia=ia, bnd=pr["bnd"], tol=1e-10, grid=3)
    assert a[0] == b[0] == 0 and a[2] == b[2] and a[3] == b[3]
    assert np.array_equal(a[1], b[1])


def test_edge_cases(pr):
    n, k, L, ja, bnd = pr["n"], pr["k"], pr["L"], pr["ja"], pr["bnd"]
    # f = 0: the solution is zero whatever the guess
    st, u, it, rel = O.bicgstab(L, ja, np.zeros(n), np.ones(n), k=k, bnd=bnd)
    assert st == 0 and it == 0 and not u.any()
    # a guess that already satisfies the tolerance: no iteration
    _, us, _, _ = O.bicgstab(L, ja, pr["f"], np.zeros(n), k=k, bnd=bnd, tol=1e-12)
    st, u, it, rel = O.bicgstab(L, ja, pr["f"], us, k=k, bnd=bnd, tol=1e-9)
    assert st == 0 and it == 0 and np.array_equal(u, us)
    # maxit runs out
    st, u, it, rel = O.bicgstab(L, ja, pr["f"], np.zeros(n), k=k, bnd=bnd, tol=1e-14, maxit=3)
    assert st == -10 and it == 3 and rel > 1e-14
    st, u, it, rel = O.bicgstab(L, ja, pr["f"], np.zeros(n), k=k, bnd=bnd, maxit=0)
    assert st == -10 and it == 0
    # a boundary index outside [0, n), or a bad argument
    with pytest.raises(ValueError):
        O.bicgstab(L, ja, pr["f"], np.zeros(n), k=k, bnd=np.array([n], np.int32))
    with pytest.raises(ValueError):
        O.bicgstab(L, ja, pr["f"], np.zeros(n), k=k, bnd=bnd, tol=-1.0)
    # empty system
    st, u, it, rel = O.bicgstab(np.zeros(0), np.zeros(0, np.int32), np.zeros(0), np.zeros(0), k=k)
    assert st == 0 and it == 0 and u.size == 0


def test_grid_and_identity_operator():
    """The reduction grid follows the CUDA launch rule; on an operator that is
    all identity (boundary) rows one iteration returns f exactly."""
    rng = np.random.default_rng(0)
    for n in (1, 255, 256, 257, 10_000, 300_001):
        for sms in (1, 148):
            assert O.solve_grid(n, sms) == max(1, min((n + 255) // 256, 6 * sms))
        f = rng.standard_normal(n)
        st, u, it, rel = O.bicgstab(np.zeros(0), np.zeros(0, np.int32), f, np.zeros(n),
                                    ia=np.zeros(n + 1, np.int32), bnd=np.arange(n, dtype=np.int32),
                                    tol=0.0, maxit=1, grid=O.solve_grid(n, 148))
        assert st == 0 and it == 1 and rel == 0.0 and np.array_equal(u, f)


@pytest.mark.parametrize("seed", range(4))
def test_random_stencil_operators(seed):
    """Random diagonally dominant operators with stencil rows (self first),
    fixed-width or ragged, some rows identity: the oracle's iterate solves
    the dense system."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(50, 400))
    ragged = seed % 2 == 1
    kv = rng.integers(3, 12, size=n) if ragged else np.full(n, 7)
    ia = np.zeros(n + 1, np.int64)
    ia[1:] = np.cumsum(kv)
    ja = np.empty(ia[-1], np.int32)
    vals = np.empty(ia[-1])
    A = np.zeros((n, n))
    for s in range(n):
        others = rng.choice(np.delete(np.arange(n), s), size=kv[s] - 1, replace=False)
        cols = np.concatenate([[s], others])
        w = rng.uniform(-1.0, 1.0, size=kv[s])
        w[0] = np.abs(w[1:]).sum() + rng.uniform(0.5, 2.0)
        ja[ia[s]:ia[s + 1]] = cols
        vals[ia[s]:ia[s + 1]] = w
        A[s, cols] = w
    bnd = np.sort(rng.choice(n, size=n // 10, replace=False)).astype(np.int32)
    A[bnd] = 0.0
    A[bnd, bnd] = 1.0
    f = rng.standard_normal(n)
    kw = dict(ia=ia.astype(np.int32)) if ragged else dict(k=7)
    st, u, it, rel = O.bicgstab(vals, ja, f, np.zeros(n), bnd=bnd, tol=1e-13, maxit=2000,
                                grid=O.solve_grid(n, 148), **kw)
    assert st == 0 and rel <= 1e-13
    ud = np.linalg.solve(A, f)
    assert np.abs(u - ud).max() <= 1e-10 * np.abs(ud).max()
