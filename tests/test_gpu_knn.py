"""Parity of the uniform-grid k-NN kernel with the reference's searches.

Index-exact on tie-free clouds (seeded jittered grids) against the
reference's own nanoflann (open plane) and ckdtree (periodic) output, and
against the reference's shipped periodic graphs; on node sets with exact
distance ties (lattices, the node files read off paper figures) the
reference's own contract applies: squared distances equal position by
position, so that differing indices sit on ties (test/test_spatial.cpp:84-101).
"""
import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from conftest import golden
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu


def knn(ctx, torch, x, y, k, period=None):
    xd = torch.as_tensor(np.ascontiguousarray(x)).cuda()
    yd = torch.as_tensor(np.ascontiguousarray(y)).cuda()
    ja = torch.full((len(x) * k,), -1, dtype=torch.int32, device="cuda")
    ctx.knn_stencils(xd, yd, k, ja, period=period)
    assert ctx.knn_status() == 0
    return ja.cpu().numpy()


def same_distances(x, y, a, b, k, period=None):
    da = O.stencil_d2(x, y, a, k, period)
    db = O.stencil_d2(x, y, b, k, period)
    np.testing.assert_array_equal(da, db)


def test_seeded_open_exact_vs_nanoflann(ctx, torch_cuda):
    g = golden("square69_k21")
    ja = knn(ctx, torch_cuda, g["x"], g["y"], 21)
    np.testing.assert_array_equal(ja, g["ja_nanoflann"])


def test_seeded_periodic_exact_vs_ckdtree(ctx, torch_cuda):
    g = golden("periodic64_k35")
    ja = knn(ctx, torch_cuda, g["x"], g["y"], 35, period=(1.0, 1.0))
    np.testing.assert_array_equal(ja, g["ja_ckdtree"])


@pytest.mark.parametrize("case", ["poisson_32_21", "poisson_32_64"])
def test_reference_periodic_graphs(ctx, torch_cuda, case):
    g = golden(case)
    k = int(g["k"])
    ja = knn(ctx, torch_cuda, g["x"], g["y"], k, period=tuple(g["box"]))
    np.testing.assert_array_equal(ja, g["ja"])


def test_lattice_ties(ctx, torch_cuda):
    g = golden("cartesian_32_21")
    ja = knn(ctx, torch_cuda, g["x"], g["y"], 21, period=tuple(g["box"]))
    same_distances(g["x"], g["y"], ja, g["ja"], 21, tuple(g["box"]))
    # ties broken by index, as the oracle does
    np.testing.assert_array_equal(ja, O.knn_brute(g["x"], g["y"], 21, period=tuple(g["box"])))


@pytest.mark.parametrize("case", ["shu_square_4786", "barnett_disk_817", "wright_square_hole_892"])
def test_node_files(ctx, torch_cuda, case):
    g = golden(case)
    ja = knn(ctx, torch_cuda, g["x"], g["y"], 21)
    same_distances(g["x"], g["y"], ja, g["ja_nanoflann"], 21)
    np.testing.assert_array_equal(ja, O.knn_brute(g["x"], g["y"], 21))


def test_large_periodic_against_oracle_sample(ctx, torch_cuda):
    # 256 x 256 periodic grid, k=35: every row checked against brute force on a sample
    x, y, _ = NS.jittered_grid(256, 0.3, seed=11, periodic=True)
    ja = knn(ctx, torch_cuda, x, y, 35, period=(1.0, 1.0)).reshape(-1, 35)
    rows = np.random.default_rng(0).choice(x.size, 400, replace=False)
    ref = O.knn_brute(x, y, 35, xq=x[rows], yq=y[rows], period=(1.0, 1.0)).reshape(-1, 35)
    np.testing.assert_array_equal(ja[rows], ref)
    assert (ja[:, 0] == np.arange(x.size)).all()


def test_query_points(ctx, torch_cuda):
    x, y, _ = NS.jittered_grid(40, 0.3, seed=5)
    rng = np.random.default_rng(9)
    xq, yq = rng.uniform(-0.1, 1.1, 300), rng.uniform(-0.1, 1.1, 300)
    T = torch_cuda
    # 300 queries against 1600 nodes: the rows after the 300th (a guard region
    # as long as the node set) stay untouched
    buf = T.full((x.size * 16,), -1, dtype=T.int32, device="cuda")
    ja = buf[: 300 * 16]
    ctx.knn_query(T.as_tensor(x).cuda(), T.as_tensor(y).cuda(), T.as_tensor(xq).cuda(),
                  T.as_tensor(yq).cuda(), 16, ja)
    np.testing.assert_array_equal(ja.cpu().numpy(), O.knn_brute(x, y, 16, xq=xq, yq=yq))
    assert (buf[300 * 16:].cpu().numpy() == -1).all()


def test_edge_cases(ctx, torch_cuda):
    # k = n; all points identical (every distance ties at 0); collinear points
    x, y, _ = NS.jittered_grid(6, 0.3, seed=2)
    ja = knn(ctx, torch_cuda, x, y, x.size)
    np.testing.assert_array_equal(ja, O.knn_brute(x, y, x.size))
    x = np.full(50, 0.3)
    y = np.full(50, 0.7)
    ja = knn(ctx, torch_cuda, x, y, 10).reshape(-1, 10)
    assert (ja == np.arange(10)[None, :]).all()  # ties at distance 0 -> lowest indices
    x = np.linspace(0, 1, 200)
    y = np.zeros(200)
    ja = knn(ctx, torch_cuda, x, y, 7)
    np.testing.assert_array_equal(ja, O.knn_brute(x, y, 7))


def test_bad_arguments(ctx, torch_cuda):
    T = torch_cuda
    x = T.zeros(10, dtype=T.float64, device="cuda")
    ja = T.zeros(10 * 11, dtype=T.int32, device="cuda")
    with pytest.raises(R.RbfError):
        ctx.knn_stencils(x, x, 11, ja)  # k > n
