"""The oracle against the reference's own known answers.

* data/poisson_32_{21,64}: periodic 32 x 32 k-NN graphs shipped with the
  reference; ckdtree's order, index for index.
* data/cartesian_32_21: the same on a lattice, where exact ties exist; the
  reference's own contract applies (test/test_spatial.cpp:84-101): distances
  agree to 1e-12(1+d), indices only where the distance is distinct.
* the reference's nanoflann NodeSet::stencils(21) and ckdtree
  KdTree::knn_stencils on its node files and on seeded clouds.
* the oracle's FP64 weights on the first 200 stencils, pinned.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden


def tie_contract(x, y, ja_a, ja_b, k, period=None):
    """The reference's contract for two k-NN tables (test/test_spatial.cpp:
    84-101): rows agree in distance, and in index wherever the distance is
    not tied. With both tables' squared distances formed in the same
    arithmetic, that is: the squared distances agree position by position,
    exactly; a differing index then necessarily sits on a tie."""
    da = O.stencil_d2(x, y, ja_a, k, period).reshape(-1, k)
    db = O.stencil_d2(x, y, ja_b, k, period).reshape(-1, k)
    np.testing.assert_array_equal(da, db)
    A, B = ja_a.reshape(-1, k), ja_b.reshape(-1, k)
    for s, t in zip(*np.nonzero(A != B)):
        # the two points differ but are equidistant from node s
        assert da[s, t] == db[s, t]


@pytest.mark.parametrize("case", ["poisson_32_21", "poisson_32_64"])
def test_periodic_graph_exact(case):
    g = golden(case)
    k = int(g["k"])
    ja = O.knn_brute(g["x"], g["y"], k, period=tuple(g["box"]))
    np.testing.assert_array_equal(ja, g["ja"])


def test_lattice_graph_tie_contract():
    g = golden("cartesian_32_21")
    k = int(g["k"])
    ja = O.knn_brute(g["x"], g["y"], k, period=tuple(g["box"]))
    tie_contract(g["x"], g["y"], ja, g["ja"], k, tuple(g["box"]))
    # same neighbour sets wherever the k-th distance is not tied across the cut
    assert (ja.reshape(-1, k)[:, 0] == np.arange(1024)).all()


@pytest.mark.parametrize("case", ["shu_square_4786", "barnett_disk_817", "wright_square_hole_892"])
def test_node_files_tie_contract(case):
    g = golden(case)
    k = int(g["k"])
    ja = O.knn_brute(g["x"], g["y"], k)
    tie_contract(g["x"], g["y"], ja, g["ja_nanoflann"], k)
    tie_contract(g["x"], g["y"], ja, g["ja_ckdtree"], k)


def test_seeded_cloud_exact():
    g = golden("square69_k21")
    ja = O.knn_brute(g["x"], g["y"], 21)
    np.testing.assert_array_equal(ja, g["ja_nanoflann"])
    assert (ja.reshape(-1, 21)[:, 0] == np.arange(g["x"].size)).all()  # self first


def test_seeded_periodic_exact():
    g = golden("periodic64_k35")
    ja = O.knn_brute(g["x"], g["y"], 35, period=tuple(g["box"]))
    np.testing.assert_array_equal(ja, g["ja_ckdtree"])


def test_reference_search_live_if_built():
    if O.ref() is None:
        pytest.skip("reference search library not built here")
    g = golden("square69_k21")
    np.testing.assert_array_equal(O.ref_nodeset_stencils(g["x"], g["y"], 21), g["ja_nanoflann"])


@pytest.mark.parametrize("name,src,key", [("weights_square69", "square69_k21", "ja_nanoflann"),
                                          ("weights_shu", "shu_square_4786", "ja_nanoflann")])
def test_oracle_weights_pinned(name, src, key):
    w = golden(name)
    g = golden(src)
    k = int(w["k"])
    n = 200
    W, info = O.assemble(g["x"], g["y"], g[key], k, int(w["P"]))
    np.testing.assert_array_equal(info[:n], w["info"])
    err = O.max_rel_err(W[:, : n * k], w["w"], k)
    assert err.max() <= 1e-14, err
