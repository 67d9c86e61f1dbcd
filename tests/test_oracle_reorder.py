"""The renumbering oracle (curve keys, curve order, boundary-last partition,
stencil renumbering) against the known answers of the reference's own
tests (test/test_reorder.cpp) and against independent restatements."""
import numpy as np

import oracle as O


def grid4():
    """4 x 4 cell centres in [0, 4]^2, row-major (test_reorder.cpp:61-70)."""
    j, i = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    return (i.ravel() + 0.5).astype(np.float64), (j.ravel() + 0.5).astype(np.float64)


def interleave(ix, iy, ndiv):
    """The reference test's Morton key: x bits in the even positions
    (test_reorder.cpp:21-28)."""
    z = 0
    for b in range(ndiv - 1, -1, -1):
        z = (z << 2) | (((iy >> b) & 1) << 1) | ((ix >> b) & 1)
    return z


def test_morton_keys_known_answer():
    # test_reorder.cpp:72-80
    x, y = grid4()
    keys = O.curve_keys(x, y, 2, O.MORTON, bbox=(0, 0, 4, 4))
    for j in range(4):
        for i in range(4):
            assert keys[j * 4 + i] == interleave(i, j, 2)


def test_hilbert_keys_known_answer():
    # test_reorder.cpp:82-102: keys are 0..15 and consecutive keys are grid neighbours
    x, y = grid4()
    keys = O.curve_keys(x, y, 2, O.HILBERT, bbox=(0, 0, 4, 4))
    assert sorted(keys.tolist()) == list(range(16))
    cell_of_key = np.empty(16, np.int64)
    cell_of_key[keys] = np.arange(16)
    for k in range(1, 16):
        a, b = cell_of_key[k - 1], cell_of_key[k]
        assert abs(a % 4 - b % 4) + abs(a // 4 - b // 4) == 1


def test_hilbert_is_a_curve_at_depth():
    # deeper levels: still a permutation of 0..4^ndiv - 1 with unit steps
    nd = 5
    m = 1 << nd
    j, i = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    x, y = (i.ravel() + 0.5), (j.ravel() + 0.5)
    keys = O.curve_keys(x, y, nd, O.HILBERT, bbox=(0, 0, m, m))
    assert sorted(keys.tolist()) == list(range(m * m))
    cell = np.empty(m * m, np.int64)
    cell[keys] = np.arange(m * m)
    steps = np.abs(np.diff(cell % m)) + np.abs(np.diff(cell // m))
    assert (steps == 1).all()


def test_morton_keys_match_cell_interleave():
    # random points: the bisection keys equal the interleaved cell indices
    # whenever no point sits within rounding of a cell boundary
    rng = np.random.default_rng(3)
    x = rng.uniform(0.0, 1.0, 5000)
    y = rng.uniform(0.0, 1.0, 5000)
    nd = 10
    keys = O.curve_keys(x, y, nd, O.MORTON, bbox=(0.0, 0.0, 1.0, 1.0))
    ix = np.minimum((x * (1 << nd)).astype(np.int64), (1 << nd) - 1)
    iy = np.minimum((y * (1 << nd)).astype(np.int64), (1 << nd) - 1)
    # points exactly on a boundary go to the lower cell in the reference (px > cx)
    on_edge = (x * (1 << nd) == np.floor(x * (1 << nd))) | (y * (1 << nd) == np.floor(y * (1 << nd)))
    for t in np.flatnonzero(~on_edge)[:2000]:
        assert keys[t] == interleave(int(ix[t]), int(iy[t]), nd)


def test_curve_order_is_a_stable_sort():
    rng = np.random.default_rng(4)
    x = rng.uniform(-2.0, 3.0, 4000)
    y = rng.uniform(1.0, 1.5, 4000)
    for curve in (O.MORTON, O.HILBERT):
        for nd in (3, 16):  # nd = 3: many equal keys, the stable order decides
            keys = O.curve_keys(x, y, nd, curve)
            perm = O.curve_order(x, y, nd, curve)
            np.testing.assert_array_equal(perm, np.argsort(keys, kind="stable"))


def test_boundary_last_known_answer():
    # test_reorder.cpp:104-117
    flag = np.array([0, 1, 0, 1, 0, 0, 2], np.int32)
    np.testing.assert_array_equal(O.boundary_last(flag), [0, 2, 4, 5, 1, 3, 6])


def test_renumber_stencils_known_answer():
    # test_reorder.cpp:119-139: 4 nodes, k = 2, ring graph, p = {2, 0, 3, 1}
    ja = np.array([0, 1, 1, 2, 2, 3, 3, 0], np.int32)
    p = np.array([2, 0, 3, 1], np.int32)
    inv = np.empty(4, np.int32)
    inv[p] = np.arange(4)
    out = O.renumber_stencils(ja, 2, p)
    for s in range(4):
        assert out[2 * s] == s
        assert out[2 * s + 1] == inv[(p[s] + 1) % 4]
    ia = np.arange(0, 10, 2, dtype=np.int32)
    ia2, ja2 = O.renumber_csr(ia, ja, p)
    np.testing.assert_array_equal(ja2, out)
    np.testing.assert_array_equal(ia2, [0, 2, 4, 6, 8])


def test_nodeset_chain():
    # test_reorder.cpp:141-186: Morton order, then boundary last; the chained
    # permutation maps every node back to file order
    x, y = grid4()
    flag = np.array([(i in (0, 3) or j in (0, 3)) for j in range(4) for i in range(4)], np.int32)
    p1 = O.curve_order(x, y, 2, O.MORTON, bbox=(0, 0, 4, 4))
    x1, y1, f1 = x[p1], y[p1], flag[p1]
    p2 = O.boundary_last(f1)
    fo = p1[p2]  # file order of the final numbering ("p1, then p2")
    assert (f1[p2][:4] == 0).all() and (f1[p2][4:] != 0).all()
    np.testing.assert_array_equal(x[fo], x1[p2])
    np.testing.assert_array_equal(y[fo], y1[p2])
