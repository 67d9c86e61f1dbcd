"""Device renumbering through the C ABI against the oracle: curve keys and
orders bit-exact, the boundary-last partition and the stencil / CSR
renumbering exact, and the assembly of a renumbered node set equal to the
renumbered assembly of the original."""
import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu


def dev(T, a):
    return T.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("curve", [R.MORTON, R.HILBERT])
def test_curve_keys_and_order_match_oracle(ctx, torch_cuda, curve):
    T = torch_cuda
    rng = np.random.default_rng(11)
    n = 300_000
    x = rng.uniform(-1.0, 3.0, n)
    y = rng.uniform(0.5, 1.25, n)
    xd, yd = dev(T, x), dev(T, y)
    for nd, bbox in ((16, None), (31, None), (4, (-1.0, 0.0, 3.0, 2.0))):
        keys = T.empty(n, dtype=T.int64, device="cuda")
        ctx.curve_keys(xd, yd, keys, ndiv=nd, curve=curve, bbox=bbox)
        ko = O.curve_keys(x, y, nd, curve, bbox=bbox)
        np.testing.assert_array_equal(keys.cpu().numpy(), ko)
        perm = T.empty(n, dtype=T.int32, device="cuda")
        inv = T.empty(n, dtype=T.int32, device="cuda")
        sk = T.empty(n, dtype=T.int64, device="cuda")
        ctx.curve_order(xd, yd, perm, inv=inv, keys=sk, ndiv=nd, curve=curve, bbox=bbox)
        po = O.curve_order(x, y, nd, curve, bbox=bbox)  # stable: ties keep node order
        np.testing.assert_array_equal(perm.cpu().numpy(), po)
        np.testing.assert_array_equal(sk.cpu().numpy(), ko[po])
        iv = inv.cpu().numpy()
        np.testing.assert_array_equal(iv[po], np.arange(n))


def test_reference_known_answers_on_device(ctx, torch_cuda):
    T = torch_cuda
    j, i = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    x, y = i.ravel() + 0.5, j.ravel() + 0.5
    keys = T.empty(16, dtype=T.int64, device="cuda")
    ctx.curve_keys(dev(T, x), dev(T, y), keys, ndiv=2, curve=R.MORTON, bbox=(0, 0, 4, 4))
    expect = [(((jj >> 1) & 1) << 3) | (((ii >> 1) & 1) << 2) | ((jj & 1) << 1) | (ii & 1)
              for jj in range(4) for ii in range(4)]
    assert keys.cpu().tolist() == expect
    flag = dev(T, np.array([0, 1, 0, 1, 0, 0, 2], np.int32))
    perm = T.empty(7, dtype=T.int32, device="cuda")
    ctx.boundary_last(flag, perm)
    assert perm.cpu().tolist() == [0, 2, 4, 5, 1, 3, 6]


def test_boundary_last_and_permute(ctx, torch_cuda):
    T = torch_cuda
    c = NS.config_disk_uneven(n=200_000, nb=4096, seed=7)
    flag = c["flag"].astype(np.int32)
    rng = np.random.default_rng(2)
    flag = flag[rng.permutation(flag.size)]  # boundary spread through the numbering
    perm = T.empty(flag.size, dtype=T.int32, device="cuda")
    inv = T.empty(flag.size, dtype=T.int32, device="cuda")
    ctx.boundary_last(dev(T, flag), perm, inv)
    po = O.boundary_last(flag)
    np.testing.assert_array_equal(perm.cpu().numpy(), po)
    np.testing.assert_array_equal(inv.cpu().numpy()[po], np.arange(flag.size))
    xd = dev(T, c["x"])
    out = T.empty_like(xd)
    R.permute(perm, xd, out)
    np.testing.assert_array_equal(out.cpu().numpy(), c["x"][po])
    fo = T.empty_like(perm)
    R.permute(perm, dev(T, flag), fo)
    np.testing.assert_array_equal(fo.cpu().numpy(), flag[po])


def test_renumber_stencils_and_csr(ctx, torch_cuda):
    T = torch_cuda
    x, y, _ = NS.jittered_grid(200, 0.3, seed=5)
    n, k = x.size, 21
    ja = T.empty(n * k, dtype=T.int32, device="cuda")
    xd, yd = dev(T, x), dev(T, y)
    ctx.knn_stencils(xd, yd, k, ja)
    perm = T.empty(n, dtype=T.int32, device="cuda")
    inv = T.empty(n, dtype=T.int32, device="cuda")
    ctx.curve_order(xd, yd, perm, inv=inv, curve=R.HILBERT)
    out = T.empty_like(ja)
    R.renumber_stencils(n, k, ja, perm, inv, out)
    ja_h, p_h = ja.cpu().numpy(), perm.cpu().numpy()
    o = out.cpu().numpy()
    np.testing.assert_array_equal(o, O.renumber_stencils(ja_h, k, p_h))
    assert (o.reshape(n, k)[:, 0] == np.arange(n)).all()  # self first survives
    # ragged rows: keep a varying prefix of each row
    kv = np.random.default_rng(1).integers(5, k + 1, size=n).astype(np.int32)
    ia = np.zeros(n + 1, np.int32)
    ia[1:] = np.cumsum(kv)
    jr = np.concatenate([ja_h[s * k: s * k + kv[s]] for s in range(n)]).astype(np.int32)
    ia_o = T.empty(n + 1, dtype=T.int32, device="cuda")
    ja_o = T.empty(jr.size, dtype=T.int32, device="cuda")
    ctx.renumber_csr(dev(T, ia), dev(T, jr), perm, inv, ia_o, ja_o)
    ia_ref, ja_ref = O.renumber_csr(ia, jr, p_h)
    np.testing.assert_array_equal(ia_o.cpu().numpy(), ia_ref)
    np.testing.assert_array_equal(ja_o.cpu().numpy(), ja_ref)


def test_renumbered_assembly_is_the_renumbered_operator(ctx, torch_cuda):
    # A' = P A P^T: stencils and weights of the Morton-renumbered node set
    # equal the original ones moved to the new rows and relabelled
    T = torch_cuda
    rng = np.random.default_rng(9)
    n, k = 60_000, 21
    x = rng.uniform(0.0, 1.0, n)
    y = rng.uniform(0.0, 1.0, n)
    xd, yd = dev(T, x), dev(T, y)
    ja = T.empty(n * k, dtype=T.int32, device="cuda")
    ctx.knn_stencils(xd, yd, k, ja)
    d = R.make_desc(2, precision=R.FP64)
    W = [T.empty(n * k, dtype=T.float64, device="cuda") for _ in range(3)]
    ctx.assemble(d, xd, yd, k, ja, W)
    perm = T.empty(n, dtype=T.int32, device="cuda")
    inv = T.empty(n, dtype=T.int32, device="cuda")
    ctx.curve_order(xd, yd, perm, inv=inv)
    x2, y2 = T.empty_like(xd), T.empty_like(yd)
    R.permute(perm, xd, x2)
    R.permute(perm, yd, y2)
    ja2 = T.empty_like(ja)
    ctx.knn_stencils(x2, y2, k, ja2)
    W2 = [T.empty_like(w) for w in W]
    ctx.assemble(d, x2, y2, k, ja2, W2)
    T.cuda.synchronize()
    p = perm.cpu().numpy()
    np.testing.assert_array_equal(ja2.cpu().numpy(), O.renumber_stencils(ja.cpu().numpy(), k, p))
    for a, b in zip(W, W2):
        np.testing.assert_array_equal(b.cpu().numpy().reshape(n, k), a.cpu().numpy().reshape(n, k)[p])


def test_edge_cases_and_errors(ctx, torch_cuda):
    T = torch_cuda
    e = T.empty(0, dtype=T.float64, device="cuda")
    ctx.curve_order(e, e, T.empty(0, dtype=T.int32, device="cuda"))
    one = T.ones(1, dtype=T.float64, device="cuda")
    p1 = T.empty(1, dtype=T.int32, device="cuda")
    ctx.curve_order(one, one, p1)  # a single node: its box is a point
    assert p1.item() == 0
    with pytest.raises(R.RbfError):
        ctx.curve_keys(one, one, T.empty(1, dtype=T.int64, device="cuda"), ndiv=32)
    with pytest.raises(R.RbfError):
        ctx.curve_keys(one, one, T.empty(1, dtype=T.int64, device="cuda"), curve=2)
    with pytest.raises(R.RbfError):
        R.renumber_stencils(1, 1, p1, p1, p1, p1)  # in place is refused
