"""Parity of the CUDA assembly (through the C ABI) with the CPU oracle.

Tolerances: the FP64 kernel performs the oracle's operations in the oracle's
order, so its weights are expected bit-identical; the test allows 1e-12
relative (per stencil and operator, infinity norm), the north-star bound.
FP32 factorisation + FP64 refinement: <= 1e-10 relative.
"""
import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from conftest import golden
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOLMIX = 1e-10


def dev(torch, a, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def run(ctx, torch, x, y, ja, k, P, precision, ops=R.DEFAULT_OPS, period=None, scale=True,
        xc=None, yc=None):
    n = len(x)
    nrhs = R.num_rhs(ops, 0 if xc is None else len(xc))
    xd, yd = dev(torch, x), dev(torch, y)
    jd = dev(torch, ja, torch.int32)
    vals = [torch.empty(n * k, dtype=torch.float64, device="cuda") for _ in range(nrhs)]
    info = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    xcd = None if xc is None else dev(torch, xc)
    ycd = None if yc is None else dev(torch, yc)
    d = R.make_desc(P, 0, ops, precision, scale, period=period, xc=xcd, yc=ycd,
                    nc=0 if xc is None else len(xc))
    st = ctx.assemble(d, xd, yd, k, jd, vals, info, stats=True)
    torch.cuda.synchronize()
    W = np.stack([v.cpu().numpy() for v in vals])
    return W, info.cpu().numpy(), st


@pytest.mark.parametrize("src,key", [("square69_k21", "ja_nanoflann"), ("shu_square_4786", "ja_nanoflann")])
def test_fp64_matches_oracle(ctx, torch_cuda, src, key):
    g = golden(src)
    W, info, st = run(ctx, torch_cuda, g["x"], g["y"], g[key], 21, 2, R.FP64)
    Wo, io = O.assemble(g["x"], g["y"], g[key], 21, 2)
    np.testing.assert_array_equal(info, io)
    err = O.max_rel_err(W, Wo, 21)
    assert err.max() <= TOL64, err
    assert st["singular"] == 0 and st["stencils"] == g["x"].size


def test_fp64_bit_identical_to_oracle(ctx, torch_cuda):
    g = golden("square69_k21")
    W, info, _ = run(ctx, torch_cuda, g["x"], g["y"], g["ja_nanoflann"], 21, 2, R.FP64)
    Wo, _ = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2)
    # same operations, same order: bit-identical
    np.testing.assert_array_equal(W, Wo)


@pytest.mark.parametrize("src,key", [("square69_k21", "ja_nanoflann"), ("shu_square_4786", "ja_nanoflann")])
def test_mixed_matches_oracle(ctx, torch_cuda, src, key):
    g = golden(src)
    W, info, st = run(ctx, torch_cuda, g["x"], g["y"], g[key], 21, 2, R.FP32_IR)
    Wo, _ = O.assemble(g["x"], g["y"], g[key], 21, 2)
    assert (info == 0).all()
    err = O.max_rel_err(W, Wo, 21)
    assert err.max() <= TOLMIX, err
    assert st["max_sweeps_used"] >= 1


def test_periodic_k35_fp64_and_mixed(ctx, torch_cuda):
    g = golden("periodic64_k35")
    Wo, io = O.assemble(g["x"], g["y"], g["ja_ckdtree"], 35, 3, period=(1.0, 1.0))
    for prec, tol in ((R.FP64, TOL64), (R.FP32_IR, TOLMIX)):
        W, info, st = run(ctx, torch_cuda, g["x"], g["y"], g["ja_ckdtree"], 35, 3, prec,
                          period=(1.0, 1.0))
        np.testing.assert_array_equal(info, io)
        err = O.max_rel_err(W, Wo, 35)
        assert err.max() <= tol, (prec, err, st)


def test_unscaled_fp64(ctx, torch_cuda):
    g = golden("square69_k21")
    W, info, _ = run(ctx, torch_cuda, g["x"], g["y"], g["ja_nanoflann"], 21, 2, R.FP64, scale=False)
    Wo, _ = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2, scale=False)
    assert O.max_rel_err(W, Wo, 21).max() <= TOL64


def test_second_derivative_and_interp_ops(ctx, torch_cuda):
    g = golden("square69_k21")
    ops = R.OP_LAPLACE | R.OP_DXX | R.OP_DYY
    W, info, _ = run(ctx, torch_cuda, g["x"], g["y"], g["ja_nanoflann"], 21, 2, R.FP64, ops=ops)
    Wo, _ = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2, ops=ops)
    assert O.max_rel_err(W, Wo, 21).max() <= TOL64
    xc = np.array([0.25, -0.1]) / 69
    yc = np.array([0.1, 0.3]) / 69
    ops = R.OP_INTERP | R.OP_DX
    W, info, _ = run(ctx, torch_cuda, g["x"], g["y"], g["ja_nanoflann"], 21, 2, R.FP64, ops=ops,
                     xc=xc, yc=yc)
    Wo, _ = O.assemble(g["x"], g["y"], g["ja_nanoflann"], 21, 2, ops=ops, xc=xc, yc=yc)
    assert W.shape[0] == 3
    assert O.max_rel_err(W, Wo, 21).max() <= TOL64


def test_singular_stencils_flagged(ctx, torch_cuda):
    c = NS.config_small()
    ja = golden("square69_k21")["ja_nanoflann"].copy().reshape(-1, 21)
    ja[7, 5] = ja[7, 4]
    ja[300, 9] = ja[300, 2]
    for prec in (R.FP64, R.FP32_IR):
        W, info, st = run(ctx, torch_cuda, c["x"], c["y"], ja.ravel(), 21, 2, prec)
        assert info[7] != 0 and info[300] != 0
        assert (np.delete(info, [7, 300]) == 0).all()
        assert np.isnan(W[:, 7 * 21:8 * 21]).all()
        assert st["singular"] == 2


def test_empty_and_single_stencil(ctx, torch_cuda):
    g = golden("square69_k21")
    x, y, ja = g["x"], g["y"], g["ja_nanoflann"]
    d = R.make_desc(2)
    xd, yd, jd = dev(torch_cuda, x), dev(torch_cuda, y), dev(torch_cuda, ja, torch_cuda.int32)
    vals = [torch_cuda.zeros(21, dtype=torch_cuda.float64, device="cuda") for _ in range(3)]
    # zero stencils: nothing written, no error
    assert R.lib().rbfb_assemble(ctx.h, d, 0, xd.data_ptr(), yd.data_ptr(), 21, jd.data_ptr(),
                                 (R.C.c_void_p * 3)(*[v.data_ptr() for v in vals]), None, None,
                                 None) == 0
    torch_cuda.cuda.synchronize()
    assert all(float(v.abs().sum()) == 0.0 for v in vals)


def test_unsupported_shape_is_an_error(ctx, torch_cuda):
    g = golden("square69_k21")
    with pytest.raises(R.RbfError) as e:
        run(ctx, torch_cuda, g["x"], g["y"], g["ja_nanoflann"], 21, 1, R.FP64)  # P=1 not compiled
    assert e.value.status == R.EUNSUPPORTED


@pytest.mark.parametrize("k", [49, 64])
def test_degree4_large_stencils(ctx, torch_cuda, k):
    # shared-memory elimination shapes: r^7 + degree 4, n = k + 15 <= 79
    x, y, _ = NS.gaussian_bump(6000, seed=4)
    ja = O.knn_brute(x, y, k)
    Wo, io = O.assemble(x, y, ja, k, 4)
    W, info, st = run(ctx, torch_cuda, x, y, ja, k, 4, R.FP64)
    np.testing.assert_array_equal(info, io)
    assert O.max_rel_err(W, Wo, k).max() <= TOL64
    # the blocked shared-memory elimination performs the oracle's operations
    # in the oracle's order: bit-identical
    np.testing.assert_array_equal(W, Wo)
    # FP32 factorisation at cond ~ 1e6..1e8: refinement contracts slowly or not
    # at all; such stencils go to the FP64 kernel and are counted. At this
    # conditioning the FP64 oracle is itself ~1e-9..1e-8 away from the exact
    # weights (measured against an x87 long double solve), so the refined
    # result is held to that: its worst and 99th-percentile distance from the
    # long double weights at most twice those of the FP64 weights.
    W, info, st = run(ctx, torch_cuda, x, y, ja, k, 4, R.FP32_IR)
    assert (info == 0).all()
    assert 0 <= st["fallback"] <= x.size
    Wl, _ = O.assemble_ld(x, y, ja, k, 4)
    n = x.size

    def per_stencil(a, b):
        a3, b3 = a.reshape(3, n, k), b.reshape(3, n, k)
        return (np.abs(a3 - b3).max(axis=2) / np.abs(b3).max(axis=2)).max(axis=0)

    e64 = per_stencil(Wo, Wl)
    emix = per_stencil(W, Wl)
    assert emix.max() <= 2.0 * e64.max(), (emix.max(), e64.max())
    assert np.percentile(emix, 99) <= 2.0 * np.percentile(e64, 99) + 1e-12
