"""Every compiled kernel shape, pinned one at a time (rbfb_select_variant),
against the oracle through the C ABI.

FP64 shapes (register kernel `f64_*`, blocked shared-memory kernel `b64_*`)
perform the oracle's operations in its order: their weights must be
bit-identical to it, whatever the shape's lanes, panels or slot size. Shapes
of the refined form (`mix_*`, `bmx_*`) are held to 1e-10 relative against the
FP64 oracle at degree 2-3, and at degree 4 (cond ~1e6-1e8, many stencils
fall back to FP64) to twice the FP64 oracle's own distance from the
long-double solution, as in test_gpu_assembly.
"""
import re

import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu

TOLMIX = 1e-10


def _shapes():
    out = []
    for i, nm in enumerate(R.variant_names()):
        m = re.match(r"(f64|b64|mix|bmx)_p(\d)q(\d)_n(\d+)", nm)
        assert m, nm
        kind, P, Q, ntp = m.group(1), int(m.group(2)), int(m.group(3)), int(m.group(4))
        nrhs = 8 if "_r8" in nm else 3
        out.append((i, nm, kind in ("mix", "bmx"), P, Q, ntp, nrhs))
    return out


def _nodes(P, ntp):
    """A node set and the largest stencil size the shape takes (k + npoly(P) <= ntp)."""
    k = min(64, ntp - O.npoly(P))
    if P == 4:
        x, y, _ = NS.gaussian_bump(1500, seed=4)
    else:
        x, y, _ = NS.jittered_grid(36, 0.3, seed=9, periodic=True)
    return x, y, k


@pytest.mark.parametrize("shape", _shapes(), ids=lambda s: s[1])
def test_shape_against_oracle(ctx, torch_cuda, shape):
    T = torch_cuda
    idx, name, mixed, P, Q, ntp, nrhs = shape
    x, y, k = _nodes(P, ntp)
    period = None if P == 4 else (1.0, 1.0)
    n = x.size
    ja = O.knn_brute(x, y, k, period=period)
    if nrhs == 8:
        pts = np.linspace(-0.01, 0.01, 8)
        xc, yc = pts, pts[::-1].copy()
        ops = R.OP_INTERP
    else:
        xc = yc = None
        ops = R.DEFAULT_OPS
    xcd = None if xc is None else T.as_tensor(xc).cuda()
    ycd = None if yc is None else T.as_tensor(yc).cuda()
    d = R.make_desc(P, Q, ops, R.FP32_IR if mixed else R.FP64, True, period=period, xc=xcd,
                    yc=ycd, nc=0 if xc is None else len(xc))
    ctx.select_variant(d, k, idx)
    xd, yd = T.as_tensor(x).cuda(), T.as_tensor(y).cuda()
    jd = T.as_tensor(ja).cuda()
    m = R.num_rhs(ops, 0 if xc is None else len(xc))
    vals = [T.full((n * k,), 7.0, dtype=T.float64, device="cuda") for _ in range(m)]
    info = T.full((n,), -7, dtype=T.int32, device="cuda")
    st = ctx.assemble(d, xd, yd, k, jd, vals, info, stats=True)
    T.cuda.synchronize()
    W = np.stack([v.cpu().numpy() for v in vals])
    Wo, io = O.assemble(x, y, ja, k, P, Q, ops=ops, xc=xc, yc=yc, period=period)
    if not mixed:
        np.testing.assert_array_equal(info.cpu().numpy(), io)
        np.testing.assert_array_equal(W, Wo)
        return
    assert (info.cpu().numpy() == 0).all()
    if P < 4:
        assert O.max_rel_err(W, Wo, k).max() <= TOLMIX
        return
    Wl, _ = O.assemble_ld(x, y, ja, k, P, Q, period=period)

    def worst(a, b):
        a3, b3 = a.reshape(3, n, k), b.reshape(3, n, k)
        return (np.abs(a3 - b3).max(axis=2) / np.abs(b3).max(axis=2)).max()

    assert worst(W, Wl) <= 2.0 * worst(Wo, Wl)
    assert 0 <= st["fallback"] <= n
