"""rbfb_knn_stencils_static, the k-NN search that allocates nothing.

It is meant for callers that may not allocate device memory while running
(a solver loop past its set-up phase, a host whose device memory belongs to
another allocator). Checked here through the C ABI against the ordinary
entry point rbfb_knn_stencils: the stencils are integer indices, so the two
must agree exactly, and they must keep agreeing on a second call in a row
(the fixed scratch keeps the previous call's contents). On a tie-free
non-uniform cloud it is also checked on its own against the oracle's
brute-force search. This file is named to be collected last.
"""
import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu


def _cases():
    x, y, _ = NS.jittered_grid(69, 0.3, seed=1)                 # open plane, 4,761 nodes
    yield x, y, 21, None
    x, y, _ = NS.jittered_grid(200, 0.3, seed=8, periodic=True)  # periodic, 40,000 nodes
    yield x, y, 35, (1.0, 1.0)
    x, y, _ = NS.gaussian_bump(20000, seed=4)                   # non-uniform density
    yield x, y, 64, None


def test_static_search_matches_the_ordinary_one(torch_cuda):
    T = torch_cuda
    with R.Context(0) as ctx:
        for x, y, k, period in _cases():
            n = x.size
            xd, yd = T.as_tensor(x).cuda(), T.as_tensor(y).cuda()
            ref = T.full((n * k,), -1, dtype=T.int32, device="cuda")
            ctx.knn_stencils(xd, yd, k, ref, period=period)
            for call in range(2):  # two calls in a row on the same scratch
                ja = T.full((n * k,), -1, dtype=T.int32, device="cuda")
                R.knn_stencils_static(xd, yd, k, ja, period=period)
                assert R.knn_static_status() == 0, f"call {call}: a query gave up"
                T.cuda.synchronize()
                np.testing.assert_array_equal(ja.cpu().numpy(), ref.cpu().numpy(),
                                              err_msg=f"call {call}, n={n}, k={k}")


def test_static_search_against_the_oracle(torch_cuda):
    """Gaussian-bump density (a 4x range of spacings, so the fixed cell grid
    holds crowded and sparse cells), k = 64 and k = 21: index-exact against
    the oracle's brute force, with the completion status read back."""
    T = torch_cuda
    x, y, _ = NS.gaussian_bump(6000, seed=11)
    xd, yd = T.as_tensor(x).cuda(), T.as_tensor(y).cuda()
    for k in (64, 21):
        ja = T.full((x.size * k,), -1, dtype=T.int32, device="cuda")
        R.knn_stencils_static(xd, yd, k, ja)
        assert R.knn_static_status() == 0
        T.cuda.synchronize()
        np.testing.assert_array_equal(ja.cpu().numpy(), O.knn_brute(x, y, k), err_msg=f"k={k}")


def test_static_search_rejects_oversize(torch_cuda):
    T = torch_cuda
    n = R.STATIC_MAX_NODES + 1
    x = T.rand(n, dtype=T.float64, device="cuda")
    ja = T.empty(n * 4, dtype=T.int32, device="cuda")
    with pytest.raises(R.RbfError) as e:
        R.knn_stencils_static(x, x, 4, ja)
    assert e.value.status == R.ETOOBIG


def test_static_search_argument_codes(torch_cuda):
    """The same status codes as the ordinary entry point for the same bad
    arguments; an extreme periodic aspect ratio overflows the fixed cell grid
    (ETOOBIG). None of these cases launches a kernel."""
    T = torch_cuda
    n = 1000
    x = T.rand(n, dtype=T.float64, device="cuda")
    ja = T.empty(n * 130, dtype=T.int32, device="cuda")
    with R.Context(0) as ctx:
        for k, period in ((n + 1, None), (129, None), (0, None), (8, (1.0, 0.0))):
            with pytest.raises(R.RbfError) as e_ord:
                ctx.knn_stencils(x, x, k, ja, period=period)
            with pytest.raises(R.RbfError) as e_st:
                R.knn_stencils_static(x, x, k, ja, period=period)
            assert e_st.value.status == e_ord.value.status, (k, period)
    assert R.knn_static_status() == 0  # still the last completed search's
    m = 60000
    xm = T.rand(m, dtype=T.float64, device="cuda")
    jm = T.empty(m * 4, dtype=T.int32, device="cuda")
    with pytest.raises(R.RbfError) as e:
        R.knn_stencils_static(xm, xm, 4, jm, period=(1.0e6, 1.0e-6))
    assert e.value.status == R.ETOOBIG
