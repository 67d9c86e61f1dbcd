"""The CUDA BiCGSTAB solve on an assembled operator (rbfb_solve_bicgstab,
the step after the reference's mv_op, src/main.cpp:57-68) against the CPU
restatement: both take every sum in the same order, so the iterate, the
iteration count and the residual agree bit for bit."""
import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from rbf_b200 import nodesets as NS
from test_oracle_solve import lap_exact, poisson_disk, u_exact

pytestmark = pytest.mark.gpu


def _sms(T):
    return T.cuda.get_device_properties(0).multi_processor_count


def _dev(T, a):
    return T.as_tensor(np.ascontiguousarray(a)).cuda()


def _solve_both(ctx, T, L, ja, f, u0, k=None, ia=None, bnd=None, tol=1e-10, maxit=10000,
                stream=None):
    n = f.size
    ud = _dev(T, u0.astype(np.float64))
    args = dict(k=k, ia=None if ia is None else _dev(T, ia), bnd=None if bnd is None else _dev(T, bnd),
                tol=tol, maxit=maxit)
    if stream is not None:
        with T.cuda.stream(stream):
            g = ctx.solve_bicgstab(_dev(T, L), _dev(T, ja), _dev(T, f), ud, stream=stream, **args)
        stream.synchronize()
    else:
        g = ctx.solve_bicgstab(_dev(T, L), _dev(T, ja), _dev(T, f), ud, **args)
    o = O.bicgstab(L, ja, f, u0, k=k, ia=ia, bnd=bnd, tol=tol, maxit=maxit,
                   grid=O.solve_grid(n, _sms(T)))
    return g, ud.cpu().numpy(), o


@pytest.mark.parametrize("n,nb,use_stream", [(2000, 160, False), (2000, 160, True),
                                              (32000, 640, True)])
def test_solve_bit_identical(ctx, torch_cuda, n, nb, use_stream):
    T = torch_cuda
    pr = poisson_disk(n=n, nb=nb)
    s = T.cuda.Stream() if use_stream else None
    (st, it, rel), u, (ost, ou, oit, orel) = _solve_both(
        ctx, T, pr["L"], pr["ja"], pr["f"], np.zeros(n), k=pr["k"], bnd=pr["bnd"], tol=1e-12,
        maxit=20000, stream=s)
    assert st == R.OK and ost == 0
    assert it == oit and rel == orel
    np.testing.assert_array_equal(u, ou)
    assert np.abs(u - u_exact(pr["x"], pr["y"])).max() < 2e-3


def test_solve_unaligned_operator_arrays(ctx, torch_cuda):
    """Weights and columns that start off a 16-byte boundary: the operator
    passes then walk the rows with scalar loads instead of staging them with
    16-byte copies. The iterate is the same, bit for bit."""
    T = torch_cuda
    pr = poisson_disk(n=2000, nb=160)
    L, ja, f, n = pr["L"], pr["ja"], pr["f"], pr["n"]
    Lb = T.empty(L.size + 1, dtype=T.float64, device="cuda")
    jb = T.empty(ja.size + 1, dtype=T.int32, device="cuda")
    Ld, jd = Lb[1:], jb[1:]  # 8 and 4 bytes past the allocation's start
    assert Ld.data_ptr() % 16 and jd.data_ptr() % 16
    Ld.copy_(T.as_tensor(L))
    jd.copy_(T.as_tensor(ja))
    ud = T.zeros(n, dtype=T.float64, device="cuda")
    st, it, rel = ctx.solve_bicgstab(Ld, jd, _dev(T, f), ud, k=pr["k"], bnd=_dev(T, pr["bnd"]),
                                     tol=1e-12, maxit=20000)
    ost, ou, oit, orel = O.bicgstab(L, ja, f, np.zeros(n), k=pr["k"], bnd=pr["bnd"], tol=1e-12,
                                    maxit=20000, grid=O.solve_grid(n, _sms(T)))
    assert st == R.OK and ost == 0
    assert it == oit and rel == orel
    np.testing.assert_array_equal(ud.cpu().numpy(), ou)


def test_solve_graph_replay_and_launches(ctx, torch_cuda):
    # a non-default stream captures one chunk of 8 iterations (5 kernels
    # each) once and replays it
    T = torch_cuda
    pr = poisson_disk()
    s = T.cuda.Stream()
    res, launches = [], []
    for _ in range(3):
        l0 = ctx.launches()
        g, u, o = _solve_both(ctx, T, pr["L"], pr["ja"], pr["f"], np.zeros(pr["n"]), k=pr["k"],
                              bnd=pr["bnd"], tol=1e-11, stream=s)
        launches.append(ctx.launches() - l0)
        res.append((g, u))
    it = res[0][0][1]
    chunks = -(-it // 8)
    assert launches[0] == launches[1] == launches[2] == 2 + 40 * chunks
    for g, u in res[1:]:
        assert g == res[0][0]
        np.testing.assert_array_equal(u, res[0][1])


def test_solve_ragged_csr(ctx, torch_cuda):
    # the uneven disk batch: ragged CSR rows assembled on the device, then solved
    T = torch_cuda
    c = NS.config_disk_uneven(n=3000, nb=120, seed=17)
    x, y, kvec, deg, flag = c["x"], c["y"], c["kvec"], c["degree"], c["flag"]
    n = x.size
    kmax = int(kvec.max())
    jaf = O.knn_brute(x, y, kmax).reshape(n, kmax)
    ia = np.zeros(n + 1, np.int32)
    ia[1:] = np.cumsum(kvec)
    ja = np.concatenate([jaf[s, : kvec[s]] for s in range(n)]).astype(np.int32)
    vals = [T.empty(int(ia[-1]), dtype=T.float64, device="cuda")]
    ctx.assemble_csr(R.make_desc(2, ops=R.OP_LAPLACE), _dev(T, x), _dev(T, y), _dev(T, ia),
                     _dev(T, ja), vals, degree=_dev(T, deg))
    L = vals[0].cpu().numpy()
    bnd = np.flatnonzero(flag).astype(np.int32)
    f = lap_exact(x, y)
    f[bnd] = u_exact(x[bnd], y[bnd])
    (st, it, rel), u, (ost, ou, oit, orel) = _solve_both(ctx, T, L, ja, f, np.zeros(n), ia=ia,
                                                         bnd=bnd, tol=1e-12)
    assert st == R.OK and ost == 0 and it == oit and rel == orel
    np.testing.assert_array_equal(u, ou)
    assert np.abs(u - u_exact(x, y)).max() < 1e-3


def test_solve_edge_cases(ctx, torch_cuda):
    T = torch_cuda
    pr = poisson_disk()
    n, k, L, ja, bnd, f = pr["n"], pr["k"], pr["L"], pr["ja"], pr["bnd"], pr["f"]
    # f = 0: u is set to zero
    (st, it, rel), u, _ = _solve_both(ctx, T, L, ja, np.zeros(n), np.ones(n), k=k, bnd=bnd)
    assert st == R.OK and it == 0 and not u.any()
    # maxit runs out: the same iterate as the restatement after 3 steps
    (st, it, rel), u, (ost, ou, oit, orel) = _solve_both(ctx, T, L, ja, f, np.zeros(n), k=k,
                                                         bnd=bnd, tol=1e-14, maxit=3)
    assert st == R.ENOCONV and ost == -10 and it == oit == 3 and rel == orel
    np.testing.assert_array_equal(u, ou)
    # a guess that already meets the tolerance takes no iteration and is
    # returned unchanged
    _, us, _, _ = O.bicgstab(L, ja, f, np.zeros(n), k=k, bnd=bnd, tol=1e-12)
    (st, it, rel), u, _ = _solve_both(ctx, T, L, ja, f, us, k=k, bnd=bnd, tol=1e-9)
    assert st == R.OK and it == 0
    np.testing.assert_array_equal(u, us)
    # an out-of-range boundary index is an argument error and leaves u alone
    ud = _dev(T, np.full(n, 7.0))
    with pytest.raises(R.RbfError):
        ctx.solve_bicgstab(_dev(T, L), _dev(T, ja), _dev(T, f), ud, k=k,
                           bnd=_dev(T, np.array([0, n], np.int32)))
    assert (ud.cpu().numpy() == 7.0).all()
    # an empty system
    e = T.empty(0, dtype=T.float64, device="cuda")
    assert ctx.solve_bicgstab(e, T.empty(0, dtype=T.int32, device="cuda"), e, e, k=k) == (R.OK, 0, 0.0)
