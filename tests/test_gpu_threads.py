"""Host threads. The C ABI's unit of thread safety is the context: one per
host thread (the reference's NodeSet / KdTree are const-thread-safe,
src/rbf_spatial.h:129-131). Two threads, each with its own context and CUDA
stream, search and assemble different node sets at the same time, several
times over, in both forms; every result equals the same calls made alone on
the main thread, bit for bit (the FP64 weights also equal the oracle's)."""
import threading

import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu

K = 35
REPS = 4


def _case(i):
    """Node set i: a periodic grid and an open one of other sizes."""
    if i == 0:
        x, y, _ = NS.jittered_grid(96, 0.3, seed=21, periodic=True)
        return x, y, (1.0, 1.0)
    x, y, _ = NS.jittered_grid(80, 0.3, seed=22, periodic=False)
    return x, y, None


def _run(T, ctx, x, y, period, precision, stream):
    """k-NN stencils and the weights of node set (x, y) on `stream`."""
    n = x.size
    with T.cuda.stream(stream):
        xd, yd = T.as_tensor(x).cuda(), T.as_tensor(y).cuda()
        ja = T.empty(n * K, dtype=T.int32, device="cuda")
        vals = [T.empty(n * K, dtype=T.float64, device="cuda") for _ in range(3)]
        info = T.full((n,), -1, dtype=T.int32, device="cuda")
    ctx.knn_stencils(xd, yd, K, ja, period=period, stream=stream)
    d = R.make_desc(3, 5, R.DEFAULT_OPS, precision, True, period=period)
    ctx.assemble(d, xd, yd, K, ja, vals, info, stream=stream)
    stream.synchronize()
    return (ja.cpu().numpy(), np.stack([v.cpu().numpy() for v in vals]), info.cpu().numpy())


@pytest.mark.parametrize("precision", [R.FP64, R.FP32_IR], ids=["fp64", "mixed"])
def test_two_threads_two_contexts(torch_cuda, precision):
    T = torch_cuda
    cases = [_case(0), _case(1)]
    alone = []
    with R.Context(0) as c:
        s = T.cuda.Stream()
        for x, y, per in cases:
            alone.append(_run(T, c, x, y, per, precision, s))
    if precision == R.FP64:
        for (x, y, per), (ja, W, info) in zip(cases, alone):
            Wo, io = O.assemble(x, y, ja, K, 3, 5, period=per)
            np.testing.assert_array_equal(W, Wo)
            np.testing.assert_array_equal(info, io)

    results = [[], []]
    errors = []
    start = threading.Barrier(2)

    def work(i):
        try:
            x, y, per = cases[i]
            with R.Context(0) as c:
                s = T.cuda.Stream()
                start.wait(timeout=60)
                for _ in range(REPS):
                    results[i].append(_run(T, c, x, y, per, precision, s))
        except Exception as e:  # reported on the main thread
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not any(t.is_alive() for t in threads), "a worker thread did not finish"
    assert not errors, errors
    for i in range(2):
        assert len(results[i]) == REPS
        for ja, W, info in results[i]:
            np.testing.assert_array_equal(ja, alone[i][0])
            np.testing.assert_array_equal(W, alone[i][1])
            np.testing.assert_array_equal(info, alone[i][2])
