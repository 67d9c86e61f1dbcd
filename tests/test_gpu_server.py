"""Continuous-batching server: results are the same alone and in the mix,
requests beyond the HBM budget are refused, waits are bounded."""
import time

import numpy as np
import pytest

import rbf_b200 as R
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu


def requests():
    out = []
    for i, (m, k, P, geo) in enumerate([(40, 21, 2, "square"), (70, 35, 3, "square"),
                                        (55, 21, 2, "disk"), (90, 35, 3, "square"),
                                        (30, 21, 2, "disk"), (60, 35, 3, "disk")]):
        req = dict(n=m * m, geometry=geo, k=k, P=P, Q=2 * P - 1, seed=100 + i)
        x, y = NS.request_nodes(req)
        out.append((x, y, k, P))
    return out


def run_alone(x, y, k, P, prec):
    """The same request through a fresh context, nothing else on the device."""
    n = x.size
    d = R.make_desc(P, precision=prec)
    vals = [np.empty(n * k) for _ in range(3)]
    ja = np.empty(n * k, np.int32)
    with R.Context(0) as c:
        c.assemble_host(d, x, y, k, vals, ja_out_h=ja)
    return ja, vals


def test_same_alone_and_in_the_mix(torch_cuda):
    reqs = requests()
    for prec in (R.FP64, R.FP32_IR):
        srv = R.Server(0, hbm_budget=2 << 30, max_slots=4)
        try:
            tickets = [srv.submit(x, y, k, R.make_desc(P, precision=prec)) for x, y, k, P in reqs]
            for t, (x, y, k, P) in zip(tickets, reqs):
                st, res = srv.poll(t, wait_ms=60000)
                assert st == 0 and res.status == 0 and res.singular == 0
                vals, ja = srv.fetch(t, x.size, k, 3, with_ja=True)
                ja1, vals1 = run_alone(x, y, k, P, prec)
                np.testing.assert_array_equal(ja, ja1)
                for a, b in zip(vals, vals1):
                    np.testing.assert_array_equal(a, b)  # bit-identical
                assert res.end_ms >= res.start_ms >= res.submit_ms
                assert srv.release(t) == 0
            assert srv.resident_bytes() == 0
        finally:
            srv.close()


def test_budget_and_bounded_waits(torch_cuda):
    srv = R.Server(0, hbm_budget=1 << 20, max_slots=2)  # 1 MiB
    try:
        x, y, _ = NS.jittered_grid(200, 0.3, seed=1)
        with pytest.raises(R.RbfError) as e:
            srv.submit(x, y, 21, R.make_desc(2))
        assert e.value.status == R.EBUDGET
        x, y, _ = NS.jittered_grid(20, 0.3, seed=1)
        t = srv.submit(x, y, 21, R.make_desc(2))
        st, _ = srv.poll(t, wait_ms=30000)
        assert st == 0
        assert srv.poll(t + 999, wait_ms=0)[0] == R.ENOTFOUND
        assert srv.release(t) == 0
    finally:
        srv.close()


def test_requests_overlap_on_the_device(torch_cuda):
    """Continuous batching: requests submitted together run in different
    slots at the same time, so on the device clock (events around each
    request's kernels) some request's work starts before another's ends.
    The server is warmed up first (first launches load the kernels), and
    each request carries about 10 ms of device work, well above the host
    time the worker spends enqueueing one. Each result still equals the one
    computed alone (bit for bit)."""
    reqs = []
    for i in range(4):
        req = dict(n=700 * 700, geometry="square", k=35, P=3, Q=5, seed=300 + i)
        x, y = NS.request_nodes(req)
        reqs.append((x, y, 35, 3))
    srv = R.Server(0, hbm_budget=8 << 30, max_slots=4)
    try:
        xw, yw = NS.request_nodes(dict(n=20000, geometry="square", k=35, P=3, Q=5, seed=299))
        tw = [srv.submit(xw, yw, 35, R.make_desc(3)) for _ in range(4)]
        for t in tw:
            assert srv.poll(t, wait_ms=60000)[0] == 0
            assert srv.release(t) == 0
        tickets = [srv.submit(x, y, k, R.make_desc(P)) for x, y, k, P in reqs]
        wins, got = [], []
        for t, (x, y, k, P) in zip(tickets, reqs):
            st, res = srv.poll(t, wait_ms=60000)
            assert st == 0 and res.status == 0
            assert 0.0 <= res.dev_start_ms <= res.dev_end_ms
            wins.append((res.dev_start_ms, res.dev_end_ms))
            got.append(srv.fetch(t, x.size, k, 3)[0])
            assert srv.release(t) == 0
        for vals, (x, y, k, P) in zip(got, reqs):
            _, vals1 = run_alone(x, y, k, P, R.FP64)
            for a, b in zip(vals, vals1):
                np.testing.assert_array_equal(a, b)
        overlapping = [(i, j) for i in range(4) for j in range(i + 1, 4)
                       if wins[i][0] < wins[j][1] and wins[j][0] < wins[i][1]]
        assert overlapping, f"no two requests overlapped on the device: {wins}"
    finally:
        srv.close()
