"""End-to-end host call, the uneven (CSR, bucketed) batch and the autotuner,
each against the oracle or against the fixed-width device path."""
import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from conftest import golden
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu


def test_host_pipeline_equals_device_path(ctx, torch_cuda):
    T = torch_cuda
    g = golden("square69_k21")
    x, y = g["x"], g["y"]
    n, k = x.size, 21
    for prec in (R.FP64, R.FP32_IR):
        d = R.make_desc(2, precision=prec)
        vals_h = [np.empty(n * k) for _ in range(3)]
        ja_out = np.empty(n * k, np.int32)
        info = np.empty(n, np.int32)
        st = ctx.assemble_host(d, x, y, k, vals_h, ja_out_h=ja_out, info_h=info)
        np.testing.assert_array_equal(ja_out, g["ja_nanoflann"])
        assert (info == 0).all() and st["stencils"] == n
        Wo, _ = O.assemble(x, y, g["ja_nanoflann"], k, 2)
        tol = 1e-12 if prec == R.FP64 else 1e-10
        assert O.max_rel_err(np.stack(vals_h), Wo, k).max() <= tol


def test_host_pipeline_given_stencils_many_chunks(ctx, torch_cuda):
    # 300 x 300 periodic grid: several chunks, k=35 degree 3, given stencils
    x, y, _ = NS.jittered_grid(300, 0.3, seed=21, periodic=True)
    n, k = x.size, 35
    T = torch_cuda
    ja = T.empty(n * k, dtype=T.int32, device="cuda")
    ctx.knn_stencils(T.as_tensor(x).cuda(), T.as_tensor(y).cuda(), k, ja, period=(1.0, 1.0))
    ja_h = ja.cpu().numpy()
    d = R.make_desc(3, precision=R.FP32_IR, period=(1.0, 1.0))
    vals_h = [np.empty(n * k) for _ in range(3)]
    ctx.assemble_host(d, x, y, k, vals_h, ja_h=ja_h)
    rows = np.arange(0, n, 997)
    idx = (rows[:, None] * k + np.arange(k)[None, :]).ravel()
    Wo, _ = O.assemble(x, y, ja_h, k, 3, period=(1.0, 1.0))
    W = np.stack(vals_h)
    assert O.max_rel_err(W[:, idx], Wo[:, idx], k).max() <= 1e-10


def test_csr_uneven_matches_oracle(ctx, torch_cuda):
    T = torch_cuda
    # small disk: boundary nodes k in [48, 64] degree 4, interior k in {21, 28, 35}
    # degree 2/3: four kernel shapes in one call
    c = NS.config_disk_uneven(n=6000, nb=200, seed=13)
    kvec = c["kvec"]
    deg = c["degree"]
    x, y = c["x"], c["y"]
    n = x.size
    kmax = int(kvec.max())
    jaf = O.knn_brute(x, y, kmax).reshape(n, kmax)
    ia = np.zeros(n + 1, np.int32)
    ia[1:] = np.cumsum(kvec)
    ja = np.concatenate([jaf[s, : kvec[s]] for s in range(n)]).astype(np.int32)
    for prec, tol in ((R.FP64, 1e-12), (R.FP32_IR, 1e-10)):
        d = R.make_desc(2, precision=prec)
        vals = [T.empty(int(ia[-1]), dtype=T.float64, device="cuda") for _ in range(3)]
        info = T.full((n,), -3, dtype=T.int32, device="cuda")
        st = ctx.assemble_csr(d, T.as_tensor(x).cuda(), T.as_tensor(y).cuda(),
                              T.as_tensor(ia).cuda(), T.as_tensor(ja).cuda(), vals,
                              degree=T.as_tensor(deg).cuda(), info=info, stats=True)
        T.cuda.synchronize()
        assert (info.cpu().numpy() == 0).all()
        # FP64: the whole batch in one launch; the refined form: one bucket
        # per kernel shape (four here)
        assert st["buckets"] == 1 if prec == R.FP64 else st["buckets"] >= 4
        Wo, io = O.assemble_csr(x, y, ia, ja, degree=deg, P=2, Q=0)
        W = np.stack([v.cpu().numpy() for v in vals])
        if prec == R.FP64:
            np.testing.assert_array_equal(W, Wo)  # the oracle's operations, in order
        # ragged error per stencil
        worst = 0.0
        for s in range(n):
            a, b = ia[s], ia[s + 1]
            e = np.abs(W[:, a:b] - Wo[:, a:b]).max(axis=1) / np.abs(Wo[:, a:b]).max(axis=1)
            worst = max(worst, float(e.max()))
        assert worst <= tol, (prec, worst)


def test_csr_unsupported_stencil_is_reported(ctx, torch_cuda):
    """One stencil of an unsupported degree in an FP64 uneven batch: the
    one launch skips it (it sorts into the last class) and the call reports
    EUNSUPPORTED; every other stencil is assembled, bit-identical to the
    oracle."""
    T = torch_cuda
    c = NS.config_disk_uneven(n=3000, nb=120, seed=19)
    kvec, x, y = c["kvec"], c["x"], c["y"]
    n = x.size
    kmax = int(kvec.max())
    jaf = O.knn_brute(x, y, kmax).reshape(n, kmax)
    ia = np.zeros(n + 1, np.int32)
    ia[1:] = np.cumsum(kvec)
    ja = np.concatenate([jaf[s, : kvec[s]] for s in range(n)]).astype(np.int32)
    deg = c["degree"].copy()
    bad = 7
    deg[bad] = 5  # no kernel takes degree 5
    vals = [T.full((int(ia[-1]),), float("nan"), dtype=T.float64, device="cuda") for _ in range(3)]
    info = T.full((n,), -3, dtype=T.int32, device="cuda")
    with pytest.raises(R.RbfError) as e:
        ctx.assemble_csr(R.make_desc(2), T.as_tensor(x).cuda(), T.as_tensor(y).cuda(),
                         T.as_tensor(ia).cuda(), T.as_tensor(ja).cuda(), vals,
                         degree=T.as_tensor(deg).cuda(), info=info, stats=True)
    assert e.value.status == R.EUNSUPPORTED
    T.cuda.synchronize()
    W = np.stack([v.cpu().numpy() for v in vals])
    Wo, _ = O.assemble_csr(x, y, ia, ja, degree=c["degree"], P=2, Q=0)
    keep = np.ones(int(ia[-1]), bool)
    keep[ia[bad]:ia[bad + 1]] = False
    np.testing.assert_array_equal(W[:, keep], Wo[:, keep])
    assert np.isnan(W[:, ~keep]).all()  # the skipped stencil's row is untouched
    io = info.cpu().numpy()
    assert io[bad] == -3 and (np.delete(io, bad) == 0).all()


def test_autotune_picks_a_compiled_shape(ctx, torch_cuda):
    T = torch_cuda
    g = golden("square69_k21")
    n, k = g["x"].size, 21
    d = R.make_desc(2, precision=R.FP32_IR)
    vals = [T.empty(n * k, dtype=T.float64, device="cuda") for _ in range(3)]
    v = ctx.autotune(d, T.as_tensor(g["x"]).cuda(), T.as_tensor(g["y"]).cuda(), k,
                     T.as_tensor(g["ja_nanoflann"]).cuda(), vals)
    assert v >= 0
    # the tuned shape is used and still correct
    info = T.zeros(n, dtype=T.int32, device="cuda")
    ctx.assemble(d, T.as_tensor(g["x"]).cuda(), T.as_tensor(g["y"]).cuda(), k,
                 T.as_tensor(g["ja_nanoflann"]).cuda(), vals, info)
    T.cuda.synchronize()
    Wo, _ = O.assemble(g["x"], g["y"], g["ja_nanoflann"], k, 2)
    assert O.max_rel_err(np.stack([v.cpu().numpy() for v in vals]), Wo, k).max() <= 1e-10


def test_range_and_shards_equal_the_whole(ctx, torch_cuda):
    T = torch_cuda
    from rbf_b200 import shard
    g = golden("square69_k21")
    x, y = T.as_tensor(g["x"]).cuda(), T.as_tensor(g["y"]).cuda()
    n, k = x.numel(), 21
    d = R.make_desc(2)
    full = [T.empty(n * k, dtype=T.float64, device="cuda") for _ in range(3)]
    ja = T.as_tensor(g["ja_nanoflann"]).cuda()
    ctx.assemble(d, x, y, k, ja, full)
    T.cuda.synchronize()
    # each range into outputs that start as NaN: every row written, every
    # stencil's info set
    for first, count in ((0, 1587), (1587, 1587), (3174, n - 3174)):
        jr = ja[first * k:(first + count) * k].contiguous()
        vr = [T.full((count * k,), float("nan"), dtype=T.float64, device="cuda")
              for _ in range(3)]
        ir = T.full((count,), -7, dtype=T.int32, device="cuda")
        st = ctx.assemble_range(d, first, count, x, y, k, jr, vr, ir, stats=True)
        T.cuda.synchronize()
        assert st["stencils"] == count and (ir.cpu().numpy() == 0).all(), (first, st)
        for q in range(3):
            got = vr[q].cpu().numpy()
            want = full[q][first * k:(first + count) * k].cpu().numpy()
            bad = np.flatnonzero(got != want)
            assert bad.size == 0, (first, q, bad.size, bad[:5] // k, got[bad[:3]], want[bad[:3]])
    parts_ja, parts_w = [], [[], [], []]
    ja_h = g["ja_nanoflann"]
    full_h = [f.cpu().numpy() for f in full]

    def check(rank, first, count, jr, vr, when):
        a, b = first * k, (first + count) * k
        bad_ja = np.flatnonzero(jr.cpu().numpy() != ja_h[a:b])
        assert bad_ja.size == 0, (when, rank, "ja", bad_ja.size, bad_ja[:4] // k,
                                  jr.cpu().numpy()[bad_ja[:4]])
        for q in range(3):
            bad = np.flatnonzero(vr[q].cpu().numpy() != full_h[q][a:b])
            assert bad.size == 0, (when, rank, "w", q, bad.size, bad[:4] // k)

    shards = []

    def check_all(when):
        for sh in shards:
            check(*sh, when)

    for rank in range(3):  # three "ranks" on one GPU, one after another
        # shard.assemble_shard's steps, checked in between
        first, count = shard.node_range(n, 3, rank)
        jr = T.empty(count * k, dtype=T.int32, device="cuda")
        vr = [T.empty(count * k, dtype=T.float64, device="cuda") for _ in range(3)]
        ir = T.empty(count, dtype=T.int32, device="cuda")
        xq, yq = x[first:first + count].contiguous(), y[first:first + count].contiguous()
        ctx.knn_query(x, y, xq, yq, k, jr)
        T.cuda.synchronize()
        check_all(f"after rank {rank} knn")
        bad = np.flatnonzero(jr.cpu().numpy() != ja_h[first * k:(first + count) * k])
        assert bad.size == 0, ("own ja", rank, bad.size)
        ctx.assemble_range(d, first, count, x, y, k, jr, vr, ir)
        T.cuda.synchronize()
        shards.append((rank, first, count, jr, vr))
        check_all(f"after rank {rank} assembly")
        parts_ja.append(jr)
        for q in range(3):
            parts_w[q].append(vr[q])
    # and the library's own helper
    for rank in range(3):
        first, count, jr, vr = shard.assemble_shard(ctx, d, x, y, k, rank, 3)
        T.cuda.synchronize()
        check(rank, first, count, jr, vr, "assemble_shard")
    check_all("after all calls")
    np.testing.assert_array_equal(T.cat(parts_ja).cpu().numpy(), g["ja_nanoflann"])
    for q in range(3):
        want = full[q].cpu().numpy()
        at = 0
        for rank in range(3):
            got = parts_w[q][rank].cpu().numpy()
            bad = np.flatnonzero(got != want[at:at + got.size])
            assert bad.size == 0, (rank, q, bad.size, bad[:5] // k)
            at += got.size


def test_spmv_with_boundary_fix(ctx, torch_cuda):
    T = torch_cuda
    g = golden("shu_square_4786")
    x, y = g["x"], g["y"]
    n, k = x.size, 21
    W, _ = O.assemble(x, y, g["ja_nanoflann"], k, 2)
    u = np.sin(3 * x) * np.cos(2 * y)
    bnd = np.flatnonzero(g["flag"]).astype(np.int32)
    out = T.empty(n, dtype=T.float64, device="cuda")
    ud = T.as_tensor(u).cuda()
    jad = T.as_tensor(g["ja_nanoflann"]).cuda()
    Wd = T.as_tensor(W[0]).cuda()
    bd = T.as_tensor(bnd).cuda()
    R.spmv(n, k, jad, Wd, ud, out, bd)
    T.cuda.synchronize()
    ref = O.spmv(g["ja_nanoflann"], W[0], u, k, bnd)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)  # same order, bit for bit
    # weights and columns off a 16-byte boundary: scalar loads, the same sums
    Wb = T.empty(W[0].size + 1, dtype=T.float64, device="cuda")
    jb = T.empty(n * k + 1, dtype=T.int32, device="cuda")
    Wu, ju = Wb[1:], jb[1:]
    Wu.copy_(Wd)
    ju.copy_(jad)
    out2 = T.empty_like(out)
    R.spmv(n, k, ju, Wu, ud, out2, bd)
    T.cuda.synchronize()
    np.testing.assert_array_equal(out2.cpu().numpy(), ref)
    # and it is a Laplacian: -13 u in the interior up to the discretisation error
    interior = np.setdiff1d(np.arange(n), bnd)
    assert np.abs(ref[interior] + 13 * u[interior]).max() < 0.5


def test_csr_batch_graph_replay(ctx, torch_cuda):
    # on a non-default stream the batch is captured once, then replayed
    T = torch_cuda
    c = NS.config_disk_uneven(n=3000, nb=120, seed=17)
    x, y, kvec, deg = c["x"], c["y"], c["kvec"], c["degree"]
    n = x.size
    kmax = int(kvec.max())
    jaf = O.knn_brute(x, y, kmax).reshape(n, kmax)
    ia = np.zeros(n + 1, np.int32)
    ia[1:] = np.cumsum(kvec)
    ja = np.concatenate([jaf[s, : kvec[s]] for s in range(n)]).astype(np.int32)
    xd, yd = T.as_tensor(x).cuda(), T.as_tensor(y).cuda()
    iad, jad, degd = T.as_tensor(ia).cuda(), T.as_tensor(ja).cuda(), T.as_tensor(deg).cuda()
    vals = [T.empty(int(ia[-1]), dtype=T.float64, device="cuda") for _ in range(3)]
    d = R.make_desc(2)
    s = T.cuda.Stream()
    outs, launches = [], []
    for rep in range(3):
        for v in vals:
            v.fill_(np.nan)
        l0 = ctx.launches()
        with T.cuda.stream(s):
            ctx.assemble_csr(d, xd, yd, iad, jad, vals, degree=degd, stream=s)
        s.synchronize()
        launches.append(ctx.launches() - l0)
        outs.append(np.stack([v.cpu().numpy() for v in vals]))
    assert launches[0] == launches[1] == launches[2] > 0
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])
    Wo, _ = O.assemble_csr(x, y, ia, ja, degree=deg, P=2, Q=0)
    np.testing.assert_array_equal(outs[0], Wo)  # FP64 path: bit-identical to the oracle


@pytest.mark.parametrize("workload", ["disk", "bump"])
def test_workload_runner_small(torch_cuda, capsys, workload):
    # the benchmark workloads at a small size: every stencil solved, the mixed
    # form within its bound of the FP64 form (degree 4 at cond ~1e6..1e7: the
    # mixed form's FP64 fallback keeps it within 1e-9)
    import json
    from rbf_b200 import run
    run.main(["--workload", workload, "--n", "20000", "--precision", "both", "--reps", "1"])
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["stencils"] == 20000
    for form in ("fp64", "mixed"):
        assert out[form]["bad_info"] == 0
        assert out[form]["stats"]["stencils"] == 20000
    assert out["mixed_max_rel_err_vs_fp64"] <= 1e-9
    if workload == "disk":
        assert out["fp64"]["stats"]["buckets"] == 1  # one launch for the uneven batch
        assert out["mixed"]["stats"]["buckets"] >= 3
