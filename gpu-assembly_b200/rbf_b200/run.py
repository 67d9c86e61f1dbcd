"""Runs the hot path on one of the benchmark workloads: k-NN stencils once,
then the assembly `--reps` times in each requested form. Prints one JSON line
with the device time per assembly (CUDA events), stencils/s and the call's
counters; with both forms, the mixed form's max relative weight error
against the FP64 form (which is bit-identical to the CPU restatement of the
reference's assembly, as the parity tests establish).

    python -m rbf_b200.run --grid 256 --precision mixed --reps 3
    python -m rbf_b200.run --workload disk --precision both
    python -m rbf_b200.run --workload bump --precision both
    python -m rbf_b200.run --workload disk --precision fp64 --solve 200
    python -m rbf_b200.run --workload lbm --grid 1024 --reps 20

Workloads:
  periodic  jittered m x m grid in the periodic unit square (m = --grid),
            k=35, PHS r^5 + degree 3, fixed-width stencils
  disk      4,194,304 nodes on the unit disk, 8,192 boundary nodes with
            k in [48, 64] at degree 4, interior k in {21, 28, 35} at degree
            2/3: ragged CSR stencils, bucketed by system size, graph-replayed
  bump      2,097,152 nodes with a 4x Gaussian-bump density, k=64, PHS r^7 +
            degree 4 (n=79)
  lbm       D2Q9 semi-Lagrangian lattice Boltzmann on the periodic m x m grid:
            FP64 interpolation operators (k=21, PHS r^3 + degree 2) at the 8
            departure points x - c_a h/2, assembled once, then --reps fused
            stream + collide steps (populations in --populations precision)
The single-kernel shapes are also what the profiles are captured on (e.g.
under ncu with ``-k regex:asm_kernel`` on ``--grid 512``).

--solve N (disk only) then runs N BiCGSTAB iterations (tolerance 0, so
exactly N) on the assembled FP64 Laplacian with identity rows at the
boundary nodes, for the manufactured solution u = e^x sin 2y + x^2, and
reports ms per iteration and the algorithmic bytes per iteration
(solve_bytes) over that time.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

import rbf_b200 as R
from rbf_b200 import nodesets as NS


def _events_ms(fn, reps, stream):
    """Device time of fn(stats=False) on `stream` (CUDA events, after one
    warm-up call that also fills autotune caches and captures graphs), then
    one call with stats for the counters."""
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn(False)
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        ea.record(stream)
        fn(False)
        eb.record(stream)
        torch.cuda.synchronize()
        ms.append(ea.elapsed_time(eb))
    return ms, fn(True)


def _max_rel_err(a, b, ia):
    """Per-stencil max |a - b| / max |b|, worst over stencils and right-hand
    sides (rows of ragged width given by ia)."""
    worst = 0.0
    seg = torch.repeat_interleave(torch.arange(ia.numel() - 1, device=ia.device),
                                  (ia[1:] - ia[:-1]).long())
    n = ia.numel() - 1
    for va, vb in zip(a, b):
        num = torch.zeros(n, dtype=torch.float64, device=va.device)
        den = torch.zeros(n, dtype=torch.float64, device=va.device)
        num.scatter_reduce_(0, seg, (va - vb).abs(), reduce="amax")
        den.scatter_reduce_(0, seg, vb.abs(), reduce="amax")
        worst = max(worst, float((num / den.clamp_min(1e-300)).max()))
    return worst


def solve_bytes(n, nnz):
    """Algorithmic HBM bytes of one BiCGSTAB iteration of the CUDA solver
    over n rows and nnz stored weights (ragged CSR): the two operator
    applications read 12 B per weight (value + column), 4 B of row pointer,
    1 B of boundary flag and write 8 B per row, and gather their input vector
    (p, s) once (8 B per row each); the vector passes read rh (8 B), form s
    from r and v (24 B), update p (32 B) and u, r (56 B)."""
    return 24 * nnz + n * (2 * (4 + 1 + 8) + 8 + 8 + 8 + 24 + 32 + 56)


def disk_csr(ctx, dev, n=None):
    """The uneven disk workload on the device: node coordinates, per-node k
    and degree, and the ragged CSR stencils (the k_s nearest of every node,
    from one k-NN search at the largest k, trimmed per row)."""
    c = NS.config_disk_uneven(**({"n": n} if n else {}))
    x, y = c["x"], c["y"]
    n = x.size
    xd, yd = torch.as_tensor(x, device=dev), torch.as_tensor(y, device=dev)
    kvec = torch.as_tensor(c["kvec"], device=dev)
    deg = torch.as_tensor(c["degree"], device=dev)
    kmax = int(kvec.max())
    jaf = torch.empty(n * kmax, dtype=torch.int32, device=dev)
    ctx.knn_stencils(xd, yd, kmax, jaf)
    keep = torch.arange(kmax, device=dev)[None, :] < kvec[:, None]
    ja = jaf.view(n, kmax)[keep].contiguous()
    ia = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    ia[1:] = torch.cumsum(kvec, 0).to(torch.int32)
    del jaf
    torch.cuda.synchronize()
    return dict(c=c, xd=xd, yd=yd, kvec=kvec, deg=deg, ia=ia, ja=ja, n=n, nnz=int(ia[-1]),
                kmax=kmax)


def lbm(ctx, dev, stream, a):
    """The lattice Boltzmann workload: operators assembled once, then a.reps
    fused stream + collide steps ping-ponging two population arrays. Device
    time per step (CUDA events over all steps, after 3 warm-up steps) and the
    algorithmic bytes per node over it."""
    m, k, P = a.grid, a.k or 21, a.degree or 2
    x, y, _ = NS.jittered_grid(m, 0.3, seed=2, periodic=True)
    n = x.size
    xd, yd = torch.as_tensor(x, device=dev), torch.as_tensor(y, device=dev)
    ja = torch.empty(n * k, dtype=torch.int32, device=dev)
    ctx.knn_stencils(xd, yd, k, ja, period=(1.0, 1.0))
    xc, yc = R.lbm_departure_points(0.5 / m)
    xcd, ycd = torch.as_tensor(xc, device=dev), torch.as_tensor(yc, device=dev)
    W = torch.empty(8 * n * k, dtype=torch.float64, device=dev)
    vals = [W[i * n * k:(i + 1) * n * k] for i in range(8)]
    d = R.make_desc(P, 0, R.OP_INTERP, R.FP64, True, period=(1.0, 1.0), xc=xcd, yc=ycd, nc=8)
    st = ctx.assemble(d, xd, yd, k, ja, vals, stats=True)
    dt = torch.float64 if a.populations == "fp64" else torch.float32
    rho = torch.as_tensor(1.0 + 0.02 * np.sin(2 * np.pi * x), dtype=dt, device=dev)
    ux = torch.as_tensor(0.03 * np.cos(2 * np.pi * y), dtype=dt, device=dev)
    uy = torch.as_tensor(0.01 * np.sin(2 * np.pi * (x + y)), dtype=dt, device=dev)
    bufs = [torch.empty(9 * n, dtype=dt, device=dev) for _ in range(2)]
    R.lbm_feq(rho, ux, uy, bufs[0])
    torch.cuda.synchronize()

    def step(i):
        R.lbm_stream_collide(k, ja, W, 1.5, bufs[i % 2], bufs[(i + 1) % 2], rho, ux, uy,
                             stream=stream)
    for i in range(3):
        step(i)
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ea.record(stream)
    for i in range(a.reps):
        step(i)
    eb.record(stream)
    torch.cuda.synchronize()
    ms = ea.elapsed_time(eb) / max(a.reps, 1)
    es = dt.itemsize
    per_node = 8 * k * 8 + 4 * k + 2 * 9 * es + 3 * es
    return {"nodes": n, "k": k, "degree": P, "populations": a.populations,
            "operator_assembly_ms": st["ms"], "ms_per_step": ms,
            "node_updates_per_s": n / (ms * 1e-3), "bytes_per_node": per_node,
            "algorithmic_GBps": per_node * n / (ms * 1e-3) / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["periodic", "disk", "bump", "lbm"],
                    default="periodic")
    ap.add_argument("--grid", type=int, default=256, help="periodic: grid side")
    ap.add_argument("--n", type=int, default=None, help="disk/bump: number of nodes")
    ap.add_argument("--k", type=int, default=None, help="periodic: 35, lbm: 21")
    ap.add_argument("--degree", type=int, default=None, help="periodic: 3, lbm: 2")
    ap.add_argument("--populations", choices=["fp64", "fp32"], default="fp64",
                    help="lbm: precision of the populations")
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="mixed")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tune", action="store_true", help="autotune the shape first")
    ap.add_argument("--shape", default=None,
                    help="pin this compiled kernel shape (rbf_b200.variant_names()) for the "
                         "fixed-width workloads")
    ap.add_argument("--solve", type=int, default=0,
                    help="disk: BiCGSTAB iterations on the assembled Laplacian")
    a = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)  # non-default: the CSR path replays a CUDA graph on it
    forms = ["fp64", "mixed"] if a.precision == "both" else [a.precision]
    prec = {"fp64": R.FP64, "mixed": R.FP32_IR}
    out = {"workload": a.workload}

    with R.Context(0) as ctx:
        if a.workload == "lbm":
            out.update(lbm(ctx, dev, stream, a))
        elif a.workload == "disk":
            w = disk_csr(ctx, dev, a.n)
            c, xd, yd, ia, ja, deg = w["c"], w["xd"], w["yd"], w["ia"], w["ja"], w["deg"]
            kvec = w["kvec"]
            n, nnz, kmax = w["n"], w["nnz"], w["kmax"]
            res = {}
            for f in forms:
                vals = [torch.empty(nnz, dtype=torch.float64, device=dev) for _ in range(3)]
                info = torch.empty(n, dtype=torch.int32, device=dev)
                d = R.make_desc(3, 0, R.DEFAULT_OPS, prec[f], True)
                ms, st = _events_ms(lambda sts: ctx.assemble_csr(d, xd, yd, ia, ja, vals, degree=deg,
                                                                 info=info, stats=sts,
                                                                 stream=stream),
                                    a.reps, stream)
                res[f] = vals
                out[f] = {"ms": ms, "stencils_per_s": n / (min(ms) * 1e-3), "stats": st,
                          "bad_info": int((info != 0).sum())}
            out.update(stencils=n, nnz=nnz, k_range=[int(kvec.min()), kmax],
                       degrees=sorted(set(int(v) for v in np.unique(c["degree"]))))
            if a.solve > 0:
                L = res[forms[0]][0]  # the Laplacian rows
                bnd = torch.as_tensor(np.flatnonzero(c["flag"]).astype(np.int32), device=dev)
                f = -3.0 * torch.exp(xd) * torch.sin(2.0 * yd) + 2.0
                f[bnd.long()] = (torch.exp(xd) * torch.sin(2.0 * yd) + xd * xd)[bnd.long()]
                u = torch.zeros(n, dtype=torch.float64, device=dev)
                ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()  # f and u are made on the default stream
                with torch.cuda.stream(stream):
                    ctx.solve_bicgstab(L, ja, f, u, ia=ia, bnd=bnd, tol=0.0, maxit=8,
                                       stream=stream)  # warm-up: workspace and graph
                    u.zero_()
                    ea.record(stream)
                    st_, it, rel = ctx.solve_bicgstab(L, ja, f, u, ia=ia, bnd=bnd, tol=0.0,
                                                      maxit=a.solve, stream=stream)
                    eb.record(stream)
                torch.cuda.synchronize()
                ms = ea.elapsed_time(eb)
                out["solve"] = {"status": R.lib().rbfb_status_string(st_).decode(),
                                "iterations": it, "relres": rel, "ms": ms,
                                "ms_per_iteration": ms / max(it, 1),
                                "algorithmic_GBps": solve_bytes(n, nnz) * it / (ms * 1e-3) / 1e9}
            if len(forms) == 2:
                out["mixed_max_rel_err_vs_fp64"] = _max_rel_err(res["mixed"], res["fp64"], ia)
        else:
            if a.workload == "bump":
                c = NS.config_bump(**({"n": a.n} if a.n else {}))
                x, y = c["x"], c["y"]
                k, P, per = c["k"], c["P"], None
            else:
                x, y, _ = NS.jittered_grid(a.grid, 0.3, seed=2, periodic=True)
                k, P, per = a.k or 35, a.degree or 3, (1.0, 1.0)
            n = x.size
            xd, yd = torch.as_tensor(x, device=dev), torch.as_tensor(y, device=dev)
            ja = torch.empty(n * k, dtype=torch.int32, device=dev)
            ctx.knn_stencils(xd, yd, k, ja, period=per)
            torch.cuda.synchronize()
            res = {}
            shape = None
            for f in forms:
                vals = [torch.empty(n * k, dtype=torch.float64, device=dev) for _ in range(3)]
                info = torch.empty(n, dtype=torch.int32, device=dev)
                d = R.make_desc(P, 0, R.DEFAULT_OPS, prec[f], True, period=per)
                if a.shape:
                    ctx.select_variant(d, k, R.variant_names().index(a.shape))
                    shape = a.shape
                elif a.tune:
                    shape = R.variant_name(ctx.autotune(d, xd, yd, k, ja, vals))
                ms, st = _events_ms(lambda sts: ctx.assemble(d, xd, yd, k, ja, vals, info, stats=sts,
                                                             stream=stream), a.reps, stream)
                res[f] = vals
                out[f] = {"ms": ms, "stencils_per_s": n / (min(ms) * 1e-3), "stats": st,
                          "bad_info": int((info != 0).sum()), "shape": shape}
            out.update(stencils=n, k=k, degree=P)
            if a.workload == "periodic":
                out["grid"] = a.grid
            if len(forms) == 2:
                ia = torch.arange(0, (n + 1) * k, k, dtype=torch.int32, device=dev)
                out["mixed_max_rel_err_vs_fp64"] = _max_rel_err(res["mixed"], res["fp64"], ia)
        torch.cuda.synchronize()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
