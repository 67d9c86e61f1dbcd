"""Benchmark of the RBF-FD assembly hot path on B200.

Headline workload (one step = one pass of the hot path over one node set):
the periodic 1024 x 1024 jittered grid (1,048,576 nodes, seed 2), k = 35
nearest neighbours (periodic k-NN), PHS r^5 + degree-3 polynomials (n = 45),
three operators (Laplacian, d/dx, d/dy), FP64 weights written as CSR values.
Every step runs the k-NN search and the assembly; inputs (16 MB of nodes)
are resident in HBM, the 147 MB stencil table and 881 MB of weights are
rewritten each step, so every step moves more than the 126 MB L2.

Both forms are timed on the same node set: plain FP64, and FP32
factorisation with FP64 iterative refinement (the mixed form). Each one's
max relative weight error against the FP64 CPU oracle is taken on a stencil
sample. The headline `value` is the faster form that meets the 1e-10 bound.
Also reported: the end-to-end rate through the host-buffer entry point
(pinned host memory, copies inside the timed region), the CPU baseline (the
reference's own k-NN search + the oracle's CPU assembly on the full node
set) and, at N = 1, the other configurations:

  c3  4,194,304 uneven stencils on the unit disk (ragged CSR, k 21-64,
      degree 2-4), bucketed, graph-replayed: FP64 and mixed stencils/s,
      errors on 2,048 sampled stencils against the FP64 oracle, fallbacks;
  c4  2,097,152 stencils, k = 64, r^7 + degree 4, Gaussian-bump density:
      FP64 and mixed, errors against the long-double oracle, fallbacks;
  c5  the 2,000-request serving stream under a 40 GB HBM budget: p50/p99
      latency at 80 % of the measured capacity over repeats (with spread),
      aggregate stencils/s against serial plain FP64;
  lbm the D2Q9 lattice Boltzmann step that consumes interpolation operators
      (fused semi-Lagrangian streaming + BGK collision) on the 1024^2 grid,
      with its HBM roofline fraction.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) the ranks share ONE node set of N * 1024^2 nodes
(grid side round(1024 sqrt N)), broadcast once from rank 0, and each rank
assembles the stencils of its contiguous node range (weak scaling, no
data-path collective); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gpu-assembly_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

M_GRID = 1024
K, P, Q = 35, 3, 5
NRHS = 3
N_SYS = K + (P + 1) * (P + 2) // 2  # 45
FLOP_PER_STENCIL = 2.0 / 3.0 * N_SYS ** 3 + 2 * NRHS * N_SYS ** 2  # 72,900
# algorithmic bytes of one stencil's assembly (no-reuse bound): its ja row
# (4 B per neighbour), its centre (16 B), the neighbour coordinates it
# gathers (16 B per neighbour) and NRHS weight rows (8 B per neighbour each)
HBM_BYTES_PER_STENCIL = (4 + 16 + 8 * NRHS) * K + 16  # 1,556
# compulsory HBM bytes: the gathered coordinates are the same nodes'
# coordinates again and again (L2 reuse), so only ja, centre, weights and
# the 4 B info word must cross HBM
HBM_COMPULSORY_PER_STENCIL = (4 + 8 * NRHS) * K + 16 + 4  # 1,000
METRIC = "stencils/s k=35 deg3 (periodic 1024^2 jittered grid, 3 operators)"


def n_sys(k, P_):
    return k + (P_ + 1) * (P_ + 2) // 2


def flop_per_stencil(k, P_, nrhs=NRHS):
    n = n_sys(k, P_)
    return 2.0 / 3.0 * n ** 3 + 2 * nrhs * n ** 2


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text()), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def grid_side(ws):
    """Grid side of the shared node set of `ws` ranks: about ws * 1024^2 nodes."""
    return int(round(M_GRID * math.sqrt(ws)))


# ---- CPU legs (the oracle and the reference's own search: checker/baseline) ----

def cpu_pass(x, y, cores):
    """One CPU pass of the headline workload: the reference's own ckdtree
    periodic search (oracle/_ref, when built; else the oracle's brute force)
    and the oracle's FP64 CPU assembly (the reference has no CPU assembly),
    OpenMP on `cores` threads. Returns (knn_s, assembly_s, knn_kind)."""
    import oracle as O
    O.set_threads(cores)
    t0 = time.perf_counter()
    if O.ref() is not None:
        O.ref().ref_set_threads(cores)
        ja = O.ref_kdtree_stencils(x, y, K, period=(1.0, 1.0))
        kind = "reference ckdtree (KdTree::knn_stencils)"
    else:
        ja = O.knn_brute(x, y, K, period=(1.0, 1.0))
        kind = "oracle brute force"
    t1 = time.perf_counter()
    O.assemble(x, y, ja, K, P, period=(1.0, 1.0))
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1, kind


def cpu_baseline_full(x, y):
    """The CPU path on the full headline node set, one pass, all host
    threads (run before any GPU work so the OpenMP pool never forks after
    CUDA)."""
    cores = os.cpu_count() or 1
    tk, ta, kind = cpu_pass(x, y, cores)
    n = x.size
    # one thread, on a 256 x 256 grid of the same distribution (a bounded
    # sample: the per-stencil cost is the same, the search's log n smaller)
    from rbf_b200 import nodesets as NS
    xs, ys, _ = NS.jittered_grid(256, 0.3, seed=2, periodic=True)
    tk1, ta1, _ = cpu_pass(xs, ys, 1)
    return {"value": n / (tk + ta), "unit": "stencils/s", "cores": cores, "kind": "reference"
            if kind.startswith("reference") else "port",
            "sample": f"the full periodic {M_GRID}x{M_GRID} node set ({n} stencils), one pass: "
                      f"{kind} {tk:.3f} s + oracle FP64 assembly (CPU restatement, OpenMP; the "
                      f"reference has no CPU assembly) {ta:.3f} s",
            "single_thread": {"value": xs.size / (tk1 + ta1), "unit": "stencils/s", "cores": 1,
                              "sample": f"periodic 256x256 grid of the same distribution "
                                        f"({xs.size} stencils), one pass: {kind} {tk1:.3f} s + "
                                        f"oracle FP64 assembly {ta1:.3f} s"}}


def reference_arm(args):
    """The reference's CPU implementation of the path on this box's host
    cores, on the headline workload at full size: its own ckdtree periodic
    k-NN search (compiled from its sources) + the oracle's FP64 assembly."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle as O
    from rbf_b200 import nodesets as NS
    cores = os.cpu_count() or 1
    x, y, _ = NS.jittered_grid(M_GRID, 0.3, seed=2, periodic=True)
    n = x.size
    times = []
    for i in range(args.warmup + args.steps):
        tk, ta, kind = cpu_pass(x, y, cores)
        if i >= args.warmup:
            times.append(tk + ta)
    T = sum(times)
    v = n * len(times) / T
    line = {"metric": METRIC, "value": v, "unit": "stencils/s", "impl": "reference",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * T / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered grid)",
            "config": {"workload": f"periodic {M_GRID}x{M_GRID} jittered grid (+-0.3h), k={K} "
                                   f"k-NN + assembly, PHS r^{Q} + degree {P} (n={N_SYS}), "
                                   "Laplacian/dx/dy, FP64",
                       "stencils_per_step": n, "same_config": True},
            "cpu_baseline": {"value": v, "unit": "stencils/s", "cores": cores,
                             "kind": "reference" if O.ref() is not None else "port",
                             "sample": "the full workload each step. k-NN: "
                                       f"{kind}, compiled from the reference's sources; "
                                       "assembly: the oracle's CPU restatement (the reference "
                                       "has no CPU assembly; its GPU assembly needs the closed "
                                       "cuSolverDx and is unavailable on this box)"},
            "e2e": {"value": v, "unit": "stencils/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def traffic_per_launch(form):
    """DRAM bytes per launch of the dominant kernel, from the committed ncu
    summary (profiles/), scaled to the full workload; None if absent."""
    p = ROOT / "profiles" / f"asm_{form}_periodic512.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("traffic_bytes_per_launch_full:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def sampled_oracle(O, x, y, ia_h, ja_h, rows, degree=None, P_=P, Q_=0, period=None, ld=False,
                   k=None, centres=None):
    """The oracle's weights of the sampled stencils `rows` (ragged rows of
    ia_h/ja_h, centred on nodes `centres`, by default the rows themselves):
    the nodes are renumbered so the sampled centres come first, then just
    those stencils are assembled. ld=True uses the long-double oracle (fixed
    width k). Returns (values (nrhs, nnz_sampled), ia_s)."""
    n = x.size
    centres = rows if centres is None else centres
    order = np.concatenate([centres, np.setdiff1d(np.arange(n), centres)])
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    seg = [ja_h[ia_h[r]:ia_h[r + 1]] for r in rows]
    ja_s = inv[np.concatenate(seg)].astype(np.int32)
    ia_s = np.zeros(rows.size + 1, np.int32)
    ia_s[1:] = np.cumsum([s.size for s in seg])
    if ld:
        W, _ = O.assemble_ld(x[order], y[order], ja_s, k, P_, Q_ or None, period=period,
                             nstencils=rows.size)
        return W, ia_s
    deg = None if degree is None else degree[centres].astype(np.int8)
    W, _ = O.assemble_csr(x[order], y[order], ia_s, ja_s, degree=deg, P=P_, Q=Q_,
                          period=period, nstencils=rows.size)
    return W, ia_s


def ragged_rel_err(W, Wo, ia_s):
    """Max over stencils and right-hand sides of ||w - w_ref||_inf /
    ||w_ref||_inf, stencil s spanning entries ia_s[s] .. ia_s[s+1]."""
    starts = ia_s[:-1]
    worst = 0.0
    for a, b in zip(W, Wo):
        num = np.maximum.reduceat(np.abs(a - b), starts)
        den = np.maximum.reduceat(np.abs(b), starts)
        worst = max(worst, float((num / np.where(den > 0, den, 1.0)).max()))
    return worst


def sample_values(vals, ia_h, rows):
    idx = np.concatenate([np.arange(ia_h[r], ia_h[r + 1]) for r in rows])
    return np.stack([v.cpu().numpy()[idx] for v in vals])


def events_ms(torch, stream, fn, reps):
    """Min and mean device time of fn() on `stream` (CUDA events, after one
    warm-up call)."""
    fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        fn()
        eb.record(stream)
        torch.cuda.synchronize()
        out.append(ea.elapsed_time(eb))
    return min(out), sum(out) / len(out)


def config3(R, O, torch, ctx, dev, reps=3):
    """4,194,304 uneven stencils on the unit disk, ragged CSR, bucketed by
    system size into persistent launches replayed from a CUDA graph."""
    from rbf_b200 import run as RUN
    w = RUN.disk_csr(ctx, dev)
    xd, yd, ia, ja, deg, n, nnz = w["xd"], w["yd"], w["ia"], w["ja"], w["deg"], w["n"], w["nnz"]
    stream = torch.cuda.Stream(dev)
    res = {"workload": "unit disk, 4,194,304 nodes (8,192 boundary, k 48-64, degree 4; "
                       "interior k in {21, 28, 35}, degree 2-3), ragged CSR, 3 operators",
           "stencils": n, "nnz": nnz}
    rows = np.random.default_rng(3).choice(n, 2048, replace=False)
    rows[:64] = np.arange(64)  # boundary (degree-4) stencils are always in the sample
    ia_h, ja_h = ia.cpu().numpy(), ja.cpu().numpy()
    Wo, ia_s = sampled_oracle(O, w["c"]["x"], w["c"]["y"], ia_h, ja_h, rows,
                              degree=w["c"]["degree"])
    kk, dd = w["c"]["kvec"].astype(np.int64), w["c"]["degree"].astype(np.int64)
    nsys = kk + (dd + 1) * (dd + 2) // 2
    flops = float(np.sum(2.0 / 3.0 * nsys ** 3 + 2 * NRHS * nsys ** 2))
    for form, prec in (("fp64", R.FP64), ("mixed", R.FP32_IR)):
        vals = [torch.empty(nnz, dtype=torch.float64, device=dev) for _ in range(NRHS)]
        info = torch.empty(n, dtype=torch.int32, device=dev)
        d = R.make_desc(3, 0, R.DEFAULT_OPS, prec, True)

        def call():
            ctx.assemble_csr(d, xd, yd, ia, ja, vals, degree=deg, info=info, stream=stream)
        mn, mean = events_ms(torch, stream, call, reps)
        l0 = ctx.launches()
        st = ctx.assemble_csr(d, xd, yd, ia, ja, vals, degree=deg, info=info, stats=True,
                              stream=stream)
        launches = ctx.launches() - l0
        err = ragged_rel_err(sample_values(vals, ia_h, rows), Wo, ia_s)
        res[form] = {"stencils_per_s": n / (mn * 1e-3), "ms": mn, "ms_mean": mean,
                     "tflops": flops / (mn * 1e-3) / 1e12,
                     "max_rel_weight_err_vs_fp64_oracle": err, "fallback": st["fallback"],
                     "buckets": st["buckets"], "kernel_launches_per_call": launches,
                     "singular": st["singular"]}
        del vals, info
    res["mixed_over_fp64"] = res["fp64"]["ms"] / res["mixed"]["ms"]
    res["error_sample"] = "2,048 stencils (64 boundary), FP64 CPU oracle"
    res["launches_note"] = ("fp64: one assembly launch per call, after a device counting sort "
                            "of the stencils by class (3 small kernels) and before the singular "
                            "count; mixed: one launch per bucket plus its FP64 fallback launch")
    del w
    torch.cuda.synchronize()
    return res


def config4(R, O, NS, torch, ctx, dev, reps=3):
    """2,097,152 stencils, k = 64, r^7 + degree 4 (n = 79), Gaussian-bump
    density; errors against the long-double oracle."""
    c = NS.config_bump()
    x, y, k, P_ = c["x"], c["y"], c["k"], c["P"]
    n = x.size
    xd, yd = torch.as_tensor(x, device=dev), torch.as_tensor(y, device=dev)
    ja = torch.empty(n * k, dtype=torch.int32, device=dev)
    ctx.knn_stencils(xd, yd, k, ja)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    rows = np.random.default_rng(4).choice(n, 2048, replace=False)
    ja_h = ja.cpu().numpy()
    ia_h = (np.arange(n + 1, dtype=np.int64) * k)
    Wo, ia_s = sampled_oracle(O, x, y, ia_h, ja_h, rows, P_=P_, ld=True, k=k)
    res = {"workload": "Gaussian-bump density (4x) on [0,1]^2, 2,097,152 nodes, k=64, "
                       "r^7 + degree 4 (n=79), 3 operators", "stencils": n}
    for form, prec in (("fp64", R.FP64), ("mixed", R.FP32_IR)):
        vals = [torch.empty(n * k, dtype=torch.float64, device=dev) for _ in range(NRHS)]
        info = torch.empty(n, dtype=torch.int32, device=dev)
        d = R.make_desc(P_, 0, R.DEFAULT_OPS, prec, True)

        def call():
            ctx.assemble(d, xd, yd, k, ja, vals, info, stream=stream)
        mn, mean = events_ms(torch, stream, call, reps)
        st = ctx.assemble(d, xd, yd, k, ja, vals, info, stats=True, stream=stream)
        err = ragged_rel_err(sample_values(vals, ia_h, rows), Wo, ia_s)
        res[form] = {"stencils_per_s": n / (mn * 1e-3), "ms": mn, "ms_mean": mean,
                     "tflops": flop_per_stencil(k, P_) * n / (mn * 1e-3) / 1e12,
                     "max_rel_weight_err_vs_long_double": err, "fallback": st["fallback"],
                     "singular": st["singular"]}
        del vals, info
    res["mixed_over_fp64"] = res["fp64"]["ms"] / res["mixed"]["ms"]
    res["error_sample"] = "2,048 stencils, x87 long-double oracle (same algorithm)"
    del ja, xd, yd
    torch.cuda.synchronize()
    return res


def lbm_bytes_per_node(k):
    """Compulsory HBM bytes of one stream + collide step per node: its ja row
    (4k), its 8 weight rows (64k), its 9 populations read and written, and
    rho, ux, uy written (the gathered neighbour populations are the same
    arrays again: L2 reuse)."""
    return 4 * k + 64 * k + 9 * 8 + 9 * 8 + 3 * 8


def config_lbm(R, NS, torch, ctx, dev, m=M_GRID, k=21, steps=20):
    """D2Q9 semi-Lagrangian lattice Boltzmann on the periodic m x m grid:
    interpolation operators at the 8 departure points (k = 21, r^3 +
    degree 2, dt = h/2) assembled once, then fused stream + collide steps
    (FP64), timed with CUDA events."""
    x, y, _ = NS.jittered_grid(m, 0.3, seed=2, periodic=True)
    n = x.size
    xd, yd = torch.as_tensor(x, device=dev), torch.as_tensor(y, device=dev)
    ja = torch.empty(n * k, dtype=torch.int32, device=dev)
    ctx.knn_stencils(xd, yd, k, ja, period=(1.0, 1.0))
    xc, yc = R.lbm_departure_points(0.5 / m)
    xcd, ycd = torch.as_tensor(xc, device=dev), torch.as_tensor(yc, device=dev)
    W = torch.empty(8 * n * k, dtype=torch.float64, device=dev)
    vals = [W[a * n * k:(a + 1) * n * k] for a in range(8)]
    d = R.make_desc(2, 3, R.OP_INTERP, R.FP64, True, period=(1.0, 1.0), xc=xcd, yc=ycd, nc=8)
    ctx.assemble(d, xd, yd, k, ja, vals)  # the first launch loads the kernel's module
    st = ctx.assemble(d, xd, yd, k, ja, vals, stats=True)
    rho = 1.0 + 0.02 * np.sin(2 * np.pi * x)
    ux = 0.03 * np.cos(2 * np.pi * y)
    uy = 0.01 * np.sin(2 * np.pi * (x + y))
    fa = torch.empty(9 * n, dtype=torch.float64, device=dev)
    R.lbm_feq(torch.as_tensor(rho, device=dev), torch.as_tensor(ux, device=dev),
              torch.as_tensor(uy, device=dev), fa)
    fb = torch.empty_like(fa)
    r, u, v = (torch.empty(n, dtype=torch.float64, device=dev) for _ in range(3))
    stream = torch.cuda.current_stream(dev)
    bufs = [fa, fb]

    def one(i):
        R.lbm_stream_collide(k, ja, W, 1.5, bufs[i % 2], bufs[(i + 1) % 2], r, u, v,
                             stream=stream)
    for i in range(3):
        one(i)
    torch.cuda.synchronize()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    for i in range(steps):
        one(i)
    eb.record(stream)
    torch.cuda.synchronize()
    ms = ea.elapsed_time(eb) / steps
    pk, src = peaks()
    gbs = lbm_bytes_per_node(k) * n / (ms * 1e-3) / 1e9
    out = {"workload": f"D2Q9 semi-Lagrangian LBM, periodic {m}x{m} jittered grid, k={k} "
                       "interpolation operators (r^3 + degree 2) at the 8 departure points "
                       "x - c_a h/2, FP64, fused stream + BGK collide per step",
           "nodes": n, "ms_per_step": ms, "node_updates_per_s": n / (ms * 1e-3),
           "operator_assembly_ms": st["ms"],
           "hbm": {"bytes_per_node": lbm_bytes_per_node(k), "achieved_gbs": gbs,
                   "peak_gbs": pk.get("hbm_gbs"), "frac": gbs / pk.get("hbm_gbs"),
                   "peak_source": src}}
    del W, vals, fa, fb, ja
    torch.cuda.synchronize()
    return out


def serve_sample(R, NS, device, count, form="fp64", repeats=3):
    """The serving configuration: `count` requests (sizes log-uniform in
    [1e3, 5e5], square or disk, k in {21, 35, 64} with degree {2, 3, 4})
    admitted under a 40 GB HBM budget, in the faster form.

    1. serial: plain FP64 assembly of the requests one after another (host
       in, host out) -- the reference point;
    2. capacity: after an untimed warm-up on the first 100 requests, all
       requests submitted at once; completed stencils / time;
    3. latency: Poisson arrivals at 80% of that capacity (the GPU ~80% busy),
       p50/p99 of submit -> device completion, `repeats` times; once more at
       50% of capacity."""
    reqs = NS.serving_requests(count, seed=5)
    nodes = [NS.request_nodes(r) for r in reqs]
    total = sum(r["n"] for r in reqs)
    prec = R.FP64 if form == "fp64" else R.FP32_IR
    ctx = R.Context(device)
    for r, (x, y) in list(zip(reqs, nodes))[:20]:  # warm-up: library, pinned staging
        ctx.assemble_host(R.make_desc(r["P"], precision=R.FP64), x, y, r["k"],
                          [np.empty(r["n"] * r["k"]) for _ in range(3)])
    t0 = time.perf_counter()
    for r, (x, y) in zip(reqs, nodes):
        vals = [np.empty(r["n"] * r["k"]) for _ in range(3)]
        ctx.assemble_host(R.make_desc(r["P"], precision=R.FP64), x, y, r["k"], vals)
    serial_s = time.perf_counter() - t0
    ctx.close()
    srv = R.Server(device, hbm_budget=40 << 30, max_slots=8)

    def sweep(pending, lat, win):
        # release whatever has finished, in any order (the budget recycles)
        for t in list(pending):
            st, res = srv.poll(t, wait_ms=0)
            if st == R.EBUSY:
                continue
            if st != 0 or res.status != 0:
                raise RuntimeError(f"serving request failed: {st} {res.status}")
            lat.append(res.end_ms - res.submit_ms)
            win.append((res.dev_start_ms, res.dev_end_ms))
            srv.release(t)
            del pending[t]

    def run(rq, nd, gaps):
        """Submit request i at sum(gaps[:i+1]) seconds (all at once when
        gaps is None), releasing completed requests while waiting; returns
        (latencies, device windows, seconds from first submit to last
        completion)."""
        pending, lat, win = {}, [], []
        t0 = time.perf_counter()
        tnext = t0
        for i, (r, (x, y)) in enumerate(zip(rq, nd)):
            if gaps is not None:
                tnext += gaps[i]
                while time.perf_counter() < tnext:
                    sweep(pending, lat, win)
                    time.sleep(min(max(tnext - time.perf_counter(), 0.0), 0.0005))
            pending[srv.submit(x, y, r["k"], R.make_desc(r["P"], precision=prec))] = r
            sweep(pending, lat, win)
        deadline = time.perf_counter() + 600.0
        while pending and time.perf_counter() < deadline:
            sweep(pending, lat, win)
            time.sleep(0.0005)
        if pending:
            raise RuntimeError(f"{len(pending)} serving requests did not finish")
        return np.array(lat), win, time.perf_counter() - t0

    warm = min(len(reqs), 100)
    run(reqs[:warm], nodes[:warm], None)
    _, win_b, burst_s = run(reqs, nodes, None)
    capacity = len(reqs) / burst_s
    # requests in flight together on the device (interval overlap)
    ev = sorted([(a, 1) for a, _ in win_b] + [(b, -1) for _, b in win_b])
    cur = peak = 0
    for _, dlt in ev:
        cur += dlt
        peak = max(peak, cur)
    gaps = np.array([r["gap"] for r in reqs])
    rate = 0.8 * capacity
    p50s, p99s, served = [], [], []
    for _ in range(repeats):
        lat, _, span = run(reqs, nodes, gaps / rate)
        p50s.append(float(np.percentile(lat, 50)))
        p99s.append(float(np.percentile(lat, 99)))
        served.append(total / span)
    lat50, _, _ = run(reqs, nodes, gaps / (0.5 * capacity))
    srv.close()
    return {"requests": len(reqs), "stencils": total, "form": form,
            "p50_ms": statistics.median(p50s), "p99_ms": statistics.median(p99s),
            "p50_ms_runs": p50s, "p99_ms_runs": p99s,
            "p50_spread_ms": max(p50s) - min(p50s), "p99_spread_ms": max(p99s) - min(p99s),
            "stencils_per_s": statistics.median(served), "capacity_stencils_per_s": total / burst_s,
            "serial_fp64_stencils_per_s": total / serial_s,
            "served_over_serial": statistics.median(served) / (total / serial_s),
            "max_requests_on_device_together": peak,
            "arrival_rate_per_s": rate,
            "at_50pct_load": {"p50_ms": float(np.percentile(lat50, 50)),
                              "p99_ms": float(np.percentile(lat50, 99))},
            "note": "Poisson arrivals at 80% of the measured burst capacity (medians of the "
                    "repeats); latency = submit to device completion; results released as "
                    "they complete (40 GB budget)"}


def pipe_peak_tflops(pipe):
    """CUDA-core peak of this GPU for the pipe the assembly is bound by: 2
    flops x (128 FP32 | 64 FP64) FMA lanes x SMs x max SM clock."""
    import torch
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    pk, _ = peaks()
    mhz = pk.get("sm_max_mhz") or 1965.0
    lanes = 128 if pipe == "fp32" else 64
    return 2 * lanes * props.multi_processor_count * mhz * 1e6 / 1e12, \
        f"nominal: 2 x {lanes} {pipe.upper()} FMA lanes x {props.multi_processor_count} SMs x {mhz:.0f} MHz"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-repeats", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip configurations 3-5 (headline only)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)

    from rbf_b200 import nodesets as NS
    ws, rank, local = dist_env()
    m = grid_side(ws)
    x, y, _ = NS.jittered_grid(m, 0.3, seed=2, periodic=True)
    n_all = x.size
    cpu_base = None
    if ws == 1 and not args.no_cpu:  # the host-core baseline, before any CUDA work
        cpu_base = cpu_baseline_full(x, y)

    import torch
    import oracle as O
    import rbf_b200 as R
    from rbf_b200 import shard as SH

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    dev = torch.device("cuda", local)
    xd = torch.as_tensor(x, device=dev)
    yd = torch.as_tensor(y, device=dev)
    if dist is not None:
        SH.replicate_nodes(xd, yd, src=0)  # the one exchange: 16 B per node
    first, n = SH.node_range(n_all, ws, rank)
    nk = n * K
    ja = torch.empty(nk, dtype=torch.int32, device=dev)
    vals = [torch.empty(nk, dtype=torch.float64, device=dev) for _ in range(NRHS)]
    info = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    per = (1.0, 1.0)
    ctx = R.Context(local)
    d_mix = R.make_desc(P, Q, R.DEFAULT_OPS, R.FP32_IR, True, period=per)
    d_f64 = R.make_desc(P, Q, R.DEFAULT_OPS, R.FP64, True, period=per)
    xq = xd[first:first + n].contiguous()  # this rank's stencil centres
    yq = yd[first:first + n].contiguous()

    def knn():
        if ws == 1:
            ctx.knn_stencils(xd, yd, K, ja, period=per, stream=stream)
        else:  # this rank's stencils against the whole node set
            ctx.knn_query(xd, yd, xq, yq, K, ja, period=per, stream=stream)

    def assemble(desc, stats=False):
        if ws == 1:
            return ctx.assemble(desc, xd, yd, K, ja, vals, info, stats=stats, stream=stream)
        return ctx.assemble_range(desc, first, n, xd, yd, K, ja, vals, info, stats=stats,
                                  stream=stream)

    # project autotuner: kernel shape and CTAs per SM for both precisions
    knn()
    # (N = 1; under torchrun every rank keeps the default shapes, so all agree)
    tuned = {}
    if ws == 1:
        for nm, dsc in (("mixed", d_mix), ("fp64", d_f64)):
            tuned[nm] = R.variant_name(ctx.autotune(dsc, xd, yd, K, ja, vals))

    def step(desc, stats=False):
        knn()
        return assemble(desc, stats)

    def timed(desc, steps, warmup):
        for _ in range(warmup):
            step(desc)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        l0 = ctx.launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(desc)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms), ctx.launches() - l0

    # ---- correctness of this run against the FP64 oracle on a sample
    st_mix = step(d_mix, stats=True)
    torch.cuda.synchronize()
    ja_h = ja.cpu().numpy()
    rows = np.random.default_rng(1).choice(n, 2048, replace=False)
    idx = (rows[:, None] * K + np.arange(K)[None, :]).ravel()
    W_mix = np.stack([v.cpu().numpy()[idx] for v in vals])
    step(d_f64)
    torch.cuda.synchronize()
    W_64 = np.stack([v.cpu().numpy()[idx] for v in vals])
    err_mix = err_64 = None
    if rank == 0:  # the checker: rank 0 reports it, so rank 0 alone runs it
        O.set_threads(os.cpu_count() or 1)
        ia_h = np.arange(n + 1, dtype=np.int64) * K
        Wo, _ = sampled_oracle(O, x, y, ia_h, ja_h, rows, P_=P, Q_=Q, period=per,
                               centres=rows + first)
        err_mix = float(O.max_rel_err(W_mix, Wo, K).max())
        err_64 = float(O.max_rel_err(W_64, Wo, K).max())

    # ---- timed: FP64 and mixed on the same node set
    with Clocks(local) as clk:
        ms_64, launches = timed(d_f64, args.steps, args.warmup)
        ms_mix, _ = timed(d_mix, args.steps, args.warmup)
    # dominant kernel alone: the assembly (k-NN excluded), CUDA events on its stream
    reps = 5

    def stage_ms(fn):
        fn()
        torch.cuda.synchronize()
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        for _ in range(reps):
            fn()
        eb.record(stream)
        torch.cuda.synchronize()
        return ea.elapsed_time(eb) / reps

    ms_asm = stage_ms(lambda: assemble(d_mix))
    ms_knn = stage_ms(knn)
    ms_asm64 = stage_ms(lambda: assemble(d_f64))

    # ---- end to end through the host-buffer entry point (pinned host memory)
    e2e = None
    d_head = d_f64 if ms_64 <= ms_mix else d_mix  # the faster form (both meet the bound here)
    if ws == 1:
        xh = torch.from_numpy(x).pin_memory()
        yh = torch.from_numpy(y).pin_memory()
        vh = [torch.empty(nk, dtype=torch.float64).pin_memory() for _ in range(NRHS)]
        jh = torch.empty(nk, dtype=torch.int32).pin_memory()
        e2e_steps = max(3, args.steps // 2)
        for _ in range(2):
            ctx.assemble_host(d_head, xh, yh, K, vh, ja_out_h=jh)
        t0 = time.perf_counter()
        e2e_dev_ms = 0.0
        for _ in range(e2e_steps):
            st = ctx.assemble_host(d_head, xh, yh, K, vh, ja_out_h=jh)
            e2e_dev_ms += st["ms"]
        t1 = time.perf_counter()
        e2e_ms = 1e3 * (t1 - t0) / e2e_steps
        e2e = {"value": n / (e2e_ms * 1e-3), "unit": "stencils/s",
               "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": nk * (8 * NRHS + 4),
               "device_ms": e2e_dev_ms / e2e_steps,
               "form": "fp64" if d_head is d_f64 else "mixed"}
        del xh, yh, vh, jh

    # ---- configurations 3-5 (N = 1 only: single-GPU measurements)
    configs = None
    if ws == 1 and not args.no_configs:
        del vals, ja, info
        torch.cuda.synchronize()
        configs = {"c3": config3(R, O, torch, ctx, dev), "c4": config4(R, O, NS, torch, ctx, dev),
                   "lbm": config_lbm(R, NS, torch, ctx, dev)}
        if args.serve_requests > 0:
            configs["c5"] = serve_sample(R, NS, local, args.serve_requests,
                                         "fp64" if d_head is d_f64 else "mixed",
                                         args.serve_repeats)

    if rank != 0:
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0
    pk, src = peaks()
    flops = FLOP_PER_STENCIL * n
    fp32_peak, fp32_src = pipe_peak_tflops("fp32")
    # headline: the faster of the two forms that meet the 1e-10 bound
    ok = {"mixed": err_mix <= 1e-10, "fp64": err_64 <= 1e-10}
    rate = {"mixed": n / (ms_mix * 1e-3), "fp64": n / (ms_64 * 1e-3)}
    form = max((f for f in ("mixed", "fp64") if ok[f]), key=lambda f: rate[f], default="fp64")
    ms_head = ms_mix if form == "mixed" else ms_64
    ms_kernel = ms_asm if form == "mixed" else ms_asm64
    pipe = "fp32" if form == "mixed" else "fp64"
    peak_pipe, peak_src = pipe_peak_tflops(pipe)
    achieved = flops / (ms_kernel * 1e-3) / 1e12
    line = {
        "metric": METRIC,
        "value": ws * n / (ms_head * 1e-3),
        "unit": "stencils/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_head,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if form == "fp64" else "f32+f64",
        "data": "synthetic (seeded jittered grid, numpy default_rng)",
        "config": {"workload": f"periodic {m}x{m} jittered grid (+-0.3h), k={K} k-NN + "
                               f"assembly, PHS r^{Q} + degree {P} (n={N_SYS}), Laplacian/dx/dy"
                               + ("" if ws == 1 else f", one node set split into {ws} "
                                                     "contiguous node ranges"),
                   "stencils_per_gpu": n, "l2": "inputs and outputs > L2 every step",
                   "form": form,
                   "forms": {"fp64": "FP64 fill + FP64 elimination (bit-identical to the oracle)",
                             "mixed": "FP32 elimination + FP64 residual refinement, FP64 "
                                      "fallback per stencil"}},
        "mixed": {"stencils_per_s": ws * rate["mixed"], "ms_per_step": ms_mix,
                  "asm_ms": ms_asm, "max_rel_weight_err": err_mix,
                  "fallback_stencils": st_mix["fallback"] if st_mix else None,
                  "sweeps_mean": (st_mix["sweeps"] / max(1, n)) if st_mix else None,
                  # the refined form against the FP32 pipe it factorises on
                  # (algorithmic flops; sweeps and fallbacks not counted)
                  "roofline_fp32": {"achieved": FLOP_PER_STENCIL * n / (ms_asm * 1e-3) / 1e12,
                                    "peak": fp32_peak, "unit": "TFLOP/s",
                                    "frac": FLOP_PER_STENCIL * n / (ms_asm * 1e-3) / 1e12
                                    / fp32_peak, "peak_source": fp32_src}},
        "fp64": {"stencils_per_s": ws * rate["fp64"], "ms_per_step": ms_64, "asm_ms": ms_asm64,
                 "max_rel_weight_err": err_64},
        "mixed_over_fp64": ms_64 / ms_mix,
        "max_rel_weight_err_vs": "FP64 CPU oracle, 2048 sampled stencils",
        "stages_ms": {"knn": ms_knn, "assembly_mixed": ms_asm, "assembly_fp64": ms_asm64},
        "gpu_launches": launches,
        "kernel_shapes": tuned,
        "roofline": {"bound": pipe, "achieved": achieved, "peak": peak_pipe,
                     "unit": "TFLOP/s", "frac": achieved / peak_pipe,
                     "traffic": traffic_per_launch(form),
                     "peak_source": peak_src,
                     "kernel": f"assembly ({form}), k-NN excluded",
                     "flop_per_stencil": FLOP_PER_STENCIL,
                     "hbm": {"algorithmic_bytes": n * HBM_BYTES_PER_STENCIL,
                             "bytes_per_stencil": HBM_BYTES_PER_STENCIL,
                             "compulsory_bytes_per_stencil": HBM_COMPULSORY_PER_STENCIL,
                             "achieved_gbs": n * HBM_BYTES_PER_STENCIL / (ms_kernel * 1e-3) / 1e9,
                             "peak_gbs": pk.get("hbm_gbs"), "peak_source": src}},
        "clocks": clk.summary(),
    }
    if e2e is not None:
        line["e2e"] = e2e
    if configs is not None:
        line["configs"] = configs
    if cpu_base is not None:
        line["cpu_baseline"] = cpu_base
    print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
