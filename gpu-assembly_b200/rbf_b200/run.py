"""Runs the hot path on one periodic jittered grid: k-NN stencils once, then
the assembly `--reps` times in one precision. Prints one JSON line with the
device time per assembly (CUDA events) and the call's counters.

    python -m rbf_b200.run --grid 256 --precision mixed --reps 3

Used to profile a single kernel shape on a small case (e.g. under ncu with
``-k regex:asm_kernel``); the workload is the benchmark's at a smaller size.
"""
from __future__ import annotations

import argparse
import json

import torch

import rbf_b200 as R
from rbf_b200 import nodesets as NS


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--k", type=int, default=35)
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tune", action="store_true", help="autotune the shape first")
    a = ap.parse_args(argv)
    x, y, _ = NS.jittered_grid(a.grid, 0.3, seed=2, periodic=True)
    n, k = x.size, a.k
    dev = torch.device("cuda", 0)
    xd, yd = torch.as_tensor(x, device=dev), torch.as_tensor(y, device=dev)
    ja = torch.empty(n * k, dtype=torch.int32, device=dev)
    vals = [torch.empty(n * k, dtype=torch.float64, device=dev) for _ in range(3)]
    info = torch.empty(n, dtype=torch.int32, device=dev)
    per = (1.0, 1.0)
    prec = R.FP64 if a.precision == "fp64" else R.FP32_IR
    d = R.make_desc(a.degree, 0, R.DEFAULT_OPS, prec, True, period=per)
    with R.Context(0) as ctx:
        ctx.knn_stencils(xd, yd, k, ja, period=per)
        shape = None
        if a.tune:
            shape = R.variant_name(ctx.autotune(d, xd, yd, k, ja, vals))
        ms = []
        st = None
        for _ in range(a.reps):
            st = ctx.assemble(d, xd, yd, k, ja, vals, info, stats=True)
            ms.append(st["ms"])
        torch.cuda.synchronize()
        print(json.dumps({"grid": a.grid, "stencils": n, "precision": a.precision,
                          "shape": shape, "ms": ms, "stats": st}))


if __name__ == "__main__":
    main()
