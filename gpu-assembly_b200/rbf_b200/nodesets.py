"""Seeded synthetic node sets with the shapes of the assembly workloads.

The reference measures on its own node files (``data/*.node``) and on clouds
made by its Python tooling (``data/pointclouds/generators.py``: the perturbed
grid of ``PerturbedGrid`` at :556-630, the disk of ``Disk`` at :27-157). There
is no public dataset; these generators stand in for it, seeded with
``numpy.random.default_rng`` so every machine builds the same nodes.

All node sets are returned as ``(x, y, flag)`` float64 / float64 / int32
arrays; flag 1 marks boundary nodes (the reference's boundary marker).
"""
from __future__ import annotations

import math

import numpy as np


def jittered_grid(m: int, jitter: float = 0.3, seed: int = 1, periodic: bool = False):
    """m x m grid on [0,1]^2 with spacing h = 1/m, nodes at (i+1/2)h, each
    coordinate moved by U(-jitter, jitter)*h. Row by row, x fastest. All
    nodes stay inside (0,1) for jitter < 0.5, so the periodic variant needs
    no wrapping; the flag is 0 everywhere."""
    h = 1.0 / m
    g = (np.arange(m, dtype=np.float64) + 0.5) * h
    xv, yv = np.meshgrid(g, g)
    rng = np.random.default_rng(seed)
    d = rng.uniform(-jitter, jitter, size=(2, m * m)) * h
    x = xv.ravel() + d[0]
    y = yv.ravel() + d[1]
    return x, y, np.zeros(m * m, np.int32)


def unit_disk(n: int, nb: int = 8192, seed: int = 3, jitter: float = 0.3):
    """n nodes on the unit disk: nb equispaced boundary nodes on r = 1
    (first, flag 1, the Disk generator's order) and n - nb interior nodes
    from a jittered grid clipped to r < 1 - h/2. The grid spacing is chosen
    so that slightly more than n - nb interior nodes fall inside; the
    outermost surplus (by radius, then index) is dropped."""
    ni = n - nb
    t = 2.0 * np.pi * np.arange(nb) / nb
    xb, yb = np.cos(t), np.sin(t)
    h = math.sqrt(math.pi / ni) * 0.995
    rng = np.random.default_rng(seed)
    while True:
        m = int(math.ceil(2.0 / h)) + 2
        g = -1.0 + (np.arange(m) + 0.5) * (2.0 / m)
        hh = 2.0 / m
        xv, yv = np.meshgrid(g, g)
        d = rng.uniform(-jitter, jitter, size=(2, m * m)) * hh
        xi = xv.ravel() + d[0]
        yi = yv.ravel() + d[1]
        r = np.hypot(xi, yi)
        keep = r < 1.0 - 0.5 * hh
        if keep.sum() >= ni:
            break
        h *= 0.99
    xi, yi, r = xi[keep], yi[keep], r[keep]
    order = np.lexsort((np.arange(r.size), r))[:ni]
    order.sort()
    x = np.concatenate([xb, xi[order]])
    y = np.concatenate([yb, yi[order]])
    flag = np.zeros(n, np.int32)
    flag[:nb] = 1
    return x, y, flag


def gaussian_bump(n: int, seed: int = 4, sigma: float = 0.15, ratio: float = 4.0,
                  centre=(0.5, 0.5), jitter: float = 0.3):
    """n nodes on [0,1]^2 with density proportional to
    1 + (ratio-1) exp(-|x-c|^2 / (2 sigma^2)): a jittered grid fine enough
    for the peak density, thinned by seeded rejection, then trimmed to n."""
    area = 1.0 + (ratio - 1.0) * 2.0 * math.pi * sigma * sigma
    mean_keep = area / ratio
    m = int(math.ceil(math.sqrt(n / mean_keep * 1.02)))
    rng = np.random.default_rng(seed)
    while True:
        h = 1.0 / m
        g = (np.arange(m) + 0.5) * h
        xv, yv = np.meshgrid(g, g)
        d = rng.uniform(-jitter, jitter, size=(2, m * m)) * h
        x = xv.ravel() + d[0]
        y = yv.ravel() + d[1]
        rho = 1.0 + (ratio - 1.0) * np.exp(-((x - centre[0]) ** 2 + (y - centre[1]) ** 2)
                                           / (2 * sigma * sigma))
        keep = rng.uniform(size=x.size) * ratio < rho
        if keep.sum() >= n:
            break
        m += max(1, m // 100)
    idx = np.flatnonzero(keep)
    drop = rng.choice(idx.size, size=idx.size - n, replace=False)
    mask = np.ones(idx.size, bool)
    mask[drop] = False
    idx = idx[mask]
    return x[idx], y[idx], np.zeros(n, np.int32)


def read_node_file(path):
    """A Triangle .node file: header 'n dim nattr nmarker', then
    'index x y [attrs] [marker]' lines; '#' starts a comment."""
    rows = []
    header = None
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            vals = line.split()
            if header is None:
                header = [int(v) for v in vals[:4]]
                continue
            rows.append(vals)
    n, _, nattr, nmark = header
    x = np.array([float(r[1]) for r in rows[:n]])
    y = np.array([float(r[2]) for r in rows[:n]])
    flag = (np.array([int(r[3 + nattr]) for r in rows[:n]], np.int32) if nmark
            else np.zeros(n, np.int32))
    return x, y, flag


# ---- the workloads ---------------------------------------------------------

def config_small(seed: int = 1):
    """Plain FP64, CPU-runnable: jittered 69x69 grid on [0,1]^2 (4,761 nodes),
    k=21, r^3 + degree 2, open plane."""
    x, y, f = jittered_grid(69, 0.3, seed)
    return dict(x=x, y=y, flag=f, k=21, P=2, Q=3, period=None, name="square69_k21_p2")


def config_periodic(m: int = 1024, seed: int = 2):
    """Single large node set: jittered m x m grid on the periodic unit
    square (m=1024: 1,048,576 nodes), k=35, r^5 + degree 3."""
    x, y, f = jittered_grid(m, 0.3, seed, periodic=True)
    return dict(x=x, y=y, flag=f, k=35, P=3, Q=5, period=(1.0, 1.0),
                name=f"periodic{m}x{m}_k35_p3")


def config_disk_uneven(n: int = 4194304, nb: int = 8192, seed: int = 3):
    """Uneven batch: unit disk, nb boundary nodes with k in [48, 64] and
    degree 4, interior nodes with k in {21, 28, 35} (degree 2 for k < 28,
    else 3). Q = 2P - 1. Returns per-node k and degree arrays."""
    x, y, f = unit_disk(n, nb, seed)
    rng = np.random.default_rng(seed + 1000)
    k = rng.choice(np.array([21, 28, 35], np.int32), size=n)
    k[:nb] = rng.integers(48, 65, size=nb)
    deg = np.where(k < 28, 2, 3).astype(np.int8)
    deg[:nb] = 4
    return dict(x=x, y=y, flag=f, kvec=k.astype(np.int32), degree=deg, period=None,
                name=f"disk{n}_uneven")


def config_bump(n: int = 2097152, seed: int = 4):
    """High-order stress: Gaussian-bump density on [0,1]^2 (4x ratio),
    k=64, r^7 + degree 4."""
    x, y, f = gaussian_bump(n, seed)
    return dict(x=x, y=y, flag=f, k=64, P=4, Q=7, period=None, name=f"bump{n}_k64_p4")


def serving_requests(count: int = 2000, seed: int = 5, nmin: float = 1e3, nmax: float = 5e5):
    """Request stream: sizes log-uniform in [nmin, nmax], square (jittered
    grid) or disk with probability 1/2, k from {21, 35, 64} with degree
    {2, 3, 4}; arrival gaps are exponential (Poisson process, unit mean,
    scaled by the caller)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count)).astype(np.int64)
    geo = rng.integers(0, 2, size=count)
    kk = rng.integers(0, 3, size=count)
    gaps = rng.exponential(1.0, size=count)
    reqs = []
    for i in range(count):
        k = (21, 35, 64)[kk[i]]
        P = (2, 3, 4)[kk[i]]
        reqs.append(dict(n=int(max(sizes[i], 2 * k)), geometry="square" if geo[i] == 0 else "disk",
                         k=k, P=P, Q=2 * P - 1, seed=int(seed * 100003 + i), gap=float(gaps[i])))
    return reqs


def request_nodes(req):
    """Node coordinates of one serving request."""
    n = req["n"]
    if req["geometry"] == "square":
        m = int(math.ceil(math.sqrt(n)))
        x, y, _ = jittered_grid(m, 0.3, req["seed"])
        return x[:n].copy(), y[:n].copy()
    nb = max(16, int(2 * math.sqrt(n)))
    x, y, _ = unit_disk(n, nb, req["seed"])
    return x, y
