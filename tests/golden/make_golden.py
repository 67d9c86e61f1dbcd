"""Regenerates the golden fixtures in tests/golden/ from the reference.

Run where a reference checkout is available (``--ref``, or the environment
variable ``RBFB_REFERENCE``) after ``make -C oracle`` has built the
reference's own stencil searches (oracle/_ref/libref_knn.so):

    RBFB_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Fixtures (numpy .npz, compressed):

* ``{poisson_32_21, poisson_32_64, cartesian_32_21}.npz`` -- the reference's
  own periodic k-NN known answers: ``data/<case>.points`` and
  ``data/<case>.graph`` (32 x 32 periodic box; the graph rows list each
  node's k nearest, self first), converted as they are.
* ``<node set>.npz`` for ``shu_square_4786``, ``barnett_disk_817`` and
  ``wright_square_hole_892`` -- the node file, plus the reference's own
  ``NodeSet::stencils(21)`` (nanoflann) and ``KdTree::knn_stencils(21)``
  (ckdtree, open plane) run on it.
* ``square69_k21.npz`` -- the seeded 69 x 69 jittered grid (4,761 nodes) with
  ``NodeSet::stencils(21)``; ``periodic64_k35.npz`` -- a seeded 64 x 64
  periodic jittered grid with the periodic ``KdTree::knn_stencils(35)``.
* ``weights_square69.npz`` / ``weights_shu.npz`` -- FP64 weights of the first
  200 stencils from the CPU oracle (Laplacian, d/dx, d/dy), so the oracle
  itself is pinned across machines and compilers.
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "gpu-assembly_b200"))

import oracle as O  # noqa: E402
from rbf_b200 import nodesets as NS  # noqa: E402


def read_points(path):
    lines = Path(path).read_text().split("\n")
    n = int(lines[0].split()[0])
    xy = np.array([[float(v) for v in lines[1 + i].split()[:2]] for i in range(n)])
    return xy[:, 0].copy(), xy[:, 1].copy()


def read_graph(path):
    lines = [ln for ln in Path(path).read_text().split("\n") if ln.strip()]
    n, nnz = (int(v) for v in lines[0].split()[:2])
    rows = [np.array(ln.split(), dtype=np.int32) for ln in lines[1:1 + n]]
    k = rows[0].size
    assert all(r.size == k for r in rows) and n * k == nnz
    return np.concatenate(rows), k


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("RBFB_REFERENCE"),
                    help="reference checkout (default: $RBFB_REFERENCE)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("give --ref or set RBFB_REFERENCE to the reference checkout")
    data = Path(a.ref) / "data"
    for case in ("poisson_32_21", "poisson_32_64", "cartesian_32_21"):
        x, y = read_points(data / f"{case}.points")
        ja, k = read_graph(data / f"{case}.graph")
        np.savez_compressed(HERE / f"{case}.npz", x=x, y=y, ja=ja, k=k, box=np.array([32.0, 32.0]))
        print(case, x.size, k)
    for case in ("shu_square_4786", "barnett_disk_817", "wright_square_hole_892"):
        x, y, flag = NS.read_node_file(data / f"{case}.node")
        ja_nf = O.ref_nodeset_stencils(x, y, 21)
        ja_kd = O.ref_kdtree_stencils(x, y, 21)
        np.savez_compressed(HERE / f"{case}.npz", x=x, y=y, flag=flag, k=21, ja_nanoflann=ja_nf,
                            ja_ckdtree=ja_kd)
        print(case, x.size, "nanoflann/ckdtree entries differing:", int((ja_nf != ja_kd).sum()))
    c = NS.config_small()
    ja = O.ref_nodeset_stencils(c["x"], c["y"], 21)
    np.savez_compressed(HERE / "square69_k21.npz", x=c["x"], y=c["y"], k=21, ja_nanoflann=ja)
    x, y, _ = NS.jittered_grid(64, 0.3, seed=7, periodic=True)
    ja = O.ref_kdtree_stencils(x, y, 35, period=(1.0, 1.0))
    np.savez_compressed(HERE / "periodic64_k35.npz", x=x, y=y, k=35, ja_ckdtree=ja,
                        box=np.array([1.0, 1.0]))
    # oracle weights on the first 200 stencils
    for name, (x, y, ja, k, P) in {
        "weights_square69": (c["x"], c["y"], np.load(HERE / "square69_k21.npz")["ja_nanoflann"], 21, 2),
        "weights_shu": (*NS.read_node_file(data / "shu_square_4786.node")[:2],
                        np.load(HERE / "shu_square_4786.npz")["ja_nanoflann"], 21, 2),
    }.items():
        W, info = O.assemble(x, y, ja, k, P)
        np.savez_compressed(HERE / f"{name}.npz", w=W[:, :200 * k], info=info[:200], k=k, P=P)
        print(name, W.shape)


if __name__ == "__main__":
    main()
