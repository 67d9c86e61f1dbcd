"""The multi-process split on CPU (gloo, world size 2): node ranges cover the
node set exactly once, coordinates replicate from rank 0, each rank's rows
(assembled here by the CPU oracle, standing in for a rank's GPU) gather into
exactly the single-process operator."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from rbf_b200 import shard


def test_node_ranges_partition():
    for n in (1, 2, 7, 4761, 1048576):
        for world in (1, 2, 3, 8):
            spans = [shard.node_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0
            for (f0, c0), (f1, _) in zip(spans, spans[1:]):
                assert f0 + c0 == f1
            assert sum(c for _, c in spans) == n
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    from conftest import ROOT
    for p in (ROOT / "oracle", ROOT / "gpu-assembly_b200"):
        sys.path.insert(0, str(p))
    import oracle as O
    from rbf_b200 import nodesets as NS
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        k, P = 21, 2
        if rank == 0:
            x, y, _ = NS.jittered_grid(40, 0.3, seed=12)
        else:
            x = np.zeros(1600)
            y = np.zeros(1600)
        xt, yt = torch.from_numpy(np.ascontiguousarray(x)), torch.from_numpy(np.ascontiguousarray(y))
        shard.replicate_nodes(xt, yt, src=0)
        x, y = xt.numpy(), yt.numpy()
        n = x.size
        first, count = shard.node_range(n, world, rank)
        # this rank's stencils and weights (the oracle stands in for its GPU)
        ja = O.knn_brute(x, y, k, xq=x[first:first + count], yq=y[first:first + count])
        order = np.concatenate([np.arange(first, first + count),
                                np.setdiff1d(np.arange(n), np.arange(first, first + count))])
        inv = np.empty(n, np.int64)
        inv[order] = np.arange(n)
        W, _ = O.assemble_csr(x[order], y[order], (np.arange(count + 1) * k).astype(np.int32),
                              inv[ja].astype(np.int32), P=P, nstencils=count)
        full_ja = shard.gather_rows(torch.from_numpy(ja.astype(np.int32)), n, k, world)
        full_w = [shard.gather_rows(torch.from_numpy(W[q].copy()), n, k, world) for q in range(3)]
        if rank == 0:
            out.put((full_ja.numpy(), np.stack([w.numpy() for w in full_w]), x, y))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_the_single_process_operator():
    import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ja, W, x, y = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    np.testing.assert_array_equal(ja, O.knn_brute(x, y, 21))
    W1, _ = O.assemble(x, y, ja, 21, 2)
    np.testing.assert_array_equal(W, W1)
