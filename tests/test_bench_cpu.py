"""bench.py pieces that run without a GPU: the algorithmic counts the
roofline uses, the traffic read from the committed ncu summary, and the
reference arm (the reference's CPU search + the CPU assembly), whose JSON
line must carry the contract's keys."""
import json
import subprocess
import sys

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_algorithmic_counts():
    n = bench.K + 10  # k + npoly(3)
    assert bench.N_SYS == n == 45
    assert bench.FLOP_PER_STENCIL == 2.0 / 3.0 * n ** 3 + 2 * 3 * n ** 2 == 72900.0
    assert bench.HBM_BYTES_PER_STENCIL == (4 + 16 + 24) * 35 + 16 == 1556
    assert bench.HBM_COMPULSORY_PER_STENCIL == (4 + 24) * 35 + 20 == 1000


def test_solve_byte_model():
    # one BiCGSTAB iteration: two operator passes (12 B per weight; row
    # pointer, flag, output and one gather per row) and the vector passes
    from rbf_b200 import run
    assert run.solve_bytes(1, 0) == 2 * (4 + 1 + 8) + 8 + 8 + 8 + 24 + 32 + 56 == 162
    assert run.solve_bytes(4194304, 117672830) == 24 * 117672830 + 162 * 4194304


def test_traffic_from_the_committed_profile():
    t = bench.traffic_per_launch("fp64")
    assert t is not None and 0.3e9 < t < 2e9  # DRAM bytes per full-size launch


def test_reference_arm_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["warmup"] >= 3  # the timing rules' minimum
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_sampled_oracle_matches_the_full_oracle():
    """bench.sampled_oracle renumbers the nodes so the sampled centres come
    first and assembles just those stencils: it must give the weights the
    full oracle gives for those stencils, also for ragged rows and for rows
    of a rank's range (centres offset from the rows)."""
    import numpy as np
    import oracle as O
    from rbf_b200 import nodesets as NS
    x, y, _ = NS.jittered_grid(24, 0.3, seed=3)
    n, k = x.size, 21
    ja = O.knn_brute(x, y, k)
    Wfull, _ = O.assemble(x, y, ja, k, 2)
    rows = np.array([5, 77, 300, 511])
    ia = np.arange(n + 1, dtype=np.int64) * k
    W, ia_s = bench.sampled_oracle(O, x, y, ia, ja, rows, P_=2, Q_=3)
    idx = (rows[:, None] * k + np.arange(k)[None, :]).ravel()
    np.testing.assert_array_equal(W, Wfull[:, idx])
    assert bench.ragged_rel_err(W, Wfull[:, idx], ia_s) == 0.0
    # a rank holding rows 100.. of the node set: local rows, global centres
    first = 100
    W2, _ = bench.sampled_oracle(O, x, y, ia[:n - first + 1], ja[first * k:], rows[:2], P_=2,
                                 Q_=3, centres=rows[:2] + first)
    idx2 = ((rows[:2] + first)[:, None] * k + np.arange(k)[None, :]).ravel()
    np.testing.assert_array_equal(W2, Wfull[:, idx2])


def test_lbm_byte_model():
    # ja row, 8 weight rows, 9 populations in and out, 3 moments out
    assert bench.lbm_bytes_per_node(21) == 4 * 21 + 64 * 21 + 72 + 72 + 24 == 1596
