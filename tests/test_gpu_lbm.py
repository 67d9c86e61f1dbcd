"""D2Q9 lattice Boltzmann kernels on the GPU, through the C ABI.

* feq / macros / BGK (src/lbm/d2q9_kernels.cu:13-150), float and double:
  bit-identical to the oracle's CPU restatement and, where the reference's
  own kernels were built here (oracle/_ref/ref_lbm_run, compiled without
  contraction), to the reference's kernels run on the same inputs by that
  program, a process of its own.
* the fused streaming + collision step through interpolation operators
  assembled by this library at the 8 departure points x_s - c_a dt: bit-
  identical to the oracle's restatement of its summation order on every
  path of the kernel (k = 21 fixed at compile time; other odd k; even k,
  padded rows; n*k odd, 8-byte copies); a uniform flow stays uniform.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import rbf_b200 as R
from rbf_b200 import nodesets as NS

pytestmark = pytest.mark.gpu


def _state(T, n, dtype, seed=0):
    rng = np.random.default_rng(seed)
    rho = (1.0 + 0.05 * rng.standard_normal(n)).astype(dtype)
    ux = (0.05 * rng.standard_normal(n)).astype(dtype)
    uy = (0.05 * rng.standard_normal(n)).astype(dtype)
    return rho, ux, uy


def _dev(T, a):
    return T.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_collision_kernels_match_oracle_and_reference(torch_cuda, dtype):
    T = torch_cuda
    n = 100_003  # not a multiple of the block
    rho, ux, uy = _state(T, n, dtype)
    rd, ud, vd = _dev(T, rho), _dev(T, ux), _dev(T, uy)
    pdf = T.empty(9 * n, dtype=rd.dtype, device="cuda")
    R.lbm_feq(rd, ud, vd, pdf)
    T.cuda.synchronize()
    feq = O.lbm_feq(rho, ux, uy)
    np.testing.assert_array_equal(pdf.cpu().numpy(), feq)
    # perturb, then moments and collision (both bgk forms)
    pert = (feq * (1.0 + 0.01 * np.random.default_rng(1).standard_normal(9 * n))).astype(dtype)
    pdf.copy_(_dev(T, pert))
    r2, u2, v2 = (T.empty_like(rd) for _ in range(3))
    R.lbm_macros(pdf, r2, u2, v2)
    T.cuda.synchronize()
    mo = O.lbm_macros(pert)
    for got, want in zip((r2, u2, v2), mo):
        np.testing.assert_array_equal(got.cpu().numpy(), want)
    indp = T.empty_like(rd)
    R.lbm_bgk(1.7, pdf, r2, u2, v2, indp)
    T.cuda.synchronize()
    post, ro, uo, vo, io = O.lbm_bgk(pert, 1.7)
    np.testing.assert_array_equal(pdf.cpu().numpy(), post)
    for got, want in zip((r2, u2, v2, indp), (ro, uo, vo, io)):
        np.testing.assert_array_equal(got.cpu().numpy(), want)
    pdf.copy_(_dev(T, pert))
    R.lbm_bgk(1.7, pdf, r2, u2, v2)  # bgk_kernel: no indp
    T.cuda.synchronize()
    np.testing.assert_array_equal(pdf.cpu().numpy(), post)
    # the reference's own kernels, run by a program of their own (nothing of
    # the reference loads into this process)
    ref = _reference_kernels(dtype, rho, ux, uy, pert, 1.7)
    if ref is None:
        return
    np.testing.assert_array_equal(ref["feq"], feq)
    np.testing.assert_array_equal(ref["post"], post)
    for nm, want in zip(("rho", "ux", "uy", "indp"), (ro, uo, vo, io)):
        np.testing.assert_array_equal(ref[nm], want)
    for nm, want in zip(("rho2", "ux2", "uy2"), O.lbm_macros(post)):
        np.testing.assert_array_equal(ref[nm], want)


def _reference_kernels(dtype, rho, ux, uy, pert, omega):
    """The reference's feq / bgk_kernel_split / macros kernels run on the
    given state by oracle/_ref/ref_lbm_run, a process of its own: their
    outputs, or None when the runner was not built here."""
    import subprocess
    import tempfile
    exe = Path(O.__file__).parent / "_ref" / "ref_lbm_run"
    if not exe.exists():
        return None
    n = rho.size
    with tempfile.TemporaryDirectory() as d:
        for nm, a in (("rho", rho), ("ux", ux), ("uy", uy), ("pert", pert)):
            np.ascontiguousarray(a, dtype=dtype).tofile(f"{d}/{nm}.bin")
        prec = 0 if dtype == np.float64 else 1
        r = subprocess.run([str(exe), d, str(n), str(prec), repr(float(omega))],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr[-3000:]
        out = {}
        for nm in ("feq", "post", "rho", "ux", "uy", "indp", "rho2", "ux2", "uy2"):
            out[nm] = np.fromfile(f"{d}/{nm}.bin", dtype=dtype)
        return out


def _streaming_operators(T, ctx, m=48, k=21, seed=3):
    """Interpolation operators of a periodic m x m jittered grid at the 8
    departure points x - c_a dt, dt = h/2: (ja, W (8*n*k), x, y)."""
    x, y, _ = NS.jittered_grid(m, 0.3, seed=seed, periodic=True)
    n = x.size
    xd, yd = _dev(T, x), _dev(T, y)
    ja = T.empty(n * k, dtype=T.int32, device="cuda")
    ctx.knn_stencils(xd, yd, k, ja, period=(1.0, 1.0))
    xc, yc = R.lbm_departure_points(0.5 / m)
    xcd, ycd = _dev(T, xc), _dev(T, yc)
    W = T.empty(8 * n * k, dtype=T.float64, device="cuda")
    vals = [W[a * n * k:(a + 1) * n * k] for a in range(8)]
    d = R.make_desc(2, 3, R.OP_INTERP, R.FP64, True, period=(1.0, 1.0), xc=xcd, yc=ycd, nc=8)
    st = ctx.assemble(d, xd, yd, k, ja, vals, stats=True)
    assert st["singular"] == 0
    T.cuda.synchronize()
    return ja, W, x, y


# (grid side, k): k = 21 with 16-byte copies; n*k odd (47^2 * 21): 8-byte
# copies; k = 15: odd k not fixed at compile time; k = 16: padded rows
@pytest.mark.parametrize("mk", [(48, 21), (47, 21), (48, 15), (48, 16)], ids=str)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_stream_collide_matches_oracle(ctx, torch_cuda, dtype, mk):
    T = torch_cuda
    m, k = mk
    ja, W, x, y = _streaming_operators(T, ctx, m=m, k=k)
    n = x.size
    rho = (1.0 + 0.02 * np.sin(2 * np.pi * x)).astype(dtype)
    ux = (0.03 * np.cos(2 * np.pi * y)).astype(dtype)
    uy = (0.01 * np.sin(2 * np.pi * (x + y))).astype(dtype)
    f0 = O.lbm_feq(rho, ux, uy)
    fin = _dev(T, f0)
    fout = T.empty_like(fin)
    r, u, v = (T.empty(n, dtype=fin.dtype, device="cuda") for _ in range(3))
    R.lbm_stream_collide(k, ja, W, 1.2, fin, fout, r, u, v)
    T.cuda.synchronize()
    out, ro, uo, vo = O.lbm_stream_collide(k, ja.cpu().numpy(), W.cpu().numpy(), 1.2, f0)
    np.testing.assert_array_equal(fout.cpu().numpy(), out)
    for got, want in zip((r, u, v), (ro, uo, vo)):
        np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_uniform_flow_stays_uniform(ctx, torch_cuda):
    """Interpolation reproduces constants (degree-2 polynomial
    augmentation), so streaming a uniform equilibrium changes nothing and
    the collision keeps it: 20 steps stay at the start state to ~1e-12."""
    T = torch_cuda
    k = 21
    ja, W, x, y = _streaming_operators(T, ctx)
    n = x.size
    rho, ux, uy = np.full(n, 1.0), np.full(n, 0.04), np.full(n, -0.02)
    f0 = O.lbm_feq(rho, ux, uy)
    a, b = _dev(T, f0), T.empty(9 * n, dtype=T.float64, device="cuda")
    for _ in range(20):
        R.lbm_stream_collide(k, ja, W, 1.5, a, b)
        a, b = b, a
    T.cuda.synchronize()
    np.testing.assert_allclose(a.cpu().numpy(), f0, rtol=0, atol=1e-12)


def test_stream_collide_argument_checks(torch_cuda):
    T = torch_cuda
    f = T.zeros(9 * 10, dtype=T.float64, device="cuda")
    ja = T.zeros(10 * 3, dtype=T.int32, device="cuda")
    W = T.zeros(8 * 30, dtype=T.float64, device="cuda")
    with pytest.raises(R.RbfError):
        R.lbm_stream_collide(3, ja, W, 1.0, f, f)  # in place is not allowed
    with pytest.raises(R.RbfError):
        R.lbm_stream_collide(65, ja, W, 1.0, f, T.empty_like(f))  # k above 64
