"""The oracle's restatement of the reference's D2Q9 kernels
(src/lbm/d2q9_kernels.cu:13-150): the lattice's own identities, which the
reference's arithmetic keeps to rounding, and the exact ones it keeps bit for
bit (the BGK step at omega = 1 is the equilibrium of the moments)."""
import numpy as np
import pytest

import oracle as O


def _state(n, dtype, seed=0):
    rng = np.random.default_rng(seed)
    rho = (1.0 + 0.05 * rng.standard_normal(n)).astype(dtype)
    ux = (0.05 * rng.standard_normal(n)).astype(dtype)
    uy = (0.05 * rng.standard_normal(n)).astype(dtype)
    return rho, ux, uy


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-14), (np.float32, 2e-6)])
def test_equilibrium_moments(dtype, tol):
    rho, ux, uy = _state(1000, dtype)
    pdf = O.lbm_feq(rho, ux, uy)
    r, u, v = O.lbm_macros(pdf)
    np.testing.assert_allclose(r, rho, rtol=tol)
    np.testing.assert_allclose(u, ux, atol=tol)
    np.testing.assert_allclose(v, uy, atol=tol)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-14), (np.float32, 2e-6)])
def test_bgk_conserves_mass_and_momentum(dtype, tol):
    rho, ux, uy = _state(1000, dtype, 1)
    rng = np.random.default_rng(2)
    pdf = O.lbm_feq(rho, ux, uy) * (1.0 + 0.01 * rng.standard_normal(9000)).astype(dtype)
    r0, u0, v0 = O.lbm_macros(pdf)
    post, r, u, v, indp = O.lbm_bgk(pdf, 1.3)
    np.testing.assert_array_equal(r, r0)  # bgk reports the pre-collision moments
    r1, u1, v1 = O.lbm_macros(post)
    np.testing.assert_allclose(r1, r0, rtol=tol)
    np.testing.assert_allclose(r1 * u1, r0 * u0, atol=tol)
    np.testing.assert_allclose(r1 * v1, r0 * v0, atol=tol)
    np.testing.assert_allclose(indp, 1.0 / 3.0 - 0.5 * (u0 * u0 + v0 * v0), rtol=tol)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_bgk_at_omega_one_is_the_equilibrium(dtype):
    rho, ux, uy = _state(500, dtype, 3)
    rng = np.random.default_rng(4)
    pdf = O.lbm_feq(rho, ux, uy) * (1.0 + 0.01 * rng.standard_normal(4500)).astype(dtype)
    post, r, u, v, _ = O.lbm_bgk(pdf, 1.0)
    np.testing.assert_array_equal(post, O.lbm_feq(r, u, v))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_streaming_with_identity_operators(dtype):
    """Weights that take every population from its own node (departure
    point = the node) make the step a plain collision."""
    n, k = 300, 5
    rho, ux, uy = _state(n, dtype, 5)
    pdf = O.lbm_feq(rho, ux, uy) * (1.0 + 0.01 * np.random.default_rng(6).standard_normal(9 * n)
                                    ).astype(dtype)
    ja = np.stack([np.arange(n)] + [np.random.default_rng(7 + j).integers(0, n, n)
                                    for j in range(k - 1)], axis=1).astype(np.int32).ravel()
    W = np.zeros((8, n, k))
    W[:, :, 0] = 1.0
    out, r, u, v = O.lbm_stream_collide(k, ja, W.ravel(), 0.9, pdf)
    want = O.lbm_bgk(pdf, 0.9)
    np.testing.assert_array_equal(out, want[0])
    np.testing.assert_array_equal(r, want[1])
