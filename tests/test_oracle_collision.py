"""Known answers for the collision sampler and the collision integrators of
the oracle (CPU only): DeltatrackingCollisionSampler
(include/vr_collision_sampler_DT.h), MCCollisionIntegrator
(include/maps/collision_integrator_mc.h) and GridDDACollisionIntegrator
(include/vr_collision_integrator_DDA.h)."""
import math

import numpy as np
import pytest

import oracle
from rendervous_b200 import synthetic
from tests.helpers import homogeneous, oracle_desc

RAY_X = np.array([[-2.0, 0.013, -0.021, 1.0, 0.0, 0.0]], np.float32)  # crosses the unit box along x: d = 1


def test_collision_sampler_homogeneous(oracle_lib):
    """P(collision) = 1 - exp(-sigma d), E[t - tMin | collision] in closed form, T = 1 - C."""
    s = 2.0
    sc = oracle.OracleScene(oracle_desc(homogeneous(9, s)))
    n = 40000
    out = oracle.collision_sample_fw(sc, np.repeat(RAY_X, n, axis=0), 5)
    C, t, T = out[:, 0], out[:, 1], out[:, 2]
    p = 1 - math.exp(-s)
    assert abs(C.mean() - p) < 4 * math.sqrt(p * (1 - p) / n)
    assert np.array_equal(T, 1 - C)
    hit = t[C == 1] - 1.5                                  # tMin = 1.5
    mean_t = (1 - (1 + s) * math.exp(-s)) / (s * p)        # E[t | t < 1] of Exp(s)
    assert abs(hit.mean() - mean_t) < 4 * hit.std() / math.sqrt(hit.size)
    assert np.allclose(t[C == 0], 2.5, atol=1e-5)          # no collision: t runs to the exit


@pytest.mark.parametrize("integrator", ["mc_collision", "dda_collision"])
def test_collision_integrators_homogeneous_emission(oracle_lib, integrator):
    """Emission-absorption with constant emission e and environment B:
    E[R] = (1 - T) e + T B, T = exp(-sigma d) (the DDA form is exact per ray,
    up to its stop 1e-4 before the exit)."""
    s, e, B = 1.5, np.array([0.5, 1.0, 2.0]), 1.0
    sc = oracle.OracleScene(oracle_desc(homogeneous(9, s), emission=e, env=B, exitance_mode=0))
    n = 20000 if integrator == "mc_collision" else 16
    R, cnt = oracle.radiance_fw(sc, integrator, np.repeat(RAY_X, n, axis=0), 7)
    T = math.exp(-s)
    expect = (1 - T) * e + T * B
    if integrator == "dda_collision":
        assert np.abs(R - expect).max() < 4e-4
    else:
        se = R.std(axis=0) / math.sqrt(n)
        assert (np.abs(R.mean(axis=0) - expect) <= 4 * se + 1e-6).all(), (R.mean(axis=0), expect, se)
        assert abs(cnt["vertices"] / n - (1 - T)) < 4 * math.sqrt(T * (1 - T) / n)  # vertices = collisions


def test_dda_collision_adjoint_matches_finite_differences(oracle_lib):
    """L = sum_i w_i . R_i with the same cell draws (common random numbers):
    R is smooth in the grids, so central differences of sigma and of the
    emission grid match the replay adjoint."""
    sig = synthetic.value_noise(9, 2, 6.0, seed=2)
    em = synthetic.uniform_grid(9, 0.2, 1.5, seed=3, channels=3)
    rays = synthetic.sphere_rays(64, seed=4)
    wts = np.random.default_rng(5).random((64, 3)).astype(np.float32)

    def loss(sg, eg):
        sc = oracle.OracleScene(oracle_desc(sg, env=0.7, exitance_mode=0, emission_grid=eg))
        R, _ = oracle.radiance_fw(sc, "dda_collision", rays, 11)
        return float((R.astype(np.float64) * wts).sum())

    sc = oracle.OracleScene(oracle_desc(sig, env=0.7, exitance_mode=0, emission_grid=em), with_grads=True)
    oracle.radiance_bw(sc, "dda_collision", rays, 11, wts)
    rng = np.random.default_rng(6)
    for grid, grad, name in ((sig, sc.sigma_grad, "sigma"), (em, sc.emission_grad, "emission")):
        for _ in range(8):
            idx = tuple(int(rng.integers(1, 8)) for _ in range(3)) + (int(rng.integers(0, grid.shape[3])),)
            h = 1e-2
            gp, gm = grid.copy(), grid.copy()
            gp[idx] += h
            gm[idx] -= h
            fd = (loss(gp, em) - loss(gm, em)) / (2 * h) if name == "sigma" else \
                 (loss(sig, gp) - loss(sig, gm)) / (2 * h)
            # float32 radiances limit the differences to about 1e-5 absolute
            assert abs(grad[idx] - fd) <= 1e-2 * abs(fd) + 2e-4 * np.abs(grad).max(), (name, idx, grad[idx], fd)


def test_mc_collision_adjoint_is_unbiased_for_uniform_density(oracle_lib):
    """Uniform sigma0 with constant emission a and environment b:
    d E[L] / d sigma0 = (b - a) * (-d) exp(-sigma0 d), and the node gradients
    of the defensively sampled adjoint sum to that in expectation."""
    s0, a, b = 1.2, 2.0, 0.5
    sc = oracle.OracleScene(oracle_desc(homogeneous(5, s0), emission=a, env=b, exitance_mode=0, ds_epsilon=0.1),
                            with_grads=True)
    n = 60000
    dL = np.zeros((n, 3), np.float32)
    dL[:, 0] = 1.0
    oracle.radiance_bw(sc, "mc_collision", np.repeat(RAY_X, n, axis=0), 13, dL)
    est = sc.sigma_grad.sum() / n
    expect = (b - a) * (-1.0) * math.exp(-s0)
    # spread of the per-path estimate, from repeats of smaller batches
    parts = []
    for k in range(8):
        sk = oracle.OracleScene(oracle_desc(homogeneous(5, s0), emission=a, env=b, exitance_mode=0), with_grads=True)
        oracle.radiance_bw(sk, "mc_collision", np.repeat(RAY_X, 4000, axis=0), 100 + k, dL[:4000])
        parts.append(sk.sigma_grad.sum() / 4000)
    se = np.std(parts, ddof=1) * math.sqrt(4000 / n)
    assert abs(est - expect) < 4 * se + 1e-3, (est, expect, se)
