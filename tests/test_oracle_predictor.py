"""The predictor oracle (oracle/predictor.py) on small dense systems: the least-squares projection
recovers a right-hand side in the span of the images, reduces to the scalar fit for one old solution,
and drops an image that adds nothing (predictor.hpp:37-84)."""
import numpy as np

from oracle.predictor import least_squares_projection, linear_extrapolation


def test_projection_recovers_a_combination_in_the_span():
    rng = np.random.default_rng(1)
    A = rng.uniform(-1, 1, (40, 40)) + 40 * np.eye(40)
    old = [rng.uniform(-1, 1, 40) for _ in range(3)]
    target = 2.0 * old[0] - 0.5 * old[1] + 0.25 * old[2]
    got = least_squares_projection(lambda v: A @ v, A @ target, old)
    assert np.max(np.abs(got - target)) <= 1e-10


def test_one_old_solution_is_the_scalar_fit():
    rng = np.random.default_rng(2)
    A = rng.uniform(-1, 1, (30, 30)) + 30 * np.eye(30)
    x0, rhs = rng.uniform(-1, 1, (2, 30))
    ax = A @ x0
    got = least_squares_projection(lambda v: A @ v, rhs, [x0])
    assert np.max(np.abs(got - (ax @ rhs) / (ax @ ax) * x0)) <= 1e-13


def test_a_dependent_old_solution_ends_the_basis():
    rng = np.random.default_rng(3)
    A = rng.uniform(-1, 1, (20, 20)) + 20 * np.eye(20)
    x0, rhs = rng.uniform(-1, 1, (2, 20))
    one = least_squares_projection(lambda v: A @ v, rhs, [x0])
    two = least_squares_projection(lambda v: A @ v, rhs, [x0, 3.0 * x0])
    assert np.max(np.abs(one - two)) <= 1e-12


def test_linear_extrapolation():
    s0, s1 = np.array([1.0, 2.0]), np.array([0.5, 3.0])
    assert np.allclose(linear_extrapolation(s0, s1, 2e-2, 1e-2), s0 + 2.0 * (s0 - s1))
