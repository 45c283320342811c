"""Predictors of the heat time step -- CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the C++ host layer's predictors,
never by the product path.

Restates include/meltpooldg/linear_algebra/predictor.hpp:37-84 (LeastSquaresProjection::vmult:
Gram-Schmidt of the images A x_s, break when the remaining squared norm is below 1e-16 of the first,
back substitution, combination of the old solutions) and predictor_linear.hpp (linear
extrapolation q_n + dt_{n+1} / dt_n (q_n - q_{n-1})).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def linear_extrapolation(s0: np.ndarray, s1: np.ndarray, dt_current: float, dt_old: float) -> np.ndarray:
    return s0 + dt_current / dt_old * (s0 - s1)


def least_squares_projection(apply: Callable[[np.ndarray], np.ndarray], rhs: np.ndarray,
                             old: Sequence[np.ndarray]) -> np.ndarray:
    n = len(old)
    P = np.zeros((n, n))
    V = []
    step = 0
    while step < n:
        v = apply(old[step]).astype(np.float64)
        V.append(v)
        P[0, step] = v @ V[0]
        for j in range(step):
            v += -P[j, step] / P[j, j] * V[j]
            P[j + 1, step] = v @ V[j + 1]
        if P[step, step] < 1e-16 * P[0, 0]:
            break
        step += 1
    c = np.array([V[s] @ rhs for s in range(step)])
    for s in range(step - 1, -1, -1):
        c[s] = (c[s] - sum(c[j] * P[s, j] for j in range(s + 1, step))) / P[s, s]
    out = np.zeros_like(np.asarray(old[0], dtype=np.float64))
    for s in range(step):
        out += c[s] * old[s]
    return out
