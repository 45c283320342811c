"""The oracle's discrete adjoint of the transient heat problem against central finite differences."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import unit_directions
from oracle import adjoint as OA
from tests.adjoint_case import small_case


@pytest.fixture(scope="module")
def case():
    c = small_case(m=(3, 4, 3), n_steps=5)
    args = (c["mesh"], c["cmask"], c["rho_cp"], c["dt"])
    c["target"] = OA.forward(*args, c["z_target"], c["qhat"], c["amplitude"])
    c["args"] = args
    return c


def test_gradient_matches_central_differences(case):
    args, q, A, tgt = case["args"], case["qhat"], case["amplitude"], case["target"]
    J, gz, gA = OA.gradient(*args, case["z"], q, A, tgt)
    assert J > 0 and np.all(np.isfinite(gz))
    h = 1e-6
    for d in unit_directions(case["mesh"].ncells, 3, seed=7):
        jp = OA.objective(*args, case["z"] + h * d, q, A, tgt)
        jm = OA.objective(*args, case["z"] - h * d, q, A, tgt)
        fd = (jp - jm) / (2 * h)
        assert abs(fd - gz @ d) <= 1e-6 * max(abs(fd), 1e-3 * np.linalg.norm(gz))
    jp = OA.objective(*args, case["z"], q, A * (1 + 1e-6), tgt)
    jm = OA.objective(*args, case["z"], q, A * (1 - 1e-6), tgt)
    assert abs((jp - jm) / (2e-6 * A) - gA) <= 1e-6 * abs(gA)


def test_objective_zero_at_target_field(case):
    args = case["args"]
    J, gz, gA = OA.gradient(*args, case["z_target"], case["qhat"], case["amplitude"], case["target"])
    assert J < 1e-20 and np.max(np.abs(gz)) < 1e-9 and abs(gA) < 1e-9
