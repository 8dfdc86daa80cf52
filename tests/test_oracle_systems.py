"""The oracle's restatement of evaluate, row_gap, the diagonal bound and the
BB solve (oracle/contact_oracle.cpp) against the reference library itself on
random systems that mix pair and constraint rows, signed zeros, fixed
bodies, drift and all three growth-load laws: bit for bit, including 300
iterations of a solve (cpp/cpu/cpu_contact_dynamics.cpp:40-338,
cpp/core/contact_solver.hpp:44-120)."""

import numpy as np
import pytest

from microsimulator_b200.types import ContactSolveParameters
from tests.systems import LAWS, bits, mixed_system, multipliers_for


@pytest.mark.parametrize("law", range(len(LAWS)))
@pytest.mark.parametrize("seed,bodies,rows", [(1, 40, 90), (2, 3000, 9000)])
def test_evaluation_matches_reference(oracle, reference, law, seed, bodies, rows):
    system = mixed_system(seed, bodies, rows, LAWS[law])
    m = multipliers_for(system, seed + 100)
    assert np.array_equal(bits(oracle.evaluate_contact_gaps(system, m)), bits(reference.evaluate_contact_gaps(system, m)))
    got = oracle.evaluate_contact_response(system, m)
    expected = reference.evaluate_contact_response(system, m)
    assert np.array_equal(bits(got.velocities), bits(expected.velocities))
    assert np.array_equal(bits(got.loads), bits(expected.loads))
    assert np.array_equal(bits(got.length_rates), bits(expected.length_rates))
    assert oracle.contact_system_diagonal_bound(system) == reference.contact_system_diagonal_bound(system)


@pytest.mark.parametrize("law", range(len(LAWS)))
def test_solve_matches_reference(oracle, reference, law):
    system = mixed_system(7, 2000, 5000, LAWS[law])
    system.rows["offset"] = -np.abs(system.rows["offset"])
    start = np.zeros(len(system.rows), np.float32)
    parameters = ContactSolveParameters(1e-4, 300)
    got = oracle.solve_contact_forces(system, start, parameters)
    expected = reference.solve_contact_forces(system, start, parameters)
    assert got.report == expected.report
    assert np.array_equal(bits(got.multipliers), bits(expected.multipliers))
