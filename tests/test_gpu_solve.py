"""The device-resident BB solve through the C-ABI, on the reference's
make_chain systems (tests/conformance/contact_dynamics_conformance_test.cpp:56-176)
and the reference dynamics test's 3-body system (tests/cpp/contact_dynamics_test.cpp:154-207).

The solve's FP64 BB sums are reduced in a fixed tree on the device rather
than in the reference's 256-row grains, so the iterate path can part from
the reference's in the last bits; the conformance criteria (the unique
solution's response within 2e-3, complementarity within 2 x tolerance) are
what hold.  Forces, loads and gaps of a given multiplier vector are
bit-identical to the reference's."""

import numpy as np
import pytest

from microsimulator_b200 import abi
from microsimulator_b200.types import ContactSolveParameters, ContactSystem, GrowthLoadResponse, empty_bodies, empty_rows
from tests.golden.make_golden import chain_system

pytestmark = pytest.mark.gpu

CASES = [(2, 0), (9, 0), (9, 1), (9, 2), (300, 2), (5, 1)]


@pytest.mark.parametrize("count,law", CASES)
def test_chain_solve_matches_reference(backend, golden, count, law):
    data = golden("chains")
    key = f"chain_{count}_{law}"
    system = ContactSystem(data[f"{key}__rows"], data[f"{key}__bodies"], 0.05, GrowthLoadResponse(law, 0.3, 0.2, 3.0))
    zero = np.zeros(len(system.rows), dtype=np.float32)
    params = ContactSolveParameters(2.0e-6, 200000)
    actual = backend.solve_contact_forces(system, zero, params)
    assert actual.report.status == abi.SOLVE_CONVERGED
    assert actual.report.residual <= params.tolerance
    gaps = backend.evaluate_contact_gaps(system, actual.multipliers)
    assert np.all(actual.multipliers >= 0)
    assert np.all(gaps >= -2 * params.tolerance)
    active = actual.multipliers > 0
    assert np.all(np.abs(gaps[active]) <= 2 * params.tolerance)
    response = backend.evaluate_contact_response(system, actual.multipliers)
    # tolerance 2e-3 on velocities and rates, 2e-2 (1 + load) on loads, as the conformance test states
    assert np.all(np.abs(response.velocities - data[f"{key}__velocities"]) <= 2e-3)
    assert np.all(np.abs(response.length_rates - data[f"{key}__rates"]) <= 2e-3)
    expected_loads = data[f"{key}__loads"]
    assert np.all(np.abs(response.loads - expected_loads) <= 2e-2 * (1 + expected_loads))
    again = backend.solve_contact_forces(system, actual.multipliers, params)
    assert again.report.status == abi.SOLVE_CONVERGED
    assert again.report.iterations == 0
    assert np.array_equal(again.multipliers, actual.multipliers)


@pytest.mark.parametrize("count,law", CASES)
def test_response_of_given_multipliers_bit_exact(backend, golden, count, law):
    data = golden("chains")
    key = f"chain_{count}_{law}"
    system = ContactSystem(data[f"{key}__rows"], data[f"{key}__bodies"], 0.05, GrowthLoadResponse(law, 0.3, 0.2, 3.0))
    m = data[f"{key}__multipliers"]
    response = backend.evaluate_contact_response(system, m)
    assert np.array_equal(response.velocities, data[f"{key}__velocities"])
    assert np.array_equal(response.loads, data[f"{key}__loads"])
    assert np.array_equal(response.length_rates, data[f"{key}__rates"])
    assert np.array_equal(backend.evaluate_contact_gaps(system, m), data[f"{key}__gaps"])
    assert backend.contact_system_diagonal_bound(system) == data[f"{key}__bound"]


def test_iteration_limit_and_empty(backend):
    system = chain_system(6, abi.GROWTH_LAW_LINEAR)
    zero = np.zeros(len(system.rows), dtype=np.float32)
    stopped = backend.solve_contact_forces(system, zero, ContactSolveParameters(1e-7, 3))
    assert stopped.report.status == abi.SOLVE_ITERATION_LIMIT
    assert stopped.report.iterations == 3
    assert stopped.report.residual > 1e-7
    assert np.any(stopped.multipliers > 0)
    empty = ContactSystem(empty_rows(0), system.bodies, 0.05, system.growth)
    result = backend.solve_contact_forces(empty, np.zeros(0, np.float32), ContactSolveParameters(1e-7, 3))
    assert result.report.status == abi.SOLVE_CONVERGED
    assert len(result.multipliers) == 0


def test_iteration_limit_matches_oracle(backend, oracle):
    # Few iterations from zero: the iterates agree with the FP32 oracle to
    # the rounding of the step length.
    system = chain_system(300, abi.GROWTH_LAW_LINEAR)
    zero = np.zeros(len(system.rows), dtype=np.float32)
    for iterations in (1, 2, 5):
        a = backend.solve_contact_forces(system, zero, ContactSolveParameters(1e-9, iterations))
        b = oracle.solve_contact_forces(system, zero, ContactSolveParameters(1e-9, iterations))
        assert a.report.iterations == b.report.iterations == iterations
        assert np.allclose(a.multipliers, b.multipliers, rtol=1e-4, atol=1e-6)


def test_three_body_complementarity(backend):
    bodies = empty_bodies(3)
    bodies["translational_mobility"] = 0.5
    bodies["transverse_mobility"] = 1.0
    bodies["axial_mobility"] = 8.0
    bodies["length_rate"] = 0.5
    rows = empty_rows(2)
    rows[0]["first_slot"], rows[0]["second_slot"] = 0, 1
    rows[0]["first_jacobian"] = (0, -1, 0, 0, 0, -0.3)
    rows[0]["second_jacobian"] = (0, 1, 0, 0, 0, 0.1)
    rows[0]["first_length_lever"] = 0.5
    rows[0]["offset"] = -0.02
    rows[0]["compliance"] = 1e-4
    rows[1]["first_slot"], rows[1]["second_slot"] = 1, 2
    rows[1]["first_jacobian"] = (-1, 0, 0, 0, 0, 0)
    rows[1]["second_jacobian"] = (1, 0, 0, 0, 0, 0)
    rows[1]["offset"] = 0.5
    rows[1]["compliance"] = 1e-4
    system = ContactSystem(rows, bodies, 0.05, GrowthLoadResponse(abi.GROWTH_LAW_EXPONENTIAL, 0.2))
    params = ContactSolveParameters(1e-6)
    solved = backend.solve_contact_forces(system, np.zeros(2, np.float32), params)
    assert solved.report.status == abi.SOLVE_CONVERGED
    gaps = backend.evaluate_contact_gaps(system, solved.multipliers)
    assert solved.multipliers[0] > 0 and abs(gaps[0]) <= 1e-5
    assert solved.multipliers[1] == 0 and gaps[1] > 0
    response = backend.evaluate_contact_response(system, solved.multipliers)
    assert response.loads[0] > 0
    assert response.length_rates[0] < 0.5
    assert abs(response.length_rates[2] - 0.5) <= 1e-5
    again = backend.solve_contact_forces(system, solved.multipliers, params)
    assert again.report.iterations == 0


def test_invalid_systems_raise(backend):
    system = chain_system(4, 0)
    with pytest.raises(ValueError):
        backend.solve_contact_forces(system, -np.ones(len(system.rows), np.float32))
    with pytest.raises(ValueError):
        backend.solve_contact_forces(system, np.zeros(len(system.rows), np.float32), ContactSolveParameters(0.0))
    bad = ContactSystem(system.rows.copy(), system.bodies, 0.05)
    bad.rows["first_slot"][0] = 99
    with pytest.raises(ValueError):
        backend.solve_contact_forces(bad, np.zeros(len(bad.rows), np.float32))
    # All-fixed bodies and zero compliance: no positive diagonal.
    still = ContactSystem(system.rows.copy(), empty_bodies(len(system.bodies)), 0.05)
    still.rows["compliance"] = 0
    with pytest.raises(ValueError):
        backend.solve_contact_forces(still, np.zeros(len(still.rows), np.float32))
