"""The allocation-free solve entry point, through the C-ABI.

Some callers of the contact solve cannot allocate device memory: code under
an allocator policy that forbids new device allocations after start-up, or a
real-time loop that must not wait on the driver's allocator.
msb_solve_contact_forces_no_alloc serves them from a static device array of
fixed size (16,384 rows, 8,192 bodies).  Each case below calls it twice in a
row, because every call shares that array and must clear what it needs.

Its results are checked against the allocating entry point, against the
reference's own solves of the make_chain systems (tests/golden/chains.npz)
and against the FP32 oracle, within the tolerances of the solver parity
tests.  This file runs last, so a failure here leaves every other test
already run; it passes alone in a fresh process as well as after the rest of
the suite.
"""

import ctypes

import numpy as np
import pytest

from microsimulator_b200 import abi
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactSolveParameters, ContactSystem, GrowthLoadResponse
from tests.golden.make_golden import chain_system, make_chain
from tests.systems import multipliers_for

pytestmark = pytest.mark.gpu

MAX_ROWS = 16384
MAX_BODIES = 8192


def solve_no_alloc(system, initial, parameters):
    lib = abi.load_library()
    native = system.native()
    initial = np.ascontiguousarray(initial, dtype=np.float32)
    out = np.zeros(len(system.rows), dtype=np.float32)
    report = abi.ContactSolveReport()
    prm = parameters.native()
    status = lib.msb_solve_contact_forces_no_alloc(
        ctypes.byref(native), ctypes.c_void_p(abi.ptr(initial)), ctypes.byref(prm), ctypes.c_void_p(abi.ptr(out)),
        ctypes.byref(report), None)
    return status, out, report


def chains_at_the_limit(law: int) -> ContactSystem:
    """256 independent make_chain systems of 32 bodies, each pair with a
    second contact row at the other end of the pair: exactly 8,192 bodies and
    16,384 rows, the largest system the static array takes."""
    rows, bodies = make_chain(32)
    pairs = rows[(rows["second_slot"] != abi.INVALID_SLOT) & (rows["offset"] < 1.0)]
    second = pairs.copy()
    second["first_jacobian"][:, 5] *= -1.0
    second["second_jacobian"][:, 5] *= -1.0
    second["offset"] = second["offset"] + np.float32(0.001)
    one = np.concatenate([rows, second])
    all_rows, all_bodies = [], []
    for k in range(256):
        block = one.copy()
        block["first_slot"] += 32 * k
        block["second_slot"] = np.where(block["second_slot"] == abi.INVALID_SLOT, abi.INVALID_SLOT,
                                        block["second_slot"] + 32 * k)
        all_rows.append(block)
        all_bodies.append(bodies)
    system = ContactSystem(np.concatenate(all_rows), np.concatenate(all_bodies), 0.05,
                           GrowthLoadResponse(law, 0.3, 0.2, 3.0))
    assert len(system.rows) == MAX_ROWS and len(system.bodies) == MAX_BODIES
    return system


def assert_same_solution(backend, system, multipliers, expected, tolerance):
    """The tolerances of the solver parity tests (the reference's dynamics
    conformance test): velocities and rates within 2e-3, loads within
    2e-2 (1 + load), complementarity within 2 x tolerance."""
    response = backend.evaluate_contact_response(system, multipliers)
    want = backend.evaluate_contact_response(system, expected)
    assert np.all(np.abs(response.velocities - want.velocities) <= 2e-3)
    assert np.all(np.abs(response.length_rates - want.length_rates) <= 2e-3)
    assert np.all(np.abs(response.loads - want.loads) <= 2e-2 * (1 + want.loads))
    gaps = backend.evaluate_contact_gaps(system, multipliers)
    assert np.all(multipliers >= 0)
    assert np.all(gaps >= -2 * tolerance)


@pytest.fixture(scope="module")
def allocating():
    backend = B200Backend(0)
    yield backend
    backend.close()


@pytest.mark.parametrize("count,law", [(300, abi.GROWTH_LAW_LINEAR), (9, abi.GROWTH_LAW_EXPONENTIAL)])
def test_no_alloc_solve_matches_the_allocating_entry_point(allocating, count, law):
    system = chain_system(count, law)
    zero = np.zeros(len(system.rows), dtype=np.float32)
    params = ContactSolveParameters(2.0e-6, 200000)
    expected = allocating.solve_contact_forces(system, zero, params)
    for _ in range(2):  # two calls in a row share the static scratch
        status, multipliers, report = solve_no_alloc(system, zero, params)
        assert status == abi.OK
        assert report.status == abi.SOLVE_CONVERGED
        assert report.residual <= params.tolerance
        assert_same_solution(allocating, system, multipliers, expected.multipliers, params.tolerance)


@pytest.mark.parametrize("count,law", [(2, 0), (9, 0), (9, 1), (9, 2), (300, 2), (5, 1)])
def test_no_alloc_solve_matches_the_reference(allocating, golden, count, law):
    """The reference's own solves of the make_chain systems of its dynamics
    conformance test (tests/conformance/contact_dynamics_conformance_test.cpp:56-176)."""
    data = golden("chains")
    key = f"chain_{count}_{law}"
    system = ContactSystem(data[f"{key}__rows"], data[f"{key}__bodies"], 0.05, GrowthLoadResponse(law, 0.3, 0.2, 3.0))
    zero = np.zeros(len(system.rows), dtype=np.float32)
    params = ContactSolveParameters(2.0e-6, 200000)
    for _ in range(2):
        status, multipliers, report = solve_no_alloc(system, zero, params)
        assert status == abi.OK and report.status == abi.SOLVE_CONVERGED
        response = allocating.evaluate_contact_response(system, multipliers)
        assert np.all(np.abs(response.velocities - data[f"{key}__velocities"]) <= 2e-3)
        assert np.all(np.abs(response.length_rates - data[f"{key}__rates"]) <= 2e-3)
        expected_loads = data[f"{key}__loads"]
        assert np.all(np.abs(response.loads - expected_loads) <= 2e-2 * (1 + expected_loads))
        # A restart from the solution takes no iteration and returns it unchanged.
        status, again, report = solve_no_alloc(system, multipliers, params)
        assert status == abi.OK and report.status == abi.SOLVE_CONVERGED and report.iterations == 0
        assert np.array_equal(again, multipliers)


@pytest.mark.parametrize("law", [abi.GROWTH_LAW_NONE, abi.GROWTH_LAW_LINEAR])
def test_no_alloc_at_its_limit_matches_the_allocating_path_and_the_oracle(allocating, oracle, law):
    system = chains_at_the_limit(law)
    params = ContactSolveParameters(2.0e-6, 200000)
    for initial in (np.zeros(MAX_ROWS, np.float32), np.abs(multipliers_for(system, 5))):
        expected = allocating.solve_contact_forces(system, initial, params)
        assert expected.report.status == abi.SOLVE_CONVERGED
        pinned = oracle.solve_contact_forces(system, initial, params)
        assert pinned.report.status == abi.SOLVE_CONVERGED
        for _ in range(2):
            status, multipliers, report = solve_no_alloc(system, initial, params)
            assert status == abi.OK
            assert report.status == abi.SOLVE_CONVERGED and report.residual <= params.tolerance
            assert_same_solution(allocating, system, multipliers, expected.multipliers, params.tolerance)
            assert_same_solution(allocating, system, multipliers, pinned.multipliers, params.tolerance)


def test_no_alloc_iteration_limit_matches_the_allocating_path(allocating, oracle):
    system = chain_system(6, abi.GROWTH_LAW_LINEAR)
    zero = np.zeros(len(system.rows), dtype=np.float32)
    params = ContactSolveParameters(1e-7, 3)
    expected = allocating.solve_contact_forces(system, zero, params)
    pinned = oracle.solve_contact_forces(system, zero, params)
    for _ in range(2):
        status, multipliers, report = solve_no_alloc(system, zero, params)
        assert status == abi.OK
        assert report.status == abi.SOLVE_ITERATION_LIMIT == expected.report.status
        assert report.iterations == expected.report.iterations == pinned.report.iterations == 3
        # Three iterates from zero agree with the FP32 oracle to rounding.
        assert np.allclose(multipliers, pinned.multipliers, rtol=1e-4, atol=1e-6)


def test_no_alloc_rejects_systems_beyond_its_limit():
    system = chain_system(9, abi.GROWTH_LAW_NONE)
    big = ContactSystem(np.resize(system.rows, MAX_ROWS + 1), system.bodies, 0.05, GrowthLoadResponse())
    status, _, _ = solve_no_alloc(big, np.zeros(MAX_ROWS + 1, np.float32), ContactSolveParameters())
    assert status == abi.ERR_CAPACITY
    many = ContactSystem(system.rows, np.resize(system.bodies, MAX_BODIES + 1), 0.05, GrowthLoadResponse())
    status, _, _ = solve_no_alloc(many, np.zeros(len(system.rows), np.float32), ContactSolveParameters())
    assert status == abi.ERR_CAPACITY
