"""The allocation-free solve entry point, through the C-ABI.

Some callers of the contact solve cannot allocate device memory - code that
runs while a CUDA stream is being captured, under an allocator that forbids
new allocations, or in a loop that must not wait on the driver's allocator.
msb_solve_contact_forces_no_alloc serves them from a static device array.
This file runs last, so a failure here leaves every other test already run;
it passes alone in a fresh process as well as after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

from microsimulator_b200 import abi
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactSolveParameters, ContactSystem, GrowthLoadResponse
from tests.golden.make_golden import chain_system

pytestmark = pytest.mark.gpu


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


@pytest.mark.parametrize("count,law", [(300, abi.GROWTH_LAW_LINEAR), (9, abi.GROWTH_LAW_EXPONENTIAL)])
def test_no_alloc_solve_matches_the_allocating_entry_point(count, law):
    system = chain_system(count, law)
    zero = np.zeros(len(system.rows), dtype=np.float32)
    params = ContactSolveParameters(2.0e-6, 200000)
    backend = B200Backend(0)
    try:
        expected = backend.solve_contact_forces(system, zero, params)
        expected_response = backend.evaluate_contact_response(system, expected.multipliers)
        for _ in range(2):  # two calls in a row share the static scratch
            status, multipliers, report = solve_no_alloc(system, zero, params)
            assert status == abi.OK
            assert report.status == abi.SOLVE_CONVERGED
            assert report.residual <= params.tolerance
            response = backend.evaluate_contact_response(system, multipliers)
            # the tolerances of the solver parity tests
            assert np.all(np.abs(response.velocities - expected_response.velocities) <= 2e-3)
            assert np.all(np.abs(response.length_rates - expected_response.length_rates) <= 2e-3)
            assert np.all(np.abs(response.loads - expected_response.loads) <= 2e-2 * (1 + expected_response.loads))
            gaps = backend.evaluate_contact_gaps(system, multipliers)
            assert np.all(gaps >= -2 * params.tolerance)
    finally:
        backend.close()


def test_no_alloc_rejects_systems_beyond_its_limit():
    rows, bodies = chain_system(9, abi.GROWTH_LAW_NONE).rows, chain_system(9, abi.GROWTH_LAW_NONE).bodies
    big = ContactSystem(np.resize(rows, 16385), bodies, 0.05, GrowthLoadResponse())
    status, _, _ = solve_no_alloc(big, np.zeros(16385, np.float32), ContactSolveParameters())
    assert status == abi.ERR_CAPACITY
