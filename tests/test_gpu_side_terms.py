"""The BB passes split a row's gap into two side terms: the body pass stores
jacobian . velocity - lever * elongation rate for each of its rows, and the
row pass forms offset + dt * (first + second) + compliance * multiplier, with
-0.0f as a constraint row's second term.  These systems mix pair and
constraint rows, signed-zero offsets and multipliers, zero jacobians and
levers, fixed bodies, drift and every growth law, and check gaps and
responses bit for bit (as raw float bits, so the sign of a zero counts)
against the reference library and the oracle (row_gap,
cpp/cpu/cpu_contact_dynamics.cpp:149-159), up to the exponential growth
law's one-ulp exp."""

import numpy as np
import pytest

from microsimulator_b200 import abi
from microsimulator_b200.types import ContactSolveParameters
from tests.systems import LAWS, bits, mixed_system, multipliers_for

pytestmark = pytest.mark.gpu

EXPONENTIAL = 1


@pytest.mark.parametrize("law", range(len(LAWS)))
@pytest.mark.parametrize("seed,bodies,rows", [(1, 40, 90), (2, 3000, 9000), (3, 20000, 70000)])
def test_gaps_and_response_bit_exact(backend, reference, oracle, law, seed, bodies, rows):
    system = mixed_system(seed, bodies, rows, LAWS[law])
    m = multipliers_for(system, seed + 100)
    response = backend.evaluate_contact_response(system, m)
    expected = reference.evaluate_contact_response(system, m)
    assert np.array_equal(bits(response.velocities), bits(expected.velocities))
    assert np.array_equal(bits(response.loads), bits(expected.loads))
    gaps = backend.evaluate_contact_gaps(system, m)
    expected_gaps = reference.evaluate_contact_gaps(system, m)
    if law != EXPONENTIAL:
        assert np.array_equal(bits(response.length_rates), bits(expected.length_rates))
        assert np.array_equal(bits(gaps), bits(expected_gaps))
        assert np.array_equal(bits(gaps), bits(oracle.evaluate_contact_gaps(system, m)))
        return
    # The exponential law takes exp in FP64 rounded once to FP32, where the
    # reference calls glibc's expf: the elongation rates may differ by one
    # ulp.  Rows whose bodies' rates agree keep the reference's bits; the
    # others differ by at most that ulp times dt and the levers.
    rates, ref_rates = response.length_rates, expected.length_rates
    assert np.all(np.abs(rates - ref_rates) <= np.spacing(np.abs(ref_rates)))
    same = bits(rates) == bits(ref_rates)
    first = system.rows["first_slot"].astype(np.int64)
    second = system.rows["second_slot"]
    pair = second != abi.INVALID_SLOT
    agree = same[first] & np.where(pair, same[np.where(pair, second, 0).astype(np.int64)], True)
    assert np.array_equal(bits(gaps)[agree], bits(expected_gaps)[agree])
    # The rest within the rounding bound of their sums: 16 eps times the
    # magnitudes of the terms of offset + dt * rate + compliance * m.
    r, v = system.rows, expected.velocities.astype(np.float64)
    other = np.where(pair, second, 0).astype(np.int64)
    size = (np.abs(r["first_jacobian"] * v[first]).sum(axis=1) + r["first_length_lever"] * np.abs(ref_rates[first])
            + np.where(pair, np.abs(r["second_jacobian"] * v[other]).sum(axis=1)
                       + r["second_length_lever"] * np.abs(ref_rates[other]), 0.0))
    bound = 16 * np.spacing(np.float32(1.0)) * (np.abs(r["offset"]) + system.dt * size
                                                 + np.abs(r["compliance"] * m) + np.abs(expected_gaps))
    assert np.all(np.abs(gaps.astype(np.float64) - expected_gaps) <= bound)


def test_constraint_rows_only(backend, reference):
    system = mixed_system(4, 500, 1500, LAWS[2], walls=1.0)
    m = multipliers_for(system, 5)
    assert np.array_equal(bits(backend.evaluate_contact_gaps(system, m)),
                          bits(reference.evaluate_contact_gaps(system, m)))


def test_solve_then_gaps_of_its_multipliers(backend, reference):
    # The side terms a solve's passes leave behind do not disturb the calls
    # after it: its multipliers give the reference's gaps and response bit
    # for bit.  (The response a solve itself leaves for the move is checked
    # by the stepping tests, whose positions match the reference's.)
    system = mixed_system(6, 2000, 5000, LAWS[2])
    system.rows["offset"] = -np.abs(system.rows["offset"])
    solved = backend.solve_contact_forces(system, np.zeros(len(system.rows), np.float32),
                                          ContactSolveParameters(1e-4, 5000))
    assert solved.report.status in (abi.SOLVE_CONVERGED, abi.SOLVE_ITERATION_LIMIT)
    m = solved.multipliers
    assert np.array_equal(bits(backend.evaluate_contact_gaps(system, m)),
                          bits(reference.evaluate_contact_gaps(system, m)))
    response = backend.evaluate_contact_response(system, m)
    expected = reference.evaluate_contact_response(system, m)
    assert np.array_equal(bits(response.velocities), bits(expected.velocities))
