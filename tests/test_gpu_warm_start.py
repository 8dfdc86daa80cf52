"""Warm starts of the stepper through the C-ABI (msb_set_warm_start,
msb_set_motion_guess) and the per-solve log (msb_last_step_solves).

A warm start changes only the multipliers a solve starts from.  Every solve
still converges to the stepper's tolerance and the reference's overlap test
still decides acceptance, so a warm-started step lands within the
tolerance-level spread of the zero-start step (the reference's semantics)."""

import numpy as np
import pytest

from microsimulator_b200 import abi, workloads
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactDynamicsParameters

pytestmark = pytest.mark.gpu

TOLERANCE = 5e-4
DT = 0.02


@pytest.fixture
def fresh():
    b = B200Backend(0)
    yield b
    b.close()


_SETTLED = {}


def colony(seed=3, n=2000):
    """A jammed colony whose initial overlaps have relaxed: 25 zero-start
    steps with growth and divisions."""
    key = (seed, n)
    if key not in _SETTLED:
        world = workloads.jammed(n=n, seed=seed)
        b = B200Backend(0)
        try:
            p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
            for k in range(25):
                divide(world, 1000 + k, seed)
                b.advance_contact_dynamics(world, None, DT, p)
                world.next_id = int(world.ids.max()) + 1
        finally:
            b.close()
        _SETTLED[key] = world
    return _SETTLED[key].copy()


def divide(world, k, seed=3):
    plan = workloads.plan_divisions(world, 0.02, seed=seed * 100003 + k)
    world.divide_many(plan.parents, 0.5, plan.rotations)


def run(backend, world, steps, mode, guesses=None):
    p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    reports, logs = [], []
    backend.set_warm_start(mode)
    for k in range(steps):
        divide(world, k)
        if guesses is not None:
            backend.set_motion_guess(guesses[k], DT)
        r = backend.advance_contact_dynamics(world, None, DT, p)
        world.next_id = int(world.ids.max()) + 1
        reports.append(r.report)
        logs.append(backend.last_step_solves())
    return reports, logs


def displacement(w0, w1):
    d = np.zeros((len(w0), 3), np.float32)
    d[:, 0] = w1.position_x - w0.position_x
    d[:, 1] = w1.position_y - w0.position_y
    cz = w0.direction_x * w1.direction_y - w0.direction_y * w1.direction_x
    cd = w0.direction_x * w1.direction_x + w0.direction_y * w1.direction_y
    d[:, 2] = np.arctan2(cz, cd)
    return d


def test_solve_log_accounts_for_every_iteration(fresh):
    world = colony()
    reports, logs = run(fresh, world, 3, 0)
    for report, log in zip(reports, logs):
        assert len(log) >= 1
        assert int(log["iterations"].sum()) == report.iterations
        # The last solve of an accepted step converged (status 0).
        assert log["status"][-1] == 0
        assert np.all(log["rows"] > 0)


def test_carry_over_step_lands_within_tolerance_of_zero_start(fresh):
    plain, carried = colony(), colony()
    rp, _ = run(fresh, plain, 4, 0)
    rc, logs = run(fresh, carried, 4, fresh.WARM_START_CARRY)
    assert len(plain) == len(carried)
    assert np.array_equal(plain.ids, carried.ids)
    spread = np.max(np.abs(plain.geometry()[:, :3] - carried.geometry()[:, :3]))
    # Both paths converge each solve to 0.25 * the overlap tolerance; over
    # four steps their positions stay within a few tolerances.
    assert spread < 8 * TOLERANCE, spread
    assert all(log["status"][-1] == 0 for log in logs)


def test_zero_start_mode_restores_reference_semantics(fresh):
    a, b = colony(seed=5), colony(seed=5)
    run(fresh, a, 2, fresh.WARM_START_CARRY)
    fresh.set_warm_start(0)
    # After switching back, a step from the same state repeats bit for bit.
    a2, b2 = a.copy(), a.copy()
    p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    fresh.advance_contact_dynamics(a2, None, DT, p)
    other = B200Backend(0)
    try:
        other.advance_contact_dynamics(b2, None, DT, p)
    finally:
        other.close()
    assert np.array_equal(a2.geometry(), b2.geometry())


def test_motion_guess_start_lands_within_tolerance(fresh):
    world = colony(seed=7)
    divide(world, 0)
    pre = world.copy()
    p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    plain = pre.copy()
    fresh.advance_contact_dynamics(plain, None, DT, p)
    exact = displacement(pre, plain)
    for guess in (exact, np.zeros_like(exact), 3.0 * exact):
        w = pre.copy()
        fresh.set_warm_start(fresh.WARM_START_GUESS)
        fresh.set_motion_guess(guess, DT)
        r = fresh.advance_contact_dynamics(w, None, DT, p)
        log = fresh.last_step_solves()
        assert log["status"][-1] == 0
        assert r.report.substeps >= 1
        spread = np.max(np.abs(w.geometry()[:, :3] - plain.geometry()[:, :3]))
        assert spread < 4 * TOLERANCE, spread


def test_motion_guess_serves_one_step_and_checks_its_size(fresh):
    world = colony(seed=8, n=1000)
    p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    fresh.set_warm_start(fresh.WARM_START_GUESS)
    with pytest.raises(ValueError):
        fresh.set_motion_guess(np.zeros((len(world), 2), np.float32), DT)
    fresh.set_motion_guess(np.zeros((len(world) + 1, 3), np.float32), DT)
    before = world.copy()
    with pytest.raises(ValueError):
        fresh.advance_contact_dynamics(world, None, DT, p)
    assert np.array_equal(before.geometry(), world.geometry())
    # The failed step consumed the guess: the next step runs without one.
    fresh.advance_contact_dynamics(world, None, DT, p)
    bad = np.zeros((len(world), 3), np.float32)
    bad[0, 0] = np.nan
    with pytest.raises(ValueError):
        fresh.set_motion_guess(bad, DT)


def test_warm_start_flags_are_checked(fresh):
    lib = abi.load_library()
    assert lib.msb_set_warm_start(fresh._handle, 3) == abi.OK
    assert lib.msb_set_warm_start(fresh._handle, 7) == abi.OK
    assert lib.msb_set_warm_start(fresh._handle, 8) == abi.ERR_INVALID_ARGUMENT
    assert lib.msb_set_warm_start(None, 0) == abi.ERR_INVALID_ARGUMENT
    assert lib.msb_set_warm_start(fresh._handle, 0) == abi.OK
