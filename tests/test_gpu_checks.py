"""The index-checked build (libmsb200_checked.so, MSB_DEVICE_CHECKS=1): the
hot gathers (BB body and row passes, incidence gather, narrow phase) check
every slot and row index against its bound and report a failed check as
MSB_ERR_DEVICE_CHECK instead of reading out of range.  Real workloads run
through it without a check firing, with results bit-identical to the
ordinary build's (the checks only guard; they change no arithmetic)."""

import numpy as np
import pytest

from microsimulator_b200 import build, workloads
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactDynamicsParameters, ContactParameters

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def checked():
    if not build.CHECKED_OUTPUT.exists():
        pytest.fail("libmsb200_checked.so is missing: build it with __graft_entry__.build()")
    b = B200Backend(0, library=build.CHECKED_OUTPUT)
    yield b
    b.close()


def test_checked_build_steps_a_colony_unchanged(backend, checked):
    world = workloads.jammed(40_000, seed=21)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    plain, guarded = world.copy(), world.copy()
    for k in range(3):
        for w in (plain, guarded):
            plan = workloads.plan_divisions(w, 0.02, seed=50 + k)
            w.divide_many(plan.parents, 0.5, plan.rotations)
        rp = backend.advance_contact_dynamics(plain, None, 0.02, p)
        rc = checked.advance_contact_dynamics(guarded, None, 0.02, p)
        for w in (plain, guarded):
            w.next_id = int(w.ids.max()) + 1
        assert rp.report == rc.report
        assert np.array_equal(plain.geometry(), guarded.geometry())


def test_checked_build_with_walls_and_contacts(backend, checked):
    world, walls = workloads.trap_colony(n=5000, seed=8)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    a, b = world.copy(), world.copy()
    backend.advance_contact_dynamics(a, walls, 0.02, p)
    checked.advance_contact_dynamics(b, walls, 0.02, p)
    assert np.array_equal(a.geometry(), b.geometry())
    margin = ContactParameters(activation_margin=0.1)
    assert backend.find_cell_contacts(a, margin).tobytes() == checked.find_cell_contacts(a, margin).tobytes()
