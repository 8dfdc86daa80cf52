"""Parity at the benchmark's own sizes, against the reference CPU backend
compiled from its sources (oracle/_ref/libmsref.so).

* The 1,000,000-capsule jammed colony (area fraction 0.85, log-normal
  lengths) that the benchmark steps: its contact lists at margins 0 and 0.1
  bit-exact with the reference's find_cell_contacts_cpu
  (cpp/cpu/cpu_contacts.cpp:168-219), before and after steps that move
  capsules out of the plane and divide 2 % of them.
* One step of that colony, of the 100,000-capsule trap colony with its wall
  boxes, and of a 200,000-capsule load-sensitive colony with fixed cells, at
  the tight overlap tolerance of the reference's trajectory
  conformance test (tests/conformance/trajectory_conformance_test.cpp:140-172
  uses 2e-4; 2e-5 here): the same substep structure as the reference's step
  and every position within 1e-4 capsule radius of it.

The colonies are first stepped on the GPU from their random starts (the
first step of a random jammed start takes the reference minutes); what is
compared is the next step from the same input on both paths.
"""

import numpy as np
import pytest

from microsimulator_b200 import workloads
from microsimulator_b200.types import ContactDynamicsParameters, ContactParameters, GrowthLoadLaw, GrowthLoadResponse

pytestmark = pytest.mark.gpu

RADIUS = 0.5
DT = 0.02
SETTLE = ContactDynamicsParameters(overlap_tolerance=5e-4)
TIGHT = ContactDynamicsParameters(overlap_tolerance=2e-5)


def settle(backend, world, walls, steps, seed, fraction=0.02):
    """The benchmark's steps: round(fraction * N) cells divided (daughter
    turns within +-0.02 rad), then one step at tolerance 5e-4 um."""
    for step in range(steps):
        plan = workloads.plan_divisions(world, fraction, seed=seed + step)
        world.divide_many(plan.parents, 0.5, plan.rotations)
        backend.advance_contact_dynamics(world, walls, DT, SETTLE)
        world.next_id = int(world.ids.max()) + 1
    return world


def assert_contacts_equal(backend, reference, world):
    for margin in (0.0, 0.1):
        parameters = ContactParameters(activation_margin=margin)
        expected = reference.find_cell_contacts(world, parameters)
        actual = backend.find_cell_contacts(world, parameters)
        assert len(actual) == len(expected), (margin, len(actual), len(expected))
        assert actual.tobytes() == expected.tobytes(), margin


def tight_step(backend, reference, world, walls, tight=TIGHT):
    gpu, cpu = world.copy(), world.copy()
    rg = backend.advance_contact_dynamics(gpu, walls, DT, tight).report
    rc = reference.advance_contact_dynamics(cpu, walls, DT, tight).report
    assert (rg.substeps, rg.halvings) == (rc.substeps, rc.halvings), (rg, rc)
    assert np.array_equal(gpu.ids, cpu.ids)
    spread = float(np.max(np.abs(gpu.geometry()[:, :3] - cpu.geometry()[:, :3])))
    turn = float(np.max(np.abs(gpu.geometry()[:, 3:6] - cpu.geometry()[:, 3:6])))
    print(f"{len(world)} cells: substeps {rg.substeps}, refinements {rg.refinements}/{rc.refinements}, "
          f"iterations {rg.iterations}/{rc.iterations}; max |position - reference| {spread:.3e} um, "
          f"max |direction - reference| {turn:.3e}")
    assert spread <= 1e-4 * RADIUS, spread
    assert turn <= 1e-4, turn
    assert abs(rg.max_overlap - rc.max_overlap) <= 2 * tight.overlap_tolerance


@pytest.fixture(scope="module")
def jammed_million(backend):
    """The benchmark's colony: 1,000,000 capsules (seed 42), three of its
    steps with divisions."""
    return settle(backend, workloads.jammed(n=1_000_000, seed=42), None, 3, seed=4200)


def test_million_capsule_contacts_bit_exact_at_the_start(backend, reference):
    assert_contacts_equal(backend, reference, workloads.jammed(n=1_000_000, seed=42))


def test_million_capsule_contacts_bit_exact_after_steps(backend, reference, jammed_million):
    world = jammed_million.copy()
    assert np.max(np.abs(world.position_z)) > 0.0  # crossing capsules have left the plane
    assert_contacts_equal(backend, reference, world)


def test_million_capsule_tight_step_matches_reference(backend, reference, jammed_million):
    tight_step(backend, reference, jammed_million, None)


def test_trap_colony_tight_step_with_walls_matches_reference(backend, reference):
    world, walls = workloads.trap_colony(n=100_000, seed=42)
    settle(backend, world, walls, 3, seed=77)
    for every_face in (False, True):
        expected = reference.find_external_contacts(world, walls, every_face=every_face)
        actual = backend.find_external_contacts(world, walls, every_face=every_face)
        assert actual.tobytes() == expected.tobytes()
    tight_step(backend, reference, world, walls)


def test_load_sensitive_colony_with_fixed_cells_tight_step_matches_reference(backend, reference):
    """200,000 capsules of the jammed distribution whose growth stalls under
    axial load (the linear growth-load law of contact_dynamics.cpp:600-612),
    5 % of them fixed: one step at tolerance 2e-5 um against the
    reference's.  (The exponential law's exp is FP64 rounded once here and
    glibc's expf in the reference, one ulp apart at times; in this stiff
    system, whose solves run into the iteration limit, such a difference can
    flip a halving decision, so that law is compared in lockstep on small
    colonies in test_gpu_dynamics.py instead.)"""
    law = GrowthLoadResponse(GrowthLoadLaw.LINEAR, free_load=0.05, stall_load=0.5)
    world = workloads.jammed(n=200_000, seed=7)
    world.fixed = (np.random.default_rng(8).random(len(world)) < 0.05).astype(np.uint8)
    settle_p = ContactDynamicsParameters(overlap_tolerance=5e-4, growth=law)
    for step in range(3):
        plan = workloads.plan_divisions(world, 0.02, seed=300 + step)
        world.divide_many(plan.parents, 0.5, plan.rotations)
        backend.advance_contact_dynamics(world, None, DT, settle_p)
        world.next_id = int(world.ids.max()) + 1
    tight_step(backend, reference, world, None, ContactDynamicsParameters(overlap_tolerance=2e-5, growth=law))
