"""The whole contact-dynamics step on the GPU through the C-ABI: the
scenarios of the reference's dynamics tests (tests/cpp/contact_dynamics_test.cpp)
and parity with the reference's own step on the same inputs.

Parity criteria (from the port's specification): post-step positions within
1e-4 capsule radius of the reference CPU backend at a tight solve
tolerance, and every result's error against the FP64 oracle stated."""

import math

import numpy as np
import pytest

from microsimulator_b200 import abi, workloads
from microsimulator_b200.simulation import Simulation
from microsimulator_b200.types import (
    ConstraintContactParameters,
    ContactDynamicsParameters,
    ContactParameters,
    GrowthLoadLaw,
    GrowthLoadResponse,
)
from microsimulator_b200.world import ConstraintSet, WorldState
from tests.golden.make_golden import world_from

pytestmark = pytest.mark.gpu

RADIUS = 0.5


def close(a, b, tol=1e-5):
    return abs(float(a) - float(b)) <= tol


@pytest.fixture
def sim(backend):
    return Simulation(backend=backend)


def test_separated_cells_grow_without_moving(sim):
    a = sim.add_cell(length=2.0)
    b = sim.add_cell(position=(0, 5, 0), length=2.0)
    result = sim.step(0.1, ContactDynamicsParameters())
    assert result.report.max_rows == 0
    assert close(sim.cell(a)["position"][1], 0.0) and close(sim.cell(b)["position"][1], 5.0)
    assert close(sim.cell(a)["length"], 2.2)
    assert close(result.length_increments[0], 0.2)
    assert close(result.axial_loads[0], 0.0)
    assert close(sim.time(), 0.1)


def test_end_to_end_cells_push_apart(sim):
    a = sim.add_cell(position=(-1.5, 0, 0), length=2.0)
    b = sim.add_cell(position=(1.5, 0, 0), length=2.0)
    p = ContactDynamicsParameters()
    result = sim.step(0.1, p)
    left, right = sim.cell(a), sim.cell(b)
    assert close(left["length"], 2.2) and close(right["length"], 2.2)
    assert close(left["position"][0], -right["position"][0], 1e-4)
    gap = (right["position"][0] - left["position"][0]) - 0.5 * (left["length"] + right["length"]) - 1.0
    assert -p.overlap_tolerance < gap < p.overlap_tolerance
    assert result.axial_loads[0] > 0
    assert close(result.axial_loads[0], result.axial_loads[1], 1e-3)


def test_cell_between_walls_stalls(sim):
    sim.add_plane_constraint(point=(-2, 0, 0), inward_normal=(1, 0, 0))
    sim.add_plane_constraint(point=(2, 0, 0), inward_normal=(-1, 0, 0))
    cid = sim.add_cell(length=2.0)
    p = ContactDynamicsParameters(growth=GrowthLoadResponse(GrowthLoadLaw.LINEAR, stall_load=4.0))
    p.wall_stiffness = p.contact_stiffness
    for _ in range(200):
        result = sim.step(0.05, p)
    filled = sim.cell(cid)
    wall_overlap = 4.0 / p.wall_stiffness
    assert filled["length"] >= 3.0 - 2 * p.overlap_tolerance
    assert filled["length"] <= 3.0 + 2 * (wall_overlap + p.overlap_tolerance)
    assert close(filled["position"][0], 0.0, 1e-3)
    assert 4.0 * 0.99 <= result.axial_loads[0] <= 4.0 * 1.05
    held = filled["length"]
    for _ in range(50):
        sim.step(0.05, p)
    assert close(sim.cell(cid)["length"], held, 1e-4)


def test_fixed_cell_holds_its_place(sim):
    anchor = sim.add_cell(position=(-1.5, 0, 0), length=2.0, fixed=True)
    free = sim.add_cell(position=(1.5, 0, 0), length=2.0)
    p = ContactDynamicsParameters()
    sim.step(0.1, p)
    assert close(sim.cell(anchor)["position"][0], -1.5)
    assert close(sim.cell(anchor)["length"], 2.2)
    assert close(sim.cell(free)["position"][0], 1.7, 2 * p.overlap_tolerance)


def test_container_corner_reports_every_wall(backend):
    w = WorldState()
    w.add_cell((1.1, 1.55, 0.0), (1, 0, 0), 1.0, 0.4)
    cs = ConstraintSet()
    cs.add_box(half_extents=(2, 2, 0.6), allowed_region=abi.REGION_INSIDE)
    prm = ConstraintContactParameters(activation_margin=0.1)
    assert len(backend.find_external_contacts(w, cs, prm)) == 2
    faces = backend.find_external_contacts(w, cs, prm, every_face=True)
    assert len(faces) == 3


def divide_long_cells(sim, division_length, counter):
    """Division with fixed alternating turns, as the conformance test does."""
    long = [int(i) for i, l in zip(sim.world.ids, sim.world.lengths) if l >= division_length]
    if not long:
        return counter
    rotations = []
    for _ in long:
        row = []
        for _ in range(2):
            angle = np.float32(0.004) * np.float32(counter % 7) - np.float32(0.012)
            counter += 1
            row += [np.cos(angle, dtype=np.float32), np.sin(angle, dtype=np.float32)]
        rotations.append(row)
    sim.world.divide_many(np.array(long, dtype=np.uint64), 0.5, np.array(rotations, dtype=np.float32))
    return counter


def footprint(world):
    return float(np.sum(math.pi * world.radii ** 2 + 2 * world.radii * world.lengths))


def test_closed_chamber_fills_and_holds(sim):
    sim.add_box_constraint(half_extents=(2, 2, 0.6), allowed_region=abi.REGION_INSIDE)
    sim.add_cell(length=1.0, radius=0.4)
    p = ContactDynamicsParameters(growth=GrowthLoadResponse(GrowthLoadLaw.LINEAR, stall_load=2.0))
    counter = 0
    for _ in range(300):
        counter = divide_long_cells(sim, 2.0, counter)
        sim.step(0.05, p)
    filled_count = sim.cell_count()
    filled = footprint(sim.world)
    for _ in range(200):
        counter = divide_long_cells(sim, 2.0, counter)
        sim.step(0.05, p)
    assert sim.cell_count() == filled_count
    assert abs(footprint(sim.world) - filled) < 0.02
    cover = footprint(sim.world) / 16.0
    assert 0.6 < cover < 1.0
    contacts = sim.find_cell_contacts().contacts
    assert np.all(contacts["signed_separation"] > -0.01)
    assert np.all(np.abs(sim.world.position_x) <= 2.0) and np.all(np.abs(sim.world.position_y) <= 2.0)
    assert np.all(np.abs(sim.world.position_z) < 1e-3)


def test_free_colony_grows_in_full(sim):
    sim.add_cell(length=2.0)
    p = ContactDynamicsParameters()
    counter = 0
    worst = 0.0
    expected_length = None
    for _ in range(100):
        counter = divide_long_cells(sim, 4.0, counter)
        result = sim.step(0.05, p)
        worst = max(worst, result.report.max_overlap)
    assert sim.cell_count() >= 16
    assert np.all(np.abs(sim.world.position_z) < 1e-3)
    assert worst < 0.01


def test_failed_step_leaves_state_unchanged(sim):
    for x in (-1.5, 1.5, 4.5):
        sim.add_cell(position=(x, 0, 0), length=2.0)
    before = sim.world.geometry().copy()
    p = ContactDynamicsParameters(max_iterations=1, overlap_tolerance=1e-7, max_step_halvings=2)
    with pytest.raises(RuntimeError):
        sim.step(0.1, p)
    assert sim.time() == 0.0
    assert np.array_equal(sim.world.geometry(), before)
    with pytest.raises(ValueError):
        sim.step(0.1, ContactDynamicsParameters(contact_stiffness=0.0))


# ---- parity with the reference's step -------------------------------------

def test_colony_step_matches_reference(backend, golden, oracle):
    data = golden("colony_1k")
    world = world_from(data, "world__")
    stepped = world_from(data, "stepped__")
    result = backend.advance_contact_dynamics(world, None, 0.02, ContactDynamicsParameters(overlap_tolerance=5e-4))
    report = data["step_report"]
    # Same substep structure as the reference.
    assert result.report.substeps == report[0]
    assert result.report.halvings == report[1]
    # Both solves converge to the overlap tolerance (5e-4 um) from the same
    # rows, so the positions agree to a few tolerances (measured on B200:
    # 5.7e-4 um); 1e-4 capsule radius is asserted at a tight tolerance below.
    spread = np.max(np.abs(world.geometry()[:, :3] - stepped.geometry()[:, :3]))
    assert spread <= 4 * 5e-4, spread


@pytest.mark.parametrize("seed", [1, 2])
def test_tight_step_positions_within_1e4_radius(backend, oracle, seed):
    world = workloads.colony_1k(seed=seed, n=300, side=30.0, growth_rate=0.5)
    # Settle first with the reference-identical oracle so the step is a
    # growth step of a relaxed colony.
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    for _ in range(20):
        oracle.advance_contact_dynamics(world, None, 0.02, p)
    tight = ContactDynamicsParameters(overlap_tolerance=2e-5)
    gpu, cpu, f64 = world.copy(), world.copy(), world.copy()
    rg = backend.advance_contact_dynamics(gpu, None, 0.02, tight)
    rc = oracle.advance_contact_dynamics(cpu, None, 0.02, tight)
    oracle.advance_contact_dynamics(f64, None, 0.02, tight, precision=64)
    assert rg.report.substeps == rc.report.substeps
    dpos = np.max(np.abs(gpu.geometry()[:, :3] - cpu.geometry()[:, :3]))
    assert dpos <= 1e-4 * RADIUS, dpos
    # Error against FP64 stated: both paths sit at the same distance.
    e_gpu = np.max(np.abs(gpu.geometry()[:, :3] - f64.geometry()[:, :3]))
    e_cpu = np.max(np.abs(cpu.geometry()[:, :3] - f64.geometry()[:, :3]))
    assert e_gpu <= max(2 * e_cpu, 1e-4 * RADIUS)


def test_step_with_trap_walls_matches_oracle(backend, oracle):
    world, cs = workloads.trap_colony(n=800, seed=6, area_fraction=0.5)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    a, b = world.copy(), world.copy()
    ra = backend.advance_contact_dynamics(a, cs, 0.02, p)
    rb = oracle.advance_contact_dynamics(b, cs, 0.02, p)
    assert ra.report.substeps == rb.report.substeps
    # Within a few solve tolerances (measured on B200: identical bits).
    assert np.max(np.abs(a.geometry() - b.geometry())) <= 4 * p.overlap_tolerance


def test_device_resident_step_equals_host_step(backend):
    from microsimulator_b200.backend import DeviceCells, DeviceOutputs

    world = workloads.colony_1k(seed=9, n=500, side=35.0, growth_rate=0.5)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    host = world.copy()
    rh = backend.advance_contact_dynamics(host, None, 0.02, p)
    cells = DeviceCells(world)
    outputs = DeviceOutputs(len(world))
    rd = backend.advance_contact_dynamics_device(cells, None, 0.02, p, outputs=outputs)
    device = world.copy()
    cells.download(device)
    assert rh.report == rd
    assert np.array_equal(host.geometry(), device.geometry())
    assert np.array_equal(rh.axial_loads, outputs.loads.cpu().numpy())


def test_pinned_host_step_equals_pageable_host_step(backend):
    """A world kept in page-locked host arrays (copied by DMA without the
    staging buffers) steps to the same bits, with the same outputs, as one
    in ordinary numpy arrays."""
    from microsimulator_b200.backend import PinnedCells

    world = workloads.colony_1k(seed=13, n=700, side=38.0, growth_rate=0.5)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    pageable = world.copy()
    rp = backend.advance_contact_dynamics(pageable, None, 0.02, p)
    cells = PinnedCells(1000)
    cells.load(world)
    outputs = cells.outputs()
    rq = backend.advance_contact_dynamics(cells, None, 0.02, p, outputs=outputs)
    pinned = world.copy()
    cells.store(pinned)
    assert rp.report == rq.report
    assert np.array_equal(pageable.geometry(), pinned.geometry())
    assert np.array_equal(rp.center_velocities, outputs[0]) and np.array_equal(rp.axial_loads, outputs[1])
    assert np.array_equal(rp.length_increments, outputs[2])
    with pytest.raises(ValueError):
        backend.advance_contact_dynamics(cells, None, 0.02, p, outputs=(outputs[0][:-1], outputs[1], outputs[2]))


def test_steps_are_deterministic(backend):
    """The same step from the same state gives the same bits, on the same
    context and on a fresh one (the reference's thread-invariance test,
    tests/cpp/thread_invariance_test.cpp:61-84, asks this across thread
    counts): every reduction on the device runs in a fixed order."""
    from microsimulator_b200.backend import B200Backend

    world = workloads.jammed(30_000, seed=17)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    runs = []
    for b in (backend, backend, None):
        fresh = b is None
        if fresh:
            b = B200Backend(0)
        w = world.copy()
        result = b.advance_contact_dynamics(w, None, 0.02, p)
        runs.append((w.geometry(), result.report, result.center_velocities, result.axial_loads))
        if fresh:
            b.close()
    for geometry, report, velocities, loads in runs[1:]:
        assert np.array_equal(geometry, runs[0][0])
        assert report == runs[0][1]
        assert np.array_equal(velocities, runs[0][2]) and np.array_equal(loads, runs[0][3])


def within(actual, expected, tolerance):
    """trajectory_conformance_test.cpp's comparison: abs + rel tolerance."""
    return np.all(np.abs(actual - expected) <= tolerance + tolerance * np.abs(expected))


def test_trajectory_conformance(backend, reference):
    """The mechanical part of the reference's trajectory conformance test
    (tests/conformance/trajectory_conformance_test.cpp:26-172): three cells
    (one fixed) on a plane, steps of 0.01, 0.015 and 0.02 at overlap
    tolerance 2e-4, cell 2 divided after the first; geometry within 2e-3
    (absolute plus relative) of the reference CPU backend after every step."""
    world = WorldState()
    positions = [(0.0, 0.0, 0.0), (0.0, 0.65, 0.0), (0.2, 1.3, 0.1)]
    directions = [(1.0, 0.0, 0.0), (1.0, 0.1, 0.0), (0.95, -0.1, 0.08)]
    for i in range(3):
        world.add_cell(position=positions[i], direction=directions[i], length=3.0 + 0.2 * i, radius=0.45,
                       growth_rate=0.02 + 0.01 * i, fixed=i == 0)
    walls = ConstraintSet()
    walls.add_plane(point=(0.0, 0.4, 0.0), inward_normal=(0.0, 1.0, 0.0), coefficient=1.25)
    p = ContactDynamicsParameters(overlap_tolerance=2.0e-4)
    handle = reference.world_create(world, walls)
    try:
        gpu, mirror = world.copy(), world.copy()
        for step, dt in enumerate((0.01, 0.015, 0.02)):
            rg = backend.advance_contact_dynamics(gpu, walls, dt, p).report
            rr = reference.world_step(handle, dt, p)
            reference.world_read(handle, mirror)
            assert within(rg.max_overlap, rr.max_overlap, 2.0e-3)
            assert np.array_equal(gpu.ids, mirror.ids)
            assert within(gpu.geometry(), mirror.geometry(), 2.0e-3), np.max(np.abs(gpu.geometry() - mirror.geometry()))
            if step == 0:
                identity = np.array([[1.0, 0.0, 1.0, 0.0]], np.float32)
                gpu.divide_many([2], 0.5, identity)
                mirror.divide_many([2], 0.5, identity)
                reference.world_divide(handle, [2], identity)
                reference.world_read(handle, mirror)
                assert np.array_equal(gpu.geometry(), mirror.geometry())
    finally:
        reference.world_destroy(handle)


def test_growing_colony_trajectory(backend, reference):
    """A colony of 40 cells grown for 25 steps with every cell of length >= 4
    divided (daughter turns +-0.02 rad), stepped in lockstep with the
    reference CPU backend: geometry within 2e-3 of it after every step."""
    world = workloads.colony_1k(seed=23, n=40, side=14.0, growth_rate=0.5)
    p = ContactDynamicsParameters(overlap_tolerance=2.0e-4)
    handle = reference.world_create(world)
    try:
        gpu, mirror = world.copy(), world.copy()
        for step in range(25):
            plan = workloads.plan_divisions(mirror, 1.0, seed=1000 + step, minimum_length=4.0)
            for w in (gpu, mirror):
                w.divide_many(plan.parents, 0.5, plan.rotations)
            reference.world_divide(handle, plan.parents, plan.rotations)
            backend.advance_contact_dynamics(gpu, None, 0.02, p)
            reference.world_step(handle, 0.02, p)
            reference.world_read(handle, mirror)
            gpu.next_id = mirror.next_id = int(mirror.ids.max()) + 1
            assert np.array_equal(gpu.ids, mirror.ids)
            assert within(gpu.geometry(), mirror.geometry(), 2.0e-3), (step, np.max(np.abs(gpu.geometry() - mirror.geometry())))
        assert len(gpu) > 50  # it grew and divided
    finally:
        reference.world_destroy(handle)


def lockstep(backend, reference, world, walls, steps, p, seed, tolerance=2.0e-3):
    """Steps `world` on the backend and on the reference CPU backend side by
    side, every cell of length >= 4 divided before each step (daughter turns
    +-0.02 rad, the plan taken from the reference's state); returns the
    largest geometry difference seen and asserts it within `tolerance`
    (absolute plus relative) after every step."""
    handle = reference.world_create(world, walls)
    worst = 0.0
    try:
        gpu, mirror = world.copy(), world.copy()
        for step in range(steps):
            plan = workloads.plan_divisions(mirror, 1.0, seed=seed + step, minimum_length=4.0)
            for w in (gpu, mirror):
                w.divide_many(plan.parents, 0.5, plan.rotations)
            reference.world_divide(handle, plan.parents, plan.rotations)
            backend.advance_contact_dynamics(gpu, walls, 0.02, p)
            reference.world_step(handle, 0.02, p)
            reference.world_read(handle, mirror)
            gpu.next_id = mirror.next_id = int(mirror.ids.max()) + 1
            assert np.array_equal(gpu.ids, mirror.ids)
            worst = max(worst, float(np.max(np.abs(gpu.geometry() - mirror.geometry()))))
            assert within(gpu.geometry(), mirror.geometry(), tolerance), (step, worst)
        return worst, len(gpu)
    finally:
        reference.world_destroy(handle)


@pytest.mark.parametrize("law", [GrowthLoadResponse(GrowthLoadLaw.EXPONENTIAL, sensitivity=2.0),
                                 GrowthLoadResponse(GrowthLoadLaw.LINEAR, free_load=0.05, stall_load=0.5)])
def test_load_sensitive_colony_in_lockstep(backend, reference, law):
    """A colony whose growth falls with axial load (the reference's
    load-sensitive colony, python/tests/test_contact_dynamics.py:450-…, and
    the growth-load laws of contact_dynamics.cpp:600-612), stepped in lockstep
    with the reference for 20 steps."""
    world = workloads.colony_1k(seed=31, n=60, side=12.0, growth_rate=0.5)
    p = ContactDynamicsParameters(overlap_tolerance=2.0e-4, growth=law)
    worst, cells = lockstep(backend, reference, world, None, 20, p, seed=700)
    assert cells > 62


def test_trap_colony_with_walls_in_lockstep(backend, reference):
    """Configuration 2's shape at small size: capsules in the trap with the
    trap-channel device's wall boxes, growing and dividing for 12 steps in
    lockstep with the reference."""
    world, walls = workloads.trap_colony(n=400, seed=12, area_fraction=0.6)
    p = ContactDynamicsParameters(overlap_tolerance=2.0e-4)
    worst, cells = lockstep(backend, reference, world, walls, 12, p, seed=900)
    assert cells > 400
