"""Flow drift inside the stepper (msb_set_flow_field + flow_drift) against
the reference's own Simulation::step with a signal grid that holds the same
velocity field: the Jeffery-closure drift of every body, obstacles, and the
travel limit on substeps."""

import numpy as np
import pytest

from microsimulator_b200 import workloads
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactDynamicsParameters, FlowField
from microsimulator_b200.world import WorldState

pytestmark = pytest.mark.gpu

DT = 0.02


def field(shape=(24, 20, 1), spacing=(2.0, 2.0, 1.0), origin=(-4.0, -4.0, -0.5), strength=1.0, solid=True, seed=0):
    """A swirling shear flow sampled on the faces of the lattice, with a few
    solid sites."""
    sx, sy, sz = shape
    ox, oy, oz = origin
    hx, hy, hz = spacing
    rng = np.random.default_rng(seed)
    xf = np.zeros((sx + 1, sy, sz), np.float32)
    yf = np.zeros((sx, sy + 1, sz), np.float32)
    zf = np.zeros((sx, sy, sz + 1), np.float32)
    for i in range(sx + 1):
        for j in range(sy):
            x, y = ox + i * hx, oy + (j + 0.5) * hy
            xf[i, j, :] = strength * (0.3 * y - 0.05 * x + 0.02 * rng.standard_normal())
    for i in range(sx):
        for j in range(sy + 1):
            x, y = ox + (i + 0.5) * hx, oy + j * hy
            yf[i, j, :] = strength * (-0.2 * x + 0.05 * y + 0.02 * rng.standard_normal())
    # Closed faces carry no flow: the lattice's boundary, and every face of a
    # solid site (the reference's signal grid rejects a field otherwise).
    xf[0], xf[sx] = 0.0, 0.0
    yf[:, 0], yf[:, sy] = 0.0, 0.0
    obstacles = None
    if solid:
        obstacles = np.zeros((sx, sy, sz), np.uint8)
        obstacles[3:5, 12:14, :] = 1
        obstacles[15, 4, :] = 1
        for i, j, _ in np.argwhere(obstacles):
            xf[i, j], xf[i + 1, j] = 0.0, 0.0
            yf[i, j], yf[i, j + 1] = 0.0, 0.0
    return FlowField(shape, origin, spacing, xf, yf, zf, obstacles)


def colony(n=150, seed=5):
    w = workloads.colony_1k(seed=seed, n=n, side=30.0, growth_rate=0.5)
    fresh = WorldState.from_arrays(np.stack([w.position_x, w.position_y, w.position_z], 1),
                                   np.stack([w.direction_x, w.direction_y, w.direction_z], 1), w.lengths, 0.5,
                                   growth_rates=0.5)
    return fresh


def test_drift_of_isolated_cells_is_the_references(backend, reference):
    world = WorldState()
    world.add_cell(position=(1.0, 2.0, 0.0), direction=(0.6, 0.8, 0.0), length=2.5, growth_rate=0.0)
    world.add_cell(position=(20.0, 10.0, 0.0), direction=(1.0, 0.0, 0.0), length=3.0, growth_rate=0.0)
    world.add_cell(position=(7.0, 21.0, 0.0), direction=(0.0, 1.0, 0.0), length=2.0, growth_rate=0.0)
    f = field()
    p = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    gpu, ref = world.copy(), world.copy()
    backend.set_flow_field(f)
    try:
        rg = backend.advance_contact_dynamics(gpu, None, DT, p)
    finally:
        backend.set_flow_field(None)
    rr = reference.flow_step(ref, f, DT, p)
    assert rg.report.substeps == rr.substeps
    moved = np.max(np.abs(gpu.geometry()[:, :3] - world.geometry()[:, :3]))
    assert moved > 1e-3  # the flow carried them
    # No contacts: the step is the drift alone, the same float operations.
    assert np.array_equal(gpu.geometry(), ref.geometry()), np.max(np.abs(gpu.geometry() - ref.geometry()))


@pytest.mark.parametrize("solid", [False, True])
def test_colony_in_flow_matches_reference(backend, reference, solid):
    world = colony()
    f = field(solid=solid, seed=3)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    gpu, ref = world.copy(), world.copy()
    backend.set_flow_field(f)
    try:
        rg = backend.advance_contact_dynamics(gpu, None, DT, p)
    finally:
        backend.set_flow_field(None)
    rr = reference.flow_step(ref, f, DT, p)
    assert rg.report.substeps == rr.substeps
    spread = np.max(np.abs(gpu.geometry()[:, :3] - ref.geometry()[:, :3]))
    assert spread < 4 * 5e-4, spread


def test_travel_limit_splits_the_step_as_the_reference(backend, reference):
    world = colony(n=60, seed=7)
    f = field(strength=40.0, solid=False, seed=4)  # drift far beyond a quarter spacing per step
    p = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    gpu, ref = world.copy(), world.copy()
    backend.set_flow_field(f)
    try:
        rg = backend.advance_contact_dynamics(gpu, None, DT, p)
    finally:
        backend.set_flow_field(None)
    rr = reference.flow_step(ref, f, DT, p)
    assert rr.substeps > 1
    assert rg.report.substeps == rr.substeps
    spread = np.max(np.abs(gpu.geometry()[:, :3] - ref.geometry()[:, :3]))
    assert spread < 4 * 5e-4, spread


def test_flow_drift_needs_a_field(backend):
    world = colony(n=20)
    p = ContactDynamicsParameters(flow_drift=True)
    before = world.copy()
    # Simulation::step throws logic_error (simulation.cpp:194), which the
    # reference's bindings raise as RuntimeError.
    with pytest.raises(RuntimeError, match="velocity field"):
        backend.advance_contact_dynamics(world, None, DT, p)
    assert np.array_equal(before.geometry(), world.geometry())
    with pytest.raises(ValueError):
        bad = field()
        bad.x_faces = bad.x_faces.copy()
        bad.x_faces[0, 0, 0] = np.nan
        backend.set_flow_field(bad)


def field_3d(shape=(10, 9, 4), spacing=(2.5, 2.5, 1.5), origin=(-5.0, -5.0, -3.0), seed=2, solid=False):
    """A sheared flow with a vertical component on a 3-D lattice (every face
    of the boundary closed)."""
    sx, sy, sz = shape
    ox, oy, oz = origin
    hx, hy, hz = spacing
    rng = np.random.default_rng(seed)
    xf = np.zeros((sx + 1, sy, sz), np.float32)
    yf = np.zeros((sx, sy + 1, sz), np.float32)
    zf = np.zeros((sx, sy, sz + 1), np.float32)
    for i in range(1, sx):
        for j in range(sy):
            for k in range(sz):
                y, z = oy + (j + 0.5) * hy, oz + (k + 0.5) * hz
                xf[i, j, k] = 0.2 * y + 0.1 * z + 0.02 * rng.standard_normal()
    for i in range(sx):
        for j in range(1, sy):
            for k in range(sz):
                x = ox + (i + 0.5) * hx
                yf[i, j, k] = -0.15 * x + 0.02 * rng.standard_normal()
    for i in range(sx):
        for j in range(sy):
            for k in range(1, sz):
                x = ox + (i + 0.5) * hx
                zf[i, j, k] = 0.05 * x + 0.01 * rng.standard_normal()
    obstacles = None
    if solid:
        obstacles = np.zeros((sx, sy, sz), np.uint8)
        obstacles[6, 2:4, 1:3] = 1
        for i, j, k in np.argwhere(obstacles):
            xf[i, j, k] = xf[i + 1, j, k] = 0.0
            yf[i, j, k] = yf[i, j + 1, k] = 0.0
            zf[i, j, k] = zf[i, j, k + 1] = 0.0
    return FlowField(shape, origin, spacing, xf, yf, zf, obstacles)


@pytest.mark.parametrize("solid", [False, True])
def test_drift_on_a_3d_lattice_is_the_references(backend, reference, solid):
    world = WorldState()
    world.add_cell(position=(1.0, 2.0, 0.5), direction=(0.6, 0.0, 0.8), length=2.5, growth_rate=0.0)
    world.add_cell(position=(8.0, 6.0, -1.0), direction=(0.0, 0.6, 0.8), length=1.5, growth_rate=0.0)
    world.add_cell(position=(12.0, 1.0, 2.2), direction=(1.0, 0.0, 0.0), length=2.0, growth_rate=0.0)
    world.add_cell(position=(-9.0, 30.0, 9.0), direction=(0.0, 1.0, 0.0), length=2.0, growth_rate=0.0)  # clamped
    f = field_3d(solid=solid)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    gpu, ref = world.copy(), world.copy()
    backend.set_flow_field(f)
    try:
        rg = backend.advance_contact_dynamics(gpu, None, DT, p)
    finally:
        backend.set_flow_field(None)
    rr = reference.flow_step(ref, f, DT, p)
    assert rg.report.substeps == rr.substeps
    assert np.max(np.abs(gpu.geometry()[:, 2] - world.geometry()[:, 2])) > 1e-5  # vertical drift too
    assert np.array_equal(gpu.geometry(), ref.geometry()), np.max(np.abs(gpu.geometry() - ref.geometry()))


def line_field(origin, spacing, sites, speed, obstacles=None, x_faces=None):
    """A line of sites along x (closed ends) carrying `speed` on its inner
    faces, as the reference's uniform_flow_grid does on an open line."""
    xf = np.zeros((sites + 1, 1, 1), np.float32)
    if x_faces is None:
        xf[1:sites, 0, 0] = speed
    else:
        xf[:, 0, 0] = x_faces
    yf = np.zeros((sites, 2, 1), np.float32)
    zf = np.zeros((sites, 1, 2), np.float32)
    mask = None if obstacles is None else np.asarray(obstacles, np.uint8).reshape(sites, 1, 1)
    return FlowField((sites, 1, 1), (origin, 0.0, 0.0), (spacing, 1.0, 1.0), xf, yf, zf, mask)


@pytest.mark.parametrize(("origin", "spacing"), [(0.0, 1.0), (0.1, 0.3), (-97.5, 1.65), (0.7, 5.0)])
def test_drift_clamps_at_the_lattice_ends_as_the_reference(backend, reference, origin, spacing):
    """The clamped stencil at and beyond the last site (the reference's
    test_flow_drift_clamps_endpoints_on_any_lattice, test_simulation.py:500-524),
    inside the step: bit-exact against the reference's step."""
    sites = 33
    world = WorldState()
    world.add_cell(position=(origin + spacing * (sites - 1), 0.0, 0.0), direction=(1.0, 0.0, 0.0),
                   length=2.0 * spacing, radius=0.3, growth_rate=0.0)
    world.add_cell(position=(origin + spacing * (sites + 3), 4.0, 0.0), direction=(0.0, 1.0, 0.0),
                   length=2.0 * spacing, radius=0.3, growth_rate=0.0)  # beyond the lattice
    world.add_cell(position=(origin + spacing * 7.3, -3.0, 0.0), direction=(0.6, 0.8, 0.0),
                   length=2.0 * spacing, radius=0.3, growth_rate=0.0)
    f = line_field(origin, spacing, sites, 2.0)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    gpu, ref = world.copy(), world.copy()
    backend.set_flow_field(f)
    try:
        rg = backend.advance_contact_dynamics(gpu, None, 0.1, p)
    finally:
        backend.set_flow_field(None)
    rr = reference.flow_step(ref, f, 0.1, p)
    assert rg.report.substeps == rr.substeps
    assert np.array_equal(gpu.geometry(), ref.geometry()), np.max(np.abs(gpu.geometry() - ref.geometry()))
    assert gpu.position_x[2] > world.position_x[2]  # an interior cell moved with the flow


def test_a_buried_cell_samples_no_flow(backend, reference):
    """A cell pressed into a solid site samples no flow and does not move
    (the reference's test_a_cell_inside_a_wall_samples_no_flow_and_does_not_drift,
    test_simulation.py:569-598), inside the step, bit-exact."""
    f = line_field(0.0, 1.0, 5, 2.0, obstacles=[0, 0, 1, 0, 0], x_faces=[0.0, 2.0, 0.0, 0.0, 2.0, 0.0])
    world = WorldState()
    world.add_cell(position=(2.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0), length=0.0, radius=0.3, growth_rate=0.0)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    gpu, ref = world.copy(), world.copy()
    backend.set_flow_field(f)
    try:
        backend.advance_contact_dynamics(gpu, None, 0.5, p)
    finally:
        backend.set_flow_field(None)
    reference.flow_step(ref, f, 0.5, p)
    assert gpu.position_x[0] == 2.0
    assert np.array_equal(gpu.geometry(), ref.geometry())


def test_flow_carries_cells_inside_the_solve(backend):
    """The reference's test_flow_carries_cells_inside_the_solve
    (python/tests/test_contact_dynamics.py:576-631): a uniform flow of 0.5 on a
    line of 9 sites carries a free cell at its own speed until a fixed cell
    downstream stops it at contact."""
    from microsimulator_b200.simulation import Simulation

    sim = Simulation(backend=backend)
    sites = 9
    xf = np.full((sites + 1, 1, 1), 0.5, np.float32)
    f = FlowField((sites, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), xf, np.zeros((sites, 2, 1), np.float32),
                  np.zeros((sites, 1, 2), np.float32), None)
    free = sim.add_cell(position=(2.0, 0.0, 0.0), length=1.0, radius=0.25, growth_rate=0.0)
    fixed = sim.add_cell(position=(3.6, 0.0, 0.0), length=1.0, radius=0.25, growth_rate=0.0, fixed=True)
    p = ContactDynamicsParameters(flow_drift=True)
    backend.set_flow_field(f)
    try:
        result = sim.step(0.1, p)
        assert abs(sim.cell(free)["position"][0] - 2.05) <= 1e-5
        assert result.center_velocities[sim.cell(free)["slot"]][0] == pytest.approx(0.5)
        assert result.center_velocities[sim.cell(fixed)["slot"]][0] == 0.0
        for _ in range(9):
            result = sim.step(0.1, p)
        stopped = sim.cell(free)["position"][0]
        assert 2.1 - 2e-3 <= stopped <= 2.1 + 2e-3
        assert abs(result.center_velocities[sim.cell(free)["slot"]][0]) < 2e-3
        assert result.report.max_overlap < 2e-3
        assert abs(sim.cell(fixed)["position"][0] - 3.6) <= 1e-6
        sim.step(0.1, ContactDynamicsParameters())
        assert abs(sim.cell(free)["position"][0] - stopped) <= 2e-3
    finally:
        backend.set_flow_field(None)
