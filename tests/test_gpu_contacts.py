"""Contact detection on the GPU through the C-ABI, against the reference's
golden fixtures and the FP32 oracle: pair lists, separations, points,
normals and weights bit-exact."""

import numpy as np
import pytest

from microsimulator_b200 import abi, workloads
from microsimulator_b200.types import ConstraintContactParameters, ContactParameters
from microsimulator_b200.world import ConstraintSet, WorldState
from tests.golden.make_golden import wall_set, world_from

pytestmark = pytest.mark.gpu


def test_geometry_kats_bit_exact(backend, golden):
    data = golden("geometry_kat")
    for name in data["names"]:
        world = world_from(data, f"{name}__")
        for margin in (0.01, 0.1):
            expected = data[f"{name}__contacts_{margin}"]
            actual = backend.find_cell_contacts(world, ContactParameters(activation_margin=margin))
            assert actual.tobytes() == expected.tobytes(), (name, margin)


def test_empty_and_single_cell(backend):
    assert len(backend.find_cell_contacts(WorldState())) == 0
    w = WorldState()
    w.add_cell((0, 0, 0), (1, 0, 0), 2.0, 0.5)
    assert len(backend.find_cell_contacts(w)) == 0


def test_grid_matches_exhaustive_257(backend, golden):
    data = golden("pseudo_random_257")
    world = world_from(data, "world__")
    for margin in (0.0, 0.01, 0.5):
        actual = backend.find_cell_contacts(world, ContactParameters(activation_margin=margin))
        assert actual.tobytes() == data[f"contacts_{margin}"].tobytes()


def test_colony_contacts_and_incidence(backend, golden):
    data = golden("colony_1k")
    world = world_from(data, "world__")
    actual = backend.find_cell_contacts(world, ContactParameters(activation_margin=0.1))
    assert actual.tobytes() == data["contacts_0.1"].tobytes()
    graph = backend.find_cell_contact_graph(world, ContactParameters(activation_margin=0.1))
    assert graph.contacts.tobytes() == data["contacts_0.1"].tobytes()
    assert np.array_equal(graph.incidence_offsets, data["incidence_offsets"])
    assert np.array_equal(graph.incidence_contacts, data["incidence_indices"])


def test_walls_bit_exact(backend, golden):
    data = golden("walls")
    world = world_from(golden("colony_1k"), "world__")
    cs = wall_set()
    for every_face in (0, 1):
        for margin in (0.0, 0.1):
            actual = backend.find_external_contacts(world, cs, ConstraintContactParameters(margin),
                                                    every_face=bool(every_face))
            assert actual.tobytes() == data[f"walls_{every_face}_{margin}"].tobytes(), (every_face, margin)


def test_dense_pile_many_partners(backend, oracle):
    # More than 32 partners per cell takes the global-memory sort.
    w = WorldState()
    rng = np.random.default_rng(1)
    for k in range(80):
        w.add_cell(tuple(rng.uniform(-0.3, 0.3, 3)), tuple(rng.normal(size=3)), 2.0, 0.5)
    expected = oracle.find_cell_contacts(w, ContactParameters(activation_margin=0.1))
    actual = backend.find_cell_contacts(w, ContactParameters(activation_margin=0.1))
    assert actual.tobytes() == expected.tobytes()


def test_sparse_cells_use_hashed_grid(backend, oracle):
    # Cells spread so thinly that a dense grid would exceed 8N + 4096 boxes.
    w = WorldState()
    rng = np.random.default_rng(2)
    pos = rng.uniform(-5000, 5000, (3000, 3))
    pos[:10] = [(0.1 * k, 0, 0) for k in range(10)]
    w = WorldState.from_arrays(pos, rng.normal(size=(3000, 3)), 2.0, 0.5)
    expected = oracle.find_cell_contacts(w, ContactParameters(activation_margin=0.1))
    actual = backend.find_cell_contacts(w, ContactParameters(activation_margin=0.1))
    assert len(expected) > 0
    assert actual.tobytes() == expected.tobytes()


def test_ids_out_of_slot_order_and_wide_ids(backend, oracle):
    world = workloads.colony_1k(seed=11, n=2000, side=60.0)
    rng = np.random.default_rng(3)
    world.ids = (rng.permutation(len(world)).astype(np.uint64) + np.uint64(1)) * np.uint64(3_000_000_007)
    expected = oracle.find_cell_contacts(world, ContactParameters(activation_margin=0.1))
    actual = backend.find_cell_contacts(world, ContactParameters(activation_margin=0.1))
    assert actual.tobytes() == expected.tobytes()


@pytest.mark.parametrize("n", [20_000, 200_000])
def test_jammed_colony_contacts_bit_exact(backend, oracle, n):
    world = workloads.jammed(n=n, seed=5)
    for margin in (0.0, 0.1):
        expected = oracle.find_cell_contacts(world, ContactParameters(activation_margin=margin))
        actual = backend.find_cell_contacts(world, ContactParameters(activation_margin=margin))
        assert actual.tobytes() == expected.tobytes()


def test_trap_walls_bit_exact(backend, oracle):
    world, cs = workloads.trap_colony(n=5000, seed=4)
    for every_face in (False, True):
        expected = oracle.find_external_contacts(world, cs, ConstraintContactParameters(0.1), every_face=every_face)
        actual = backend.find_external_contacts(world, cs, ConstraintContactParameters(0.1), every_face=every_face)
        assert actual.tobytes() == expected.tobytes()


def test_invalid_inputs_raise(backend):
    w = WorldState()
    w.add_cell((0, 0, 0), (1, 0, 0), 2.0, 0.5)
    w.add_cell((1, 0, 0), (1, 0, 0), 2.0, 0.5)
    with pytest.raises(ValueError):
        backend.find_cell_contacts(w, ContactParameters(parallel_sine_threshold=2.0))
    w.ids[1] = w.ids[0]
    with pytest.raises(ValueError):
        backend.find_cell_contacts(w)
    w.ids[1] = 2
    w.position_x[0] = np.nan
    with pytest.raises(ValueError):
        backend.find_cell_contacts(w)


@pytest.mark.parametrize("field,value", [("b", (0.0, 2.0, 0.0)), ("coefficient", 0.0), ("radius", -1.0),
                                         ("allowed_region", 7)])
def test_invalid_constraint_records_raise(backend, field, value):
    """Constraint records meet ConstraintSet's checks (constraints.cpp:17-80):
    a plane's inward normal normalized, a positive coefficient, positive
    radii, a known region.  A record that does not is an error, not a
    silently different wall."""
    w = WorldState()
    w.add_cell((0, 0.25, 0), (1, 0, 0), 2.0, 0.5)
    cs = ConstraintSet()
    cs.add_plane(point=(0.0, 0.0, 0.0), inward_normal=(0.0, 1.0, 0.0))
    cs.add_sphere(center=(5.0, 0.0, 0.0), radius=1.0)
    target = 1 if field == "radius" or field == "allowed_region" else 0
    cs.records[target][field] = value
    with pytest.raises(ValueError):
        backend.find_external_contacts(w, cs)


def test_constraint_conformance_fixtures(backend, reference):
    """The reference's constraint conformance test
    (tests/conformance/constraint_conformance_test.cpp:155-240): every fixture's
    ExternalContactGraph equal to the reference's (its contacts bit for bit,
    its incidence exactly), and the empty inputs."""
    from tests.constraint_fixtures import FIXTURES

    for name, build in FIXTURES.items():
        world, constraints = build()
        expected = reference.find_external_contacts(world, constraints)
        offsets, indices = reference.external_contact_graph(expected, len(world))
        graph = backend.find_external_contact_graph(world, constraints)
        assert graph.contacts.tobytes() == expected.tobytes(), name
        assert np.array_equal(graph.incidence_offsets, offsets), name
        assert np.array_equal(graph.incidence_contacts, indices), name
    empty = backend.find_external_contact_graph(WorldState(), ConstraintSet())
    assert empty.empty and empty.cell_count == 0
    one = WorldState()
    one.add_cell((0, 0, 0), (1, 0, 0), 1.0, 0.5)
    graph = backend.find_external_contact_graph(one, ConstraintSet())
    assert graph.empty and graph.cell_count == 1
