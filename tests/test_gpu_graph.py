"""The contact graph index on the device (msb_build_contact_graph,
msb_find_cell_contact_graph, msb_build_external_contact_graph) against the
reference constructors' golden fixture and the numpy oracle: incidence and
neighbour arrays equal element for element, the reference's error texts, and
the reference's Python-level ContactGraph behaviour."""

import numpy as np
import pytest

from microsimulator_b200 import abi, workloads
from microsimulator_b200.simulation import Simulation
from microsimulator_b200.types import ContactParameters
from oracle import graph_oracle
from tests.golden.make_golden import EXTERNAL_ERRORS, GRAPH_ERRORS
from tests.test_oracle_graph import graph_cases, random_contacts

pytestmark = pytest.mark.gpu


def assert_graph(graph, expected, count):
    offsets, incidence, neighbor_offsets, neighbors = expected
    assert np.array_equal(graph.incidence_offsets, offsets)
    assert np.array_equal(graph.incidence_contacts, incidence)
    assert np.array_equal(graph.neighbor_offsets, neighbor_offsets)
    assert np.array_equal(graph.packed_neighbor_ids, neighbors)
    assert len(graph) == count


def test_graph_of_fixture_lists_is_the_references(backend, golden):
    data, lists = graph_cases(golden)
    for name, contacts in lists.items():
        cell_count = int(data[f"{name}__cell_count"])
        graph = backend.build_contact_graph(contacts, cell_count)
        expected = [data[f"{name}__{key}"] for key in ("incidence_offsets", "incidence", "neighbor_offsets",
                                                       "neighbors")]
        assert_graph(graph, expected, len(contacts))
        assert graph.cell_count == cell_count


def test_found_contact_graph_is_the_references(backend, golden):
    data, lists = graph_cases(golden)
    colony = golden("colony_1k")
    from tests.golden.make_golden import world_from

    world = world_from(colony, "world__")
    graph = backend.find_cell_contact_graph(world, ContactParameters(activation_margin=0.1))
    assert np.array_equal(graph.contacts.view(np.uint8), lists["found"].view(np.uint8))
    expected = [data[f"found__{key}"] for key in ("incidence_offsets", "incidence", "neighbor_offsets",
                                                  "neighbors")]
    assert_graph(graph, expected, len(lists["found"]))


def test_external_graph_is_the_references(backend, golden):
    data = golden("contact_graph")
    walls = golden("walls")["walls_1_0.1"]
    for name, contacts in (("walls", walls), ("walls_shuffled", walls[data["walls_shuffled__order"]])):
        graph = backend.build_external_contact_graph(contacts, int(data["cell_count"]))
        assert np.array_equal(graph.incidence_offsets, data[f"{name}__incidence_offsets"])
        assert np.array_equal(graph.incidence_contacts, data[f"{name}__incidence"])


@pytest.mark.parametrize("group", ["cell_error", "external_error"])
def test_invalid_contacts_raise_the_references_text(backend, golden, group):
    data = golden("contact_graph")
    cell_count = int(data["cell_count"])
    if group == "cell_error":
        errors, base, build = GRAPH_ERRORS, golden("colony_1k")["contacts_0.1"], backend.build_contact_graph
    else:
        errors, base, build = EXTERNAL_ERRORS, golden("walls")["walls_1_0.1"], backend.build_external_contact_graph
    for (field, value), message in zip(errors, data[f"{group}__messages"]):
        bad = base.copy()
        bad[7][field] = value
        bad[11]["weight"] = -2.0
        with pytest.raises(ValueError) as error:
            build(bad, cell_count)
        assert str(error.value) == message, field


# (3, 500) and (40, 3000) put more than 64 entries in a slot: the radix path.
@pytest.mark.parametrize("cells,count", [(2, 1), (7, 40), (3, 500), (40, 3000), (300, 2000), (5000, 400),
                                         (70_000, 300_000)])
def test_random_lists_match_the_oracle(backend, cells, count):
    rng = np.random.default_rng(cells + count)
    contacts = random_contacts(rng, cells, count)
    graph = backend.build_contact_graph(contacts, cells + 3)
    assert_graph(graph, graph_oracle.contact_graph(contacts, cells + 3), count)


@pytest.mark.parametrize("hub", [64, 65])
def test_segment_limit(backend, hub):
    """A slot with exactly the per-slot sort's limit of entries, and one more."""
    rng = np.random.default_rng(hub)
    contacts = random_contacts(rng, 2000, 3000)
    spokes = random_contacts(rng, 2000, hub)
    spokes["first_slot"], spokes["first_id"] = 0, 1 + (1 << 33)
    spokes["second_slot"] = np.arange(1, hub + 1)
    spokes["second_id"] = spokes["second_slot"].astype(np.uint64) + 1 + (1 << 33)
    contacts = contacts[(contacts["first_slot"] != 0) & (contacts["second_slot"] != 0)]
    contacts = np.concatenate([contacts[:1000], spokes, contacts[1000:]])
    graph = backend.build_contact_graph(contacts, 2000)
    assert len(graph.incident_contact_indices(0)) == hub
    assert_graph(graph, graph_oracle.contact_graph(contacts, 2000), len(contacts))


def test_large_colony_graph_matches_the_oracle(backend):
    world = workloads.jammed(200_000, seed=3)
    graph = backend.find_cell_contact_graph(world, ContactParameters(activation_margin=0.05))
    assert len(graph) > 300_000
    assert_graph(graph, graph_oracle.contact_graph(graph.contacts, len(world)), len(graph.contacts))
    # size-independent properties: every contact listed under both its slots,
    # each neighbour list strictly ascending
    assert graph.incidence_offsets[-1] == 2 * len(graph)
    for slot in range(0, len(world), 997):
        ids = graph.neighbor_ids(slot)
        assert all(a < b for a, b in zip(ids, ids[1:]))


def test_device_pointers(backend):
    torch = pytest.importorskip("torch")
    import ctypes

    rng = np.random.default_rng(5)
    contacts = random_contacts(rng, 1000, 5000)
    cells = 1000
    device = torch.device("cuda", 0)
    records = torch.from_numpy(contacts.view(np.uint8).copy()).to(device)
    arrays = {name: torch.zeros(n, dtype=torch.int64, device=device) for name, n in (
        ("incidence_offsets", cells + 1), ("incidence_contacts", 2 * len(contacts)),
        ("neighbor_offsets", cells + 1), ("neighbor_ids", 2 * len(contacts)))}
    index = abi.ContactGraphIndex()
    for name, tensor in arrays.items():
        setattr(index, name, tensor.data_ptr())
    index.neighbor_capacity = 2 * len(contacts)
    torch.cuda.synchronize()
    backend._check(backend._lib.msb_build_contact_graph(backend._handle, records.data_ptr(), len(contacts), cells, 1,
                                                       ctypes.byref(index)))
    expected = graph_oracle.contact_graph(contacts, cells)
    got = [arrays[name].cpu().numpy().view(np.uint64) for name in ("incidence_offsets", "incidence_contacts",
                                                                    "neighbor_offsets", "neighbor_ids")]
    got[3] = got[3][: index.neighbor_count]
    for mine, other in zip(got, expected):
        assert np.array_equal(mine, other)


def test_neighbor_capacity_is_reported(backend):
    import ctypes

    contacts = random_contacts(np.random.default_rng(9), 50, 300)
    graph = graph_oracle.contact_graph(contacts, 50)
    offsets = np.zeros(51, dtype=np.uint64)
    incidence = np.zeros(600, dtype=np.uint64)
    neighbor_offsets = np.zeros(51, dtype=np.uint64)
    neighbors = np.zeros(4, dtype=np.uint64)
    index = abi.ContactGraphIndex()
    index.incidence_offsets, index.incidence_contacts = abi.ptr(offsets), abi.ptr(incidence)
    index.neighbor_offsets, index.neighbor_ids = abi.ptr(neighbor_offsets), abi.ptr(neighbors)
    index.neighbor_capacity = 4
    status = backend._lib.msb_build_contact_graph(backend._handle, ctypes.c_void_p(abi.ptr(contacts)), len(contacts),
                                                  50, 0, ctypes.byref(index))
    assert status == abi.ERR_CAPACITY
    assert index.neighbor_count == len(graph[3])


def test_contact_graph_through_the_simulation_api(backend):
    """The reference's test_contact_graph_is_available_through_the_public_api
    (python/tests/test_simulation.py:243-271), on this backend."""
    sim = Simulation(backend=backend)
    sim.add_cell(position=(0.0, 0.0, 0.0), length=4.0, radius=0.5)
    sim.add_cell(position=(0.0, 0.8, 0.0), length=4.0, radius=0.5)
    graph = sim.find_cell_contacts(ContactParameters())
    assert graph.cell_count == 2
    assert not graph.empty
    assert len(graph) == 2
    assert graph.incident_contact_indices(0) == [0, 1]
    assert graph.neighbor_ids(0) == [2]
    assert graph.neighbor_ids(1) == [1]
    assert graph.contacts["ordinal"].tolist() == [0, 1]
    assert np.allclose(graph.contacts["signed_separation"], -0.2, atol=1e-6)
    with pytest.raises(IndexError):
        graph.neighbor_ids(2)
    with pytest.raises(IndexError):
        graph.incident_contact_indices(5)


def test_slot_index_space_and_empty_graphs(backend):
    import ctypes

    empty = np.zeros(0, dtype=abi.CELL_CONTACT_DTYPE)
    graph = backend.build_contact_graph(empty, 0)
    assert graph.cell_count == 0 and graph.empty and graph.incidence_offsets.tolist() == [0]
    graph = backend.build_contact_graph(empty, 5)
    assert graph.incidence_offsets.tolist() == [0] * 6 and graph.neighbor_ids(4) == []
    # checked_offset_count (contact_graph.cpp:209-215): beyond the slot index space.
    index = abi.ContactGraphIndex()
    status = backend._lib.msb_build_contact_graph(backend._handle, None, 0, (1 << 32), 0, ctypes.byref(index))
    assert status == abi.ERR_OVERFLOW
    external = np.zeros(0, dtype=abi.EXTERNAL_CONTACT_DTYPE)
    assert backend.build_external_contact_graph(external, 3).incidence_offsets.tolist() == [0, 0, 0, 0]


def test_plane_constraint_graph_through_the_simulation_api(backend):
    """The reference's test_plane_constraint_graph_is_typed_and_incident
    (python/tests/test_simulation.py:323-357), on this backend."""
    sim = Simulation(backend=backend)
    cell_id = sim.add_cell(position=(0.0, 0.25, 0.0), length=2.0, radius=0.5)
    constraint_id = sim.add_plane_constraint(point=(0.0, 0.0, 0.0), inward_normal=(0.0, 2.0, 0.0), coefficient=3.0)
    graph = sim.find_external_contacts()
    assert graph.cell_count == 1
    assert len(graph) == 2
    assert graph.incident_contact_indices(0) == [0, 1]
    assert np.all(graph.contacts["cell_id"] == cell_id)
    assert np.all(graph.contacts["constraint_id"] == constraint_id)
    assert np.all(graph.contacts["constraint_kind"] == abi.CONSTRAINT_PLANE)
    assert graph.contacts["location"].tolist() == [abi.ROD_NEGATIVE, abi.ROD_POSITIVE]
    assert np.allclose(graph.contacts["signed_separation"], -0.25)
    assert np.allclose(graph.contacts["normal"][:, 1], -1.0)
    assert np.allclose(graph.contacts["point_on_cell"][:, 1], -0.25)
    assert np.allclose(graph.contacts["weight"], 3.0 / np.sqrt(2.0), rtol=1e-6)


def test_found_external_graph_is_the_references(backend, golden):
    from tests.golden.make_golden import wall_set, world_from
    from microsimulator_b200.types import ConstraintContactParameters

    data = golden("contact_graph")
    world = world_from(golden("colony_1k"), "world__")
    graph = backend.find_external_contact_graph(world, wall_set(), ConstraintContactParameters(0.1), every_face=True)
    assert graph.contacts.tobytes() == golden("walls")["walls_1_0.1"].tobytes()
    assert np.array_equal(graph.incidence_offsets, data["walls__incidence_offsets"])
    assert np.array_equal(graph.incidence_contacts, data["walls__incidence"])


def reference_graph_equal(backend, reference, world, parameters=None):
    """The backend's ContactGraph of `world` equals the reference CPU
    backend's: contacts bit for bit, incidence exactly
    (contact_conformance_test.cpp's compare_graphs at zero tolerance)."""
    parameters = parameters or ContactParameters()
    graph = backend.find_cell_contact_graph(world, parameters)
    expected = reference.find_cell_contacts(world, parameters)
    offsets, indices = reference.incidence(world, parameters)
    assert graph.contacts.tobytes() == expected.tobytes()
    assert np.array_equal(graph.incidence_offsets, offsets)
    assert np.array_equal(graph.incidence_contacts, indices)
    return graph


def capsules(*specs):
    from microsimulator_b200.world import WorldState

    w = WorldState()
    for center, axis, *length in specs:
        w.add_cell(position=center, direction=axis, length=length[0] if length else 2.0, radius=0.5)
    return w


def test_contact_conformance_fixtures(backend, reference):
    """The reference's contact conformance test
    (tests/conformance/contact_conformance_test.cpp:55-160): mixed geometry,
    31 coincident capsules (930 contacts, 60 incident on the first), margins
    and buffer reuse, and the ids after a division."""
    mixed = capsules(((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 4.0), ((0.0, 0.8, 0.0), (-1.0, 0.0, 0.0), 4.0),
                     ((4.9, 0.0, 0.0), (1.0, 0.0, 0.0), 4.0), ((10.0, 0.0, 0.0), (1.0, 0.0, 0.0)),
                     ((10.0, 0.0, 0.0), (0.0, 1.0, 0.0)), ((15.0, 0.0, 0.0), (1.0, 0.0, 0.0), 0.0),
                     ((15.0, 0.8, 0.0), (1.0, 0.0, 0.0), 0.0))
    reference_graph_equal(backend, reference, mixed)

    dense = capsules(*[((0.0, 0.0, 0.0), (1.0, 0.0, 0.0))] * 31)
    graph = reference_graph_equal(backend, reference, dense)
    assert len(graph) == 930
    assert len(graph.incident_contact_indices(0)) == 60

    reuse = capsules(((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 0.0), ((1.005, 0.0, 0.0), (1.0, 0.0, 0.0), 0.0))
    strict = reference_graph_equal(backend, reference, reuse, ContactParameters(activation_margin=0.0))
    assert strict.empty
    reference_graph_equal(backend, reference, reuse)
    reuse.add_cell(position=(0.5, 0.0, 0.0), direction=(1.0, 0.0, 0.0), length=0.0, radius=0.5)
    reference_graph_equal(backend, reference, reuse)

    divided = capsules(((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 4.0), ((0.0, 0.2, 0.0), (1.0, 0.0, 0.0), 4.0))
    divided.divide_many([int(divided.ids[0])], 0.5)
    reference_graph_equal(backend, reference, divided)
