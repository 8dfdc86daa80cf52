"""The contact graph oracle (oracle/graph_oracle.py) pinned to the
reference's ContactGraph and ExternalContactGraph constructors: the golden
fixture made from the compiled reference, and live calls on random contact
lists when the reference library is present."""

import numpy as np
import pytest

from microsimulator_b200 import abi
from oracle import graph_oracle
from tests.golden.make_golden import EXTERNAL_ERRORS, GRAPH_ERRORS

KEYS = ("incidence_offsets", "incidence", "neighbor_offsets", "neighbors")


def graph_cases(golden):
    data = golden("contact_graph")
    found = golden("colony_1k")["contacts_0.1"]
    lists = {"found": found, "shuffled": found[data["shuffled__order"]],
             "hand_made": data["hand_made__contacts"], "empty": data["empty__contacts"]}
    return data, lists


def test_oracle_matches_the_reference_graph_fixture(golden):
    data, lists = graph_cases(golden)
    for name, contacts in lists.items():
        result = graph_oracle.contact_graph(contacts, int(data[f"{name}__cell_count"]))
        for key, value in zip(KEYS, result):
            assert np.array_equal(value, data[f"{name}__{key}"]), (name, key)


def test_oracle_matches_the_reference_external_graph_fixture(golden):
    data = golden("contact_graph")
    walls = golden("walls")["walls_1_0.1"]
    for name, contacts in (("walls", walls), ("walls_shuffled", walls[data["walls_shuffled__order"]])):
        offsets, indices = graph_oracle.external_contact_graph(contacts, int(data["cell_count"]))
        assert np.array_equal(offsets, data[f"{name}__incidence_offsets"])
        assert np.array_equal(indices, data[f"{name}__incidence"])


@pytest.mark.parametrize("group", ["cell_error", "external_error"])
def test_oracle_reports_the_references_error_text(golden, group):
    data = golden("contact_graph")
    cell_count = int(data["cell_count"])
    if group == "cell_error":
        errors, base, build = GRAPH_ERRORS, golden("colony_1k")["contacts_0.1"], graph_oracle.contact_graph
    else:
        errors, base, build = EXTERNAL_ERRORS, golden("walls")["walls_1_0.1"], graph_oracle.external_contact_graph
    for (field, value), message in zip(errors, data[f"{group}__messages"]):
        bad = base.copy()
        bad[7][field] = value
        bad[11]["weight"] = -2.0
        with pytest.raises(ValueError) as error:
            build(bad, cell_count)
        assert str(error.value) == message, field


def random_contacts(rng, cells, count):
    """Valid contacts between random slots (ids = slot + 1, canonical order),
    with repeated pairs, in random order."""
    a = rng.integers(0, cells, count)
    b = (a + rng.integers(1, cells, count)) % cells
    first, second = np.minimum(a, b), np.maximum(a, b)
    out = np.zeros(count, dtype=abi.CELL_CONTACT_DTYPE)
    out["first_slot"], out["second_slot"] = first, second
    out["first_id"], out["second_id"] = first + 1 + (1 << 33), second + 1 + (1 << 33)  # ids above 32 bits
    out["ordinal"] = rng.integers(0, 2, count)
    out["normal"] = (0.6, 0.8, 0.0)
    out["weight"] = 1.0
    return out


@pytest.mark.parametrize("cells,count", [(2, 1), (7, 40), (3, 500), (300, 2000), (5000, 400)])
def test_oracle_matches_the_live_reference(reference, cells, count):
    rng = np.random.default_rng(cells + count)
    contacts = random_contacts(rng, cells, count)
    ours = graph_oracle.contact_graph(contacts, cells + 3)
    theirs = reference.contact_graph(contacts, cells + 3)
    for key, mine, other in zip(KEYS, ours, theirs):
        assert np.array_equal(mine, other), key


def test_oracle_rejects_the_slot_index_space_as_the_reference():
    with pytest.raises(OverflowError):
        graph_oracle.contact_graph(np.zeros(0, dtype=abi.CELL_CONTACT_DTYPE), 1 << 32)
