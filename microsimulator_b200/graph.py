"""Contact graphs as the reference's Python bindings expose them
(cpp/python/bindings.cpp:464-485 ``ContactGraph``, :587-602
``ExternalContactGraph``): the contact records plus, per slot, the indices
of its contacts in contact order and (cell contacts) its distinct partner
ids in ascending order.  The index arrays come from the device
(``msb_build_contact_graph``, ``msb_find_cell_contact_graph``,
``msb_build_external_contact_graph``); this module only holds and slices
them.
"""

from __future__ import annotations

import numpy as np


class ExternalContactGraph:
    """ExternalContactGraph (cpp/include/microsimulator/constraints.hpp:160-178)."""

    _incidence_range = "external contact incidence slot is out of range"

    def __init__(self, cell_count: int, contacts: np.ndarray, incidence_offsets: np.ndarray,
                 incidence_contacts: np.ndarray):
        self._cell_count = int(cell_count)
        self.contacts = contacts
        self.incidence_offsets = incidence_offsets
        self.incidence_contacts = incidence_contacts

    @property
    def cell_count(self) -> int:
        return self._cell_count

    @property
    def empty(self) -> bool:
        return len(self.contacts) == 0

    def __len__(self) -> int:
        return len(self.contacts)

    def _slot(self, slot: int, message: str) -> int:
        index = int(slot)
        if index < 0 or index >= self._cell_count:
            raise IndexError(message)
        return index

    def incident_contact_indices(self, slot: int) -> list[int]:
        """The indices of the contacts that touch `slot`, in contact order
        (contact_graph.cpp:376-384, constraints.cpp:325-333)."""
        s = self._slot(slot, self._incidence_range)
        return self.incidence_contacts[self.incidence_offsets[s]:self.incidence_offsets[s + 1]].tolist()


class ContactGraph(ExternalContactGraph):
    """ContactGraph (cpp/include/microsimulator/contact_graph.hpp:40-63)."""

    _incidence_range = "contact incidence slot is out of range"

    def __init__(self, cell_count: int, contacts: np.ndarray, incidence_offsets: np.ndarray,
                 incidence_contacts: np.ndarray, neighbor_offsets: np.ndarray, neighbor_ids: np.ndarray):
        super().__init__(cell_count, contacts, incidence_offsets, incidence_contacts)
        self.neighbor_offsets = neighbor_offsets
        self.packed_neighbor_ids = neighbor_ids

    def neighbor_ids(self, slot: int) -> list[int]:
        """The distinct ids of the cells touching `slot`, ascending
        (contact_graph.cpp:386-394)."""
        s = self._slot(slot, "contact neighbor slot is out of range")
        return self.packed_neighbor_ids[self.neighbor_offsets[s]:self.neighbor_offsets[s + 1]].tolist()


def device_index(cell_count: int, entries: int, device):
    """Device arrays for a graph index (torch int64 tensors on `device`) and
    the msb_contact_graph_index that points at them, for calls with
    device_pointers = 1.  Returns (index, tensors)."""
    import torch

    from . import abi

    tensors = {name: torch.zeros(max(1, size), dtype=torch.int64, device=device) for name, size in (
        ("incidence_offsets", cell_count + 1), ("incidence_contacts", entries), ("neighbor_offsets", cell_count + 1),
        ("neighbor_ids", entries))}
    index = abi.ContactGraphIndex()
    for name, tensor in tensors.items():
        setattr(index, name, tensor.data_ptr())
    index.neighbor_capacity = entries
    return index, tensors
