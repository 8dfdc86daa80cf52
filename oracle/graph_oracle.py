"""Test infrastructure: a numpy restatement of the contact graph index, the
checker of the device graph build (tests only; the product never imports it).

Follows the reference's constructors:
  * ContactGraph(cell_count, contacts)   cpp/core/contact_graph.cpp:302-349
      validate_contact                   contact_graph.cpp:217-237
      checked_offset_count               contact_graph.cpp:209-215
  * ExternalContactGraph(...)            cpp/core/constraints.cpp:288-307
      validate_contact                   constraints.cpp:126-145

Pinned against the reference's own constructors: tests/golden/contact_graph.npz
(made by tests/golden/make_golden.py from the compiled reference) and live
calls when the reference library is present (tests/test_oracle_graph.py).
"""

from __future__ import annotations

import numpy as np

CELL_REASONS = (
    None,
    "contact cell identifiers are not canonical",
    "contact slots are invalid",
    "cell contact ordinal exceeds the capsule-pair contract",
    "contact contains a non-finite or invalid field",
    "contact normal is not unit length",
)
EXTERNAL_REASONS = (
    None,
    "external contact has an invalid identity",
    "external contact cell slot is invalid",
    "external contact contains an invalid tag",
    "external contact contains a non-finite or invalid field",
    "external contact normal is not unit length",
)

_MAX_SLOT = 0xFFFFFFFF


def _finite(v: np.ndarray) -> np.ndarray:
    return np.all(np.isfinite(v), axis=1)


def _unit(normal: np.ndarray) -> np.ndarray:
    """|norm(n) - 1| <= 1e-4 in FP32 as types.hpp's norm: sqrt((x*x + y*y) + z*z)."""
    n = normal.astype(np.float32)
    square = (n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]
    with np.errstate(invalid="ignore"):
        return ~(np.abs(np.sqrt(square) - np.float32(1.0)) > np.float32(1.0e-4))


def _first_failure(checks, reasons) -> None:
    """Raises the reason of the lowest contact failing a check; `checks` are
    the per-contact failure masks in the reference's order of checks."""
    count = len(checks[0]) if checks else 0
    reason = np.zeros(count, dtype=np.int64)
    for code, failed in enumerate(checks, start=1):
        reason = np.where((reason == 0) & failed, code, reason)
    bad = np.flatnonzero(reason)
    if len(bad):
        raise ValueError(reasons[int(reason[bad[0]])])


def _check_cell_count(cell_count: int) -> None:
    if cell_count > _MAX_SLOT:
        raise OverflowError("contact graph exceeds the slot index space")


def validate_cell_contacts(contacts: np.ndarray, cell_count: int) -> None:
    f, s = contacts["first_id"].astype(np.uint64), contacts["second_id"].astype(np.uint64)
    a, b = contacts["first_slot"].astype(np.uint64), contacts["second_slot"].astype(np.uint64)
    point, normal = contacts["point_on_first"], contacts["normal"]
    sep, weight = contacts["signed_separation"], contacts["weight"]
    with np.errstate(invalid="ignore"):
        invalid_field = ~_finite(point) | ~_finite(normal) | ~np.isfinite(sep) | ~np.isfinite(weight) | ~(weight > 0)
    _first_failure([
        (f == 0) | (s == 0) | (f >= s),
        (a >= cell_count) | (b >= cell_count) | (a == b),
        contacts["ordinal"] > 1,
        invalid_field,
        ~_unit(normal),
    ], CELL_REASONS)


def validate_external_contacts(contacts: np.ndarray, cell_count: int) -> None:
    point, normal = contacts["point_on_cell"], contacts["normal"]
    sep, weight = contacts["signed_separation"], contacts["weight"]
    with np.errstate(invalid="ignore"):
        invalid_field = ~_finite(point) | ~_finite(normal) | ~np.isfinite(sep) | ~np.isfinite(weight) | ~(weight > 0)
    _first_failure([
        (contacts["cell_id"] == 0) | (contacts["constraint_id"] == 0),
        contacts["cell_slot"].astype(np.uint64) >= cell_count,
        (contacts["constraint_kind"] > 3) | (contacts["location"] > 2),
        invalid_field,
        ~_unit(normal),
    ], EXTERNAL_REASONS)


def _offsets(slots: np.ndarray, cell_count: int) -> np.ndarray:
    offsets = np.zeros(cell_count + 1, dtype=np.uint64)
    if len(slots):
        np.cumsum(np.bincount(slots.astype(np.int64), minlength=cell_count), out=offsets[1:])
    return offsets


def contact_graph(contacts: np.ndarray, cell_count: int):
    """(incidence offsets, incidence contact indices, neighbour offsets,
    neighbour ids) of ContactGraph(cell_count, contacts)."""
    _check_cell_count(cell_count)
    validate_cell_contacts(contacts, cell_count)
    count = len(contacts)
    # The constructor's cursor fill: contact order within each slot.
    slots = np.stack([contacts["first_slot"], contacts["second_slot"]], 1).reshape(-1).astype(np.int64)
    entries = np.repeat(np.arange(count, dtype=np.uint64), 2)
    order = np.argsort(slots, kind="stable")
    incidence_offsets = _offsets(slots, cell_count)
    incidence = entries[order]
    # Each slot's partner ids, sorted and made unique.
    partners = np.stack([contacts["second_id"], contacts["first_id"]], 1).reshape(-1).astype(np.uint64)
    by_slot = np.lexsort((partners, slots))
    s, p = slots[by_slot], partners[by_slot]
    first = np.ones(len(s), dtype=bool)
    if len(s) > 1:
        first[1:] = (s[1:] != s[:-1]) | (p[1:] != p[:-1])
    neighbor_offsets = _offsets(s[first], cell_count)
    return incidence_offsets, incidence, neighbor_offsets, p[first]


def external_contact_graph(contacts: np.ndarray, cell_count: int):
    """(incidence offsets, incidence contact indices) of
    ExternalContactGraph(cell_count, contacts)."""
    _check_cell_count(cell_count)
    validate_external_contacts(contacts, cell_count)
    slots = contacts["cell_slot"].astype(np.int64)
    order = np.argsort(slots, kind="stable")
    return _offsets(slots, cell_count), np.arange(len(contacts), dtype=np.uint64)[order]
