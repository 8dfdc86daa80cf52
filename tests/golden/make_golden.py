"""Generates the golden fixtures of the contact path from the reference
MicroSimulator CPU backend (oracle/_ref/libmsref.so, compiled from the
reference's own sources by oracle/Makefile).

Run from the repository root:  python tests/golden/make_golden.py

Cases (each saved as an .npz of input arrays and the reference's outputs):
  geometry_kat      the capsule layouts of the reference's contact geometry
                    tests (tests/cpp/contact_geometry_test.cpp:28-244)
  pseudo_random_257 the 257-capsule layout of its grid-vs-exhaustive test
                    (contact_geometry_test.cpp:174-203) at margins 0, 0.01, 0.5
  colony_1k         1,000 capsules, lengths U[2, 4], 40 x 40 um, seed 42,
                    contacts at margin 0.1 and one contact-dynamics step
  walls             colony_1k against planes, spheres, boxes and cylinders
                    inside and outside, nearest-face and every-face contacts
  chain_*           the make_chain solves of the reference's dynamics
                    conformance test (tests/conformance/contact_dynamics_conformance_test.cpp:56-109)
  contact_graph     ContactGraph / ExternalContactGraph index arrays
                    (cpp/core/contact_graph.cpp:302-349, constraints.cpp:288-307)
                    of colony_1k's contacts and walls, as found and shuffled,
                    a hand-made list with repeated partners and empty slots,
                    and the reference's error text for invalid contacts

``python tests/golden/make_golden.py contact_graph`` makes only the named cases.
"""

from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from microsimulator_b200 import abi, workloads  # noqa: E402
from microsimulator_b200.types import (  # noqa: E402
    ConstraintContactParameters,
    ContactDynamicsParameters,
    ContactParameters,
    ContactSolveParameters,
    ContactSystem,
    GrowthLoadResponse,
)
from microsimulator_b200.world import ConstraintSet, WorldState  # noqa: E402

OUT = Path(__file__).resolve().parent


def world_arrays(world: WorldState) -> dict:
    return {
        "ids": world.ids,
        "positions": np.stack([world.position_x, world.position_y, world.position_z], 1),
        "directions": np.stack([world.direction_x, world.direction_y, world.direction_z], 1),
        "lengths": world.lengths,
        "radii": world.radii,
        "growth_rates": world.growth_rates,
        "fixed": world.fixed,
    }


def world_from(data, prefix="") -> WorldState:
    w = WorldState()
    w.ids = np.ascontiguousarray(data[prefix + "ids"])
    p = data[prefix + "positions"]
    d = data[prefix + "directions"]
    w.position_x, w.position_y, w.position_z = (np.ascontiguousarray(p[:, k]) for k in range(3))
    w.direction_x, w.direction_y, w.direction_z = (np.ascontiguousarray(d[:, k]) for k in range(3))
    w.lengths = np.ascontiguousarray(data[prefix + "lengths"])
    w.radii = np.ascontiguousarray(data[prefix + "radii"])
    w.growth_rates = np.ascontiguousarray(data[prefix + "growth_rates"])
    w.fixed = np.ascontiguousarray(data[prefix + "fixed"])
    w.next_id = int(w.ids.max()) + 1 if len(w.ids) else 1
    return w


def geometry_kat_worlds() -> dict[str, WorldState]:
    """The layouts of contact_geometry_test.cpp (add_capsule with length 2,
    radius 0.5 unless stated)."""
    def make(specs):
        w = WorldState()
        for spec in specs:
            center, axis = spec[0], spec[1]
            length = spec[2] if len(spec) > 2 else 2.0
            radius = spec[3] if len(spec) > 3 else 0.5
            w.add_cell(center, axis, length, radius, 1.0)
        return w

    worlds = {
        "separated": make([((0, 0, 0), (1, 0, 0)), ((4, 0, 0), (1, 0, 0))]),
        "end_on": make([((0, 0, 0), (1, 0, 0)), ((2.9, 0, 0), (1, 0, 0))]),
        "parallel": make([((0, 0, 0), (1, 0, 0), 4.0), ((0, 0.8, 0), (1, 0, 0), 4.0)]),
        "skew": make([((0, 0, 0), (1, 0, 0)), ((0, 0, 0), (0, 1, 0))]),
        "coincident": make([((0, 0, 0), (1, 0, 0), 4.0), ((0, 0, 0), (-1, 0, 0), 4.0)]),
        "dense31": make([((0, 0, 0), (1, 0, 0))] * 31),
        "forward": make([((0, 0, 0), (1, 0, 0), 4.0), ((0, 0.8, 0), (-1, 0, 0), 4.0)]),
        "reversed": make([((0, 0.8, 0), (-1, 0, 0), 4.0), ((0, 0, 0), (1, 0, 0), 4.0)]),
        "mixed": make([
            ((0, 0, 0), (1, 0, 0), 4.0), ((0, 0.8, 0), (-1, 0, 0), 4.0), ((4.9, 0, 0), (1, 0, 0), 4.0),
            ((10, 0, 0), (1, 0, 0)), ((10, 0, 0), (0, 1, 0)), ((15, 0, 0), (1, 0, 0), 0.0),
            ((15, 0.8, 0), (1, 0, 0), 0.0),
        ]),
        "zero_length_pair": make([((0, 0, 0), (1, 0, 0), 0.0), ((1.005, 0, 0), (1, 0, 0), 0.0),
                                  ((0.5, 0, 0), (1, 0, 0), 0.0)]),
    }
    divided = make([((0, 0, 0), (1, 0, 0), 4.0), ((0, 0.2, 0), (1, 0, 0), 4.0)])
    divided.divide(1, 0.5)
    worlds["divided"] = divided
    sparse = make([((10.0 * i, 0, 0), (1, 0, 0)) for i in range(2048)])
    worlds["sparse2048"] = sparse
    return worlds


def pseudo_random_257() -> WorldState:
    """contact_geometry_test.cpp:174-187."""
    w = WorldState()
    for i in range(257):
        x = np.float32((i * 37) % 101) * np.float32(0.21)
        y = np.float32((i * 53) % 89) * np.float32(0.19)
        z = np.float32((i * 29) % 47) * np.float32(0.17)
        axis = (float((i * 7) % 13) + 1.0, float((i * 11) % 17) + 1.0, float((i * 5) % 19) + 1.0)
        length = np.float32(0.25) + np.float32(i % 11) * np.float32(0.3)
        radius = np.float32(0.15) + np.float32(i % 5) * np.float32(0.07)
        w.add_cell((x, y, z), axis, length, radius, 1.0)
    return w


def wall_set() -> ConstraintSet:
    cs = ConstraintSet()
    cs.add_box(center=(20, 20, 0), half_extents=(20, 20, 0.6), allowed_region=abi.REGION_INSIDE)
    cs.add_plane(point=(0, -0.2, 0), inward_normal=(0, 1, 0))
    cs.add_sphere(center=(10, 10, 0), radius=3.0)
    cs.add_sphere(center=(30, 10, 0), radius=25.0, allowed_region=abi.REGION_INSIDE)
    cs.add_cylinder(center=(30, 30, 0), radius=2.0, half_height=1.0)
    cs.add_cylinder(center=(20, 20, 0), radius=24.0, half_height=0.7, allowed_region=abi.REGION_INSIDE)
    cs.add_box(center=(5, 30, 0), half_extents=(2, 3, 1))
    cs.add_plane(point=(41, 0, 0), inward_normal=(-1, 0, 0), coefficient=0.5)
    return cs


def make_chain(count: int):
    """make_chain of contact_dynamics_conformance_test.cpp:56-109, in FP32."""
    f = np.float32
    bodies = np.zeros(count, dtype=abi.CONTACT_BODY_DTYPE)
    for i in range(count):
        angle = f(0.1) * f(i % 5)
        bodies[i]["axis"] = (np.cos(angle, dtype=f), np.sin(angle, dtype=f), 0.0)
        bodies[i]["translational_mobility"] = f(1.0) / (f(3.0) + f(0.1) * f(i % 7))
        bodies[i]["transverse_mobility"] = 0.9
        bodies[i]["axial_mobility"] = 20.0
        bodies[i]["length_rate"] = -0.2 if i % 4 == 3 else f(0.8) + f(0.05) * f(i % 3)
        if i + 1 == count:
            bodies[i]["translational_mobility"] = 0.0
            bodies[i]["transverse_mobility"] = 0.0
            bodies[i]["axial_mobility"] = 0.0
    rows = []
    wall = np.zeros(1, dtype=abi.CONTACT_ROW_DTYPE)
    wall["first_slot"] = 0
    wall["second_slot"] = abi.INVALID_SLOT
    wall["first_jacobian"] = (1, 0, 0, 0, 0, 0.1)
    wall["first_length_lever"] = 0.5
    wall["offset"] = -0.004
    wall["compliance"] = 1.0e-4
    rows.append(wall)
    for i in range(count - 1):
        tilt = f(0.2) * f(i % 3) - f(0.2)
        nx, ny = np.cos(tilt, dtype=f), np.sin(tilt, dtype=f)
        r = np.zeros(1, dtype=abi.CONTACT_ROW_DTYPE)
        r["first_slot"] = i
        r["second_slot"] = i + 1
        r["first_jacobian"] = (-nx, -ny, 0, 0, 0, f(-1.5) * ny)
        r["second_jacobian"] = (nx, ny, 0, 0, 0, f(-1.5) * ny)
        r["first_length_lever"] = f(0.5) * nx
        r["second_length_lever"] = f(0.5) * nx
        r["offset"] = -0.01 if i % 3 == 0 else f(0.002) * f(i % 4)
        r["compliance"] = 2.5e-5 if i % 6 == 0 else 1.0e-4
        rows.append(r)
    if count > 2:
        r = np.zeros(1, dtype=abi.CONTACT_ROW_DTYPE)
        r["first_slot"] = 0
        r["second_slot"] = count - 2
        r["first_jacobian"] = (0, -1, 0, 0, 0, 0)
        r["second_jacobian"] = (0, 1, 0, 0, 0, 0)
        r["offset"] = 5.0
        r["compliance"] = 1.0e-4
        rows.append(r)
    return np.concatenate(rows), bodies


def chain_system(count: int, law: int) -> ContactSystem:
    rows, bodies = make_chain(count)
    return ContactSystem(rows, bodies, 0.05, GrowthLoadResponse(law, 0.3, 0.2, 3.0))


def hand_made_contacts() -> np.ndarray:
    """Five cells (slots 0-4, ids 10-14) with slot 3 untouched and two
    contacts (ordinals 0, 1) between the same pair, listed out of order."""
    rows = [(11, 14, 1, 4, 0), (10, 12, 0, 2, 0), (10, 12, 0, 2, 1), (12, 14, 2, 4, 0), (10, 11, 0, 1, 0)]
    out = np.zeros(len(rows), dtype=abi.CELL_CONTACT_DTYPE)
    for i, (first_id, second_id, first_slot, second_slot, ordinal) in enumerate(rows):
        out[i]["first_id"], out[i]["second_id"] = first_id, second_id
        out[i]["first_slot"], out[i]["second_slot"], out[i]["ordinal"] = first_slot, second_slot, ordinal
        out[i]["normal"] = (0.0, 1.0, 0.0)
        out[i]["weight"] = 1.0
        out[i]["signed_separation"] = -0.01
    return out


# Invalid contacts: (field, value) planted in contact 7 of colony_1k's list,
# with contact 11 broken too so that the lowest failing contact must win.
GRAPH_ERRORS = (("first_id", 0), ("second_id", 1), ("second_slot", 1000), ("first_slot", 3), ("ordinal", 2),
                ("weight", 0.0), ("signed_separation", float("nan")), ("normal", (0.0, 0.0, 1.001)))
EXTERNAL_ERRORS = (("cell_id", 0), ("constraint_id", 0), ("cell_slot", 1000), ("constraint_kind", 4),
                   ("location", 3), ("weight", -1.0), ("point_on_cell", (float("inf"), 0.0, 0.0)),
                   ("normal", (0.0, 0.999, 0.0)))


def contact_graph_payload(ref) -> dict:
    colony = np.load(OUT / "colony_1k.npz")
    walls = np.load(OUT / "walls.npz")
    cell_count = len(colony["world__ids"])
    rng = np.random.default_rng(7)
    payload = {"cell_count": np.int64(cell_count)}
    # colony_1k's contacts_0.1 and walls' walls_1_0.1 are the lists of the
    # found and walls cases; the shuffled ones are stored as permutations.
    found = colony["contacts_0.1"]
    order = rng.permutation(len(found))
    payload["shuffled__order"] = order
    cases = {"found": found, "shuffled": found[order], "hand_made": hand_made_contacts(),
             "empty": np.zeros(0, dtype=abi.CELL_CONTACT_DTYPE)}
    counts = {"found": cell_count, "shuffled": cell_count, "hand_made": 8, "empty": 3}
    for name, contacts in cases.items():
        if name in ("hand_made", "empty"):
            payload[f"{name}__contacts"] = contacts
        payload[f"{name}__cell_count"] = np.int64(counts[name])
        for key, value in zip(("incidence_offsets", "incidence", "neighbor_offsets", "neighbors"),
                              ref.contact_graph(contacts, counts[name])):
            payload[f"{name}__{key}"] = value
    external = walls["walls_1_0.1"]
    wall_order = rng.permutation(len(external))
    payload["walls_shuffled__order"] = wall_order
    for name, contacts in (("walls", external), ("walls_shuffled", external[wall_order])):
        offsets, indices = ref.external_contact_graph(contacts, cell_count)
        payload[f"{name}__incidence_offsets"] = offsets
        payload[f"{name}__incidence"] = indices
    for group, errors, base, build in (("cell_error", GRAPH_ERRORS, found, ref.contact_graph),
                                       ("external_error", EXTERNAL_ERRORS, external, ref.external_contact_graph)):
        messages = []
        for field, value in errors:
            bad = base.copy()
            bad[7][field] = value
            bad[11]["weight"] = -2.0
            try:
                build(bad, cell_count)
                messages.append("")
            except ValueError as error:
                messages.append(str(error))
        payload[f"{group}__messages"] = np.array(messages)
    return payload


def main(only: set[str] | None = None) -> None:
    from oracle.native import Reference, build

    build(reference=True)
    ref = Reference()
    if only is not None:
        if "contact_graph" in only:
            np.savez_compressed(OUT / "contact_graph.npz", **contact_graph_payload(ref))
        return

    worlds = geometry_kat_worlds()
    payload = {}
    for name, w in worlds.items():
        for k, v in world_arrays(w).items():
            payload[f"{name}__{k}"] = v
        for margin in (0.01, 0.1):
            payload[f"{name}__contacts_{margin}"] = ref.find_cell_contacts(w, ContactParameters(activation_margin=margin))
    payload["names"] = np.array(sorted(worlds))
    np.savez_compressed(OUT / "geometry_kat.npz", **payload)

    w = pseudo_random_257()
    payload = {f"world__{k}": v for k, v in world_arrays(w).items()}
    for margin in (0.0, 0.01, 0.5):
        payload[f"contacts_{margin}"] = ref.find_cell_contacts(w, ContactParameters(activation_margin=margin))
        payload[f"exhaustive_{margin}"] = ref.find_cell_contacts(w, ContactParameters(activation_margin=margin),
                                                                 exhaustive=True)
    np.savez_compressed(OUT / "pseudo_random_257.npz", **payload)

    w = workloads.colony_1k()
    payload = {f"world__{k}": v for k, v in world_arrays(w).items()}
    payload["contacts_0.1"] = ref.find_cell_contacts(w, ContactParameters(activation_margin=0.1))
    offsets, indices = ref.incidence(w, ContactParameters(activation_margin=0.1))
    payload["incidence_offsets"] = offsets
    payload["incidence_indices"] = indices
    stepped = w.copy()
    dyn = ContactDynamicsParameters(overlap_tolerance=5.0e-4)
    result = ref.advance_contact_dynamics(stepped, None, 0.02, dyn)
    payload.update({f"stepped__{k}": v for k, v in world_arrays(stepped).items()})
    payload["step_report"] = np.array([result.report.substeps, result.report.halvings, result.report.refinements,
                                       result.report.iterations, result.report.max_rows], dtype=np.int64)
    payload["step_max_overlap"] = np.float32(result.report.max_overlap)
    payload["step_velocities"] = result.center_velocities
    payload["step_loads"] = result.axial_loads
    payload["step_increments"] = result.length_increments
    np.savez_compressed(OUT / "colony_1k.npz", **payload)

    cs = wall_set()
    payload = {"constraints": cs.records}
    for every_face in (False, True):
        for margin in (0.0, 0.1):
            payload[f"walls_{int(every_face)}_{margin}"] = ref.find_external_contacts(
                w, cs, ConstraintContactParameters(activation_margin=margin), every_face=every_face)
    np.savez_compressed(OUT / "walls.npz", **payload)

    payload = {}
    for count, law in ((2, 0), (9, 0), (9, 1), (9, 2), (300, 2), (5, 1), (6, 2)):
        system = chain_system(count, law)
        zero = np.zeros(len(system.rows), dtype=np.float32)
        solved = ref.solve_contact_forces(system, zero, ContactSolveParameters(2.0e-6, 200000))
        key = f"chain_{count}_{law}"
        payload[f"{key}__rows"] = system.rows
        payload[f"{key}__bodies"] = system.bodies
        payload[f"{key}__multipliers"] = solved.multipliers
        payload[f"{key}__report"] = np.array([solved.report.status, solved.report.iterations], dtype=np.int64)
        payload[f"{key}__residual"] = np.float32(solved.report.residual)
        response = ref.evaluate_contact_response(system, solved.multipliers)
        payload[f"{key}__velocities"] = response.velocities
        payload[f"{key}__loads"] = response.loads
        payload[f"{key}__rates"] = response.length_rates
        payload[f"{key}__gaps"] = ref.evaluate_contact_gaps(system, solved.multipliers)
        payload[f"{key}__bound"] = np.float32(ref.contact_system_diagonal_bound(system))
    np.savez_compressed(OUT / "chains.npz", **payload)
    np.savez_compressed(OUT / "contact_graph.npz", **contact_graph_payload(ref))
    for path in sorted(OUT.glob("*.npz")):
        print(path.name, path.stat().st_size)


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)
