"""Pins the CPU oracle: against the reference tests' known answers, against
the committed golden fixtures (made by the reference itself), and against the
reference library run live.  FP32 oracle results must be bit-identical; the
FP64 oracle must agree to FP32 rounding."""

import math

import numpy as np
import pytest

from microsimulator_b200 import abi, workloads
from microsimulator_b200.types import (
    ConstraintContactParameters,
    ContactDynamicsParameters,
    ContactParameters,
    ContactSolveParameters,
    ContactSystem,
    GrowthLoadResponse,
)
from microsimulator_b200.world import WorldState
from tests.golden.make_golden import chain_system, geometry_kat_worlds, pseudo_random_257, wall_set, world_from


def close(a, b, tol=1e-5):
    return abs(float(a) - float(b)) <= tol


# ---- known answers of tests/cpp/contact_geometry_test.cpp ------------------

def test_end_on_contact(oracle):
    c = oracle.find_cell_contacts(geometry_kat_worlds()["end_on"])
    assert len(c) == 1
    assert (c[0]["first_id"], c[0]["second_id"], c[0]["ordinal"]) == (1, 2, 0)
    assert close(c[0]["signed_separation"], -0.1)
    assert close(c[0]["normal"][0], 1.0)
    assert close(c[0]["point_on_first"][0], 1.5)
    assert close(c[0]["weight"], 1.0)


def test_parallel_overlap_two_weighted_contacts(oracle):
    c = oracle.find_cell_contacts(geometry_kat_worlds()["parallel"])
    assert len(c) == 2
    assert list(c["ordinal"]) == [0, 1]
    assert close(c[0]["point_on_first"][0], -2.0) and close(c[1]["point_on_first"][0], 2.0)
    for x in c:
        assert close(x["signed_separation"], -0.2)
        assert close(x["normal"][1], 1.0)
        assert close(x["weight"], math.sqrt(0.5))


def test_skew_and_coincident_normals(oracle):
    skew = oracle.find_cell_contacts(geometry_kat_worlds()["skew"])
    assert close(skew[0]["normal"][2], 1.0)
    coincident = oracle.find_cell_contacts(geometry_kat_worlds()["coincident"])
    assert len(coincident) == 2
    for x in coincident:
        assert np.all(np.isfinite(x["normal"]))
        assert close(np.linalg.norm(x["normal"]), 1.0)
        assert close(x["signed_separation"], -1.0)


def test_no_per_cell_limit_and_sparse(oracle):
    dense = oracle.find_cell_contacts(geometry_kat_worlds()["dense31"])
    assert len(dense) == 31 * 30
    assert len(oracle.find_cell_contacts(geometry_kat_worlds()["sparse2048"])) == 0


def test_pair_order_reverses_normal(oracle):
    f = oracle.find_cell_contacts(geometry_kat_worlds()["forward"])
    r = oracle.find_cell_contacts(geometry_kat_worlds()["reversed"])
    assert len(f) == len(r)
    assert np.allclose(f["normal"], -r["normal"], atol=1e-5)
    assert np.allclose(f["signed_separation"], r["signed_separation"], atol=1e-5)


def test_contacts_sorted_by_stable_identity(oracle):
    c = oracle.find_cell_contacts(geometry_kat_worlds()["divided"])
    keys = list(zip(c["first_id"], c["second_id"], c["ordinal"]))
    assert all(a < b for a, b in zip(keys, keys[1:]))
    assert all(c["first_id"] < c["second_id"])


def test_invalid_parameters_rejected(oracle):
    with pytest.raises(ValueError):
        oracle.find_cell_contacts(WorldState(), ContactParameters(parallel_sine_threshold=2.0))


# ---- the golden fixtures ---------------------------------------------------

def test_geometry_kat_fixtures_bit_exact(oracle, golden):
    data = golden("geometry_kat")
    for name in data["names"]:
        world = world_from(data, f"{name}__")
        for margin in (0.01, 0.1):
            expected = data[f"{name}__contacts_{margin}"]
            actual = oracle.find_cell_contacts(world, ContactParameters(activation_margin=margin))
            assert actual.tobytes() == expected.tobytes(), (name, margin)


def test_grid_equals_exhaustive_257(oracle, golden):
    data = golden("pseudo_random_257")
    world = world_from(data, "world__")
    for margin in (0.0, 0.01, 0.5):
        actual = oracle.find_cell_contacts(world, ContactParameters(activation_margin=margin))
        assert actual.tobytes() == data[f"contacts_{margin}"].tobytes()
        exhaustive = data[f"exhaustive_{margin}"]
        assert np.array_equal(actual[["first_id", "second_id", "ordinal"]], exhaustive[["first_id", "second_id", "ordinal"]])


def test_colony_contacts_and_step_bit_exact(oracle, golden):
    data = golden("colony_1k")
    world = world_from(data, "world__")
    contacts = oracle.find_cell_contacts(world, ContactParameters(activation_margin=0.1))
    assert contacts.tobytes() == data["contacts_0.1"].tobytes()
    result = oracle.advance_contact_dynamics(world, None, 0.02, ContactDynamicsParameters(overlap_tolerance=5e-4))
    stepped = world_from(data, "stepped__")
    assert np.array_equal(world.geometry(), stepped.geometry())
    r = result.report
    assert [r.substeps, r.halvings, r.refinements, r.iterations, r.max_rows] == list(data["step_report"])
    assert np.array_equal(result.axial_loads, data["step_loads"])
    assert np.array_equal(result.center_velocities, data["step_velocities"])


def test_walls_bit_exact(oracle, golden):
    data = golden("walls")
    world = world_from(golden("colony_1k"), "world__")
    cs = wall_set()
    assert cs.records.tobytes() == data["constraints"].tobytes()
    for every_face in (0, 1):
        for margin in (0.0, 0.1):
            actual = oracle.find_external_contacts(world, cs, ConstraintContactParameters(margin), every_face=bool(every_face))
            assert actual.tobytes() == data[f"walls_{every_face}_{margin}"].tobytes()


def test_chain_solves_bit_exact(oracle, golden):
    data = golden("chains")
    keys = sorted({k.split("__")[0] for k in data.files})
    for key in keys:
        _, count, law = key.split("_")
        system = ContactSystem(data[f"{key}__rows"], data[f"{key}__bodies"], 0.05,
                               GrowthLoadResponse(int(law), 0.3, 0.2, 3.0))
        zero = np.zeros(len(system.rows), dtype=np.float32)
        solved = oracle.solve_contact_forces(system, zero, ContactSolveParameters(2e-6, 200000))
        assert np.array_equal(solved.multipliers, data[f"{key}__multipliers"]), key
        assert [solved.report.status, solved.report.iterations] == list(data[f"{key}__report"])
        response = oracle.evaluate_contact_response(system, solved.multipliers)
        assert np.array_equal(response.velocities, data[f"{key}__velocities"])
        assert np.array_equal(response.loads, data[f"{key}__loads"])
        assert np.array_equal(oracle.evaluate_contact_gaps(system, solved.multipliers), data[f"{key}__gaps"])
        assert oracle.contact_system_diagonal_bound(system) == data[f"{key}__bound"]


def test_fp64_oracle_agrees_to_fp32_rounding(oracle, golden):
    data = golden("colony_1k")
    world = world_from(data, "world__")
    c32 = oracle.find_cell_contacts(world, ContactParameters(activation_margin=0.1))
    c64 = oracle.find_cell_contacts(world, ContactParameters(activation_margin=0.1), precision=64)
    assert len(c32) == len(c64)
    assert np.max(np.abs(c32["signed_separation"] - c64["signed_separation"])) < 1e-4
    system = chain_system(9, abi.GROWTH_LAW_LINEAR)
    zero = np.zeros(len(system.rows), dtype=np.float32)
    s32 = oracle.solve_contact_forces(system, zero, ContactSolveParameters(2e-6, 200000))
    s64 = oracle.solve_contact_forces(system, zero, ContactSolveParameters(2e-6, 200000), precision=64)
    r32 = oracle.evaluate_contact_response(system, s32.multipliers, precision=64)
    r64 = oracle.evaluate_contact_response(system, s64.multipliers, precision=64)
    assert np.max(np.abs(r32.velocities - r64.velocities)) < 2e-3


# ---- live reference ------------------------------------------------------

def test_oracle_matches_reference_live(oracle, reference):
    world = workloads.colony_1k(seed=7, n=600, side=30.0, growth_rate=0.5)
    for margin in (0.0, 0.1):
        p = ContactParameters(activation_margin=margin)
        assert oracle.find_cell_contacts(world, p).tobytes() == reference.find_cell_contacts(world, p).tobytes()
    a, b = world.copy(), world.copy()
    ra = oracle.advance_contact_dynamics(a, None, 0.02, ContactDynamicsParameters(overlap_tolerance=5e-4))
    rb = reference.advance_contact_dynamics(b, None, 0.02, ContactDynamicsParameters(overlap_tolerance=5e-4))
    assert np.array_equal(a.geometry(), b.geometry())
    assert ra.report == rb.report


def test_division_matches_reference_world(reference):
    world = workloads.colony_1k(seed=3, n=200, side=30.0)
    plan = workloads.plan_divisions(world, 0.1, seed=5)
    handle = reference.world_create(world)
    try:
        reference.world_divide(handle, plan.parents, plan.rotations)
        mirrored = WorldState()
        reference.world_read(handle, mirrored)
    finally:
        reference.world_destroy(handle)
    local = world.copy()
    local.divide_many(plan.parents, 0.5, plan.rotations)
    assert np.array_equal(local.ids, mirrored.ids)
    assert np.array_equal(local.geometry(), mirrored.geometry())


def test_constraint_conformance_fixtures(oracle, reference):
    """The reference's constraint conformance fixtures
    (tests/conformance/constraint_conformance_test.cpp:19-153): the FP32
    oracle's wall contacts equal the reference's, field for field."""
    from tests.constraint_fixtures import FIXTURES

    for name, build in FIXTURES.items():
        world, constraints = build()
        expected = reference.find_external_contacts(world, constraints)
        assert oracle.find_external_contacts(world, constraints).tobytes() == expected.tobytes(), name
