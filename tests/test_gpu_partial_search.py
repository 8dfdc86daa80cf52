"""Overlap re-checks with a partial re-search.

A re-check of a refinement round (contact_dynamics.cpp:520-521 of the
reference) takes its candidates from the substep's first search, padded by
a margin P, when no cell moved by more than P/2 since; when some cells did,
the kept pairs of the other cells are merged with a new search of the pairs
of those that moved.  Either way the touches, their order and so the step
are those of a full contact search: here a step with every kind of
re-check against the same step with full searches only, bit for bit."""

import numpy as np
import pytest

from microsimulator_b200 import sweep, workloads
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactDynamicsParameters

pytestmark = pytest.mark.gpu

DT = 0.02
DYN = ContactDynamicsParameters(overlap_tolerance=5e-4)


def step(backend, world, k):
    plan = workloads.plan_divisions(world, 0.02, seed=900 + k)
    world.divide_many(plan.parents, 0.5, plan.rotations)
    report = backend.advance_contact_dynamics(world, None, DT, DYN).report
    world.next_id = int(world.ids.max()) + 1
    return report


def test_partial_re_search_steps_as_full_searches():
    """The 1M-capsule jammed colony, four steps after three from its random
    start (steps whose re-checks meet cells that moved further than the
    padding of the kept candidates)."""
    world = workloads.jammed(n=1_000_000, seed=42)
    auto, full = B200Backend(0), B200Backend(0)
    try:
        full.set_search_reuse(2)
        for k in range(3):
            step(auto, world, k)
        kinds = {"full": 0, "kept": 0, "partial": 0}
        a, b = world.copy(), world.copy()
        for k in range(3, 7):
            ra = step(auto, a, k)
            rb = step(full, b, k)
            for name, value in auto.last_step_searches().items():
                kinds[name] += value
            assert full.last_step_searches()["partial"] == 0 and full.last_step_searches()["kept"] == 0
            assert (ra.substeps, ra.refinements, ra.iterations) == (rb.substeps, rb.refinements, rb.iterations)
            assert ra.max_rows == rb.max_rows
            assert np.array_equal(a.geometry(), b.geometry()), k
        print("re-checks", kinds)
        assert kinds["partial"] > 0
    finally:
        auto.close()
        full.close()


def test_partial_re_search_in_a_batch_steps_as_full_searches():
    """Thirty-two sweep colonies of 5,000-40,000 capsules (above the size
    from which a batch takes partial re-searches) from their loose random
    starts, stepped as one batch: every kind of re-check against full
    searches only."""
    batch = sweep.sweep_batch(count=32, low=5_000, high=40_000, seed=3)
    auto, full = B200Backend(0), B200Backend(0)
    try:
        full.set_search_reuse(2)
        worlds = [w.copy() for w in batch.worlds]
        ba = sweep.ColonyBatch([w.copy() for w in worlds], batch.drag, batch.stiffness)
        bb = sweep.ColonyBatch([w.copy() for w in worlds], batch.drag, batch.stiffness)
        kinds = {"full": 0, "kept": 0, "partial": 0}
        for k in range(4):
            ba.divide(0.02, seed=k)
            bb.divide(0.02, seed=k)
            ra, ca = ba.step(auto, DT, DYN)
            rb, cb = bb.step(full, DT, DYN)
            for name, value in auto.last_step_searches().items():
                kinds[name] += value
            assert (ra.substeps, ra.refinements) == (rb.substeps, rb.refinements)
            assert np.array_equal(ca["iterations"], cb["iterations"])
            for wa, wb in zip(ba.worlds, bb.worlds):
                assert np.array_equal(wa.geometry(), wb.geometry()), k
        print("re-checks", kinds)
    finally:
        auto.close()
        full.close()


def test_search_reuse_modes_are_checked(backend):
    for mode in (0, 1, 2):
        backend.set_search_reuse(mode)
    with pytest.raises(ValueError, match="search reuse"):
        backend.set_search_reuse(3)
    backend.set_search_reuse(0)
    assert set(backend.last_step_searches()) == {"full", "kept", "partial"}
