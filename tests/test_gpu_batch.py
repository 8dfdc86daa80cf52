"""Batched colonies through msb_advance_contact_dynamics_batch: each colony
of a batch steps as it would alone (same rows; positions within the solve's
tolerance-level spread), with its own drag, stiffness and convergence, and
colonies that overlap in space never touch."""

import numpy as np
import pytest

from microsimulator_b200 import sweep, workloads
from microsimulator_b200.backend import B200Backend, DeviceCells
from microsimulator_b200.types import ContactDynamicsParameters

pytestmark = pytest.mark.gpu

TOLERANCE = 5e-4
DT = 0.02
SIZES = [300, 1500, 700, 50, 1100, 400]
DRAG = [1.0, 0.6, 1.7, 1.2, 0.9, 2.0]
STIFFNESS = [1.0e4, 0.5e4, 2.0e4, 1.3e4, 0.8e4, 1.0e4]

_SETTLED = {}


def params(k):
    return ContactDynamicsParameters(overlap_tolerance=TOLERANCE, drag=DRAG[k], contact_stiffness=STIFFNESS[k])


def settled_worlds():
    """Each colony settled alone for 20 steps with its own parameters."""
    if "worlds" not in _SETTLED:
        b = B200Backend(0)
        worlds = []
        try:
            for k, n in enumerate(SIZES):
                w = workloads.sweep_colony(n, seed=100 + k)
                for step in range(20):
                    plan = workloads.plan_divisions(w, 0.02, seed=step * 31 + k)
                    w.divide_many(plan.parents, 0.5, plan.rotations)
                    b.advance_contact_dynamics(w, None, DT, params(k))
                    w.next_id = int(w.ids.max()) + 1
                worlds.append(w)
        finally:
            b.close()
        _SETTLED["worlds"] = worlds
    return [w.copy() for w in _SETTLED["worlds"]]


def test_each_colony_steps_as_it_would_alone(backend):
    worlds = settled_worlds()
    alone = [w.copy() for w in worlds]
    reports_alone = [backend.advance_contact_dynamics(w, None, DT, params(k)).report for k, w in enumerate(alone)]
    batch = sweep.ColonyBatch(worlds, DRAG, STIFFNESS)
    b = B200Backend(0)
    try:
        report, colonies = batch.step(b, DT, ContactDynamicsParameters(overlap_tolerance=TOLERANCE))
        tuning = b.batch_tuning()
    finally:
        b.close()
    assert tuning["cluster"] in (1, 2, 4, 8, 16) and tuning["threads"] in (256, 512)
    assert tuning["box_scale"] >= 1.0
    assert np.array_equal(colonies["cells"], np.array(SIZES_after(worlds), dtype=np.uint32))
    # These settled colonies take one substep alone and in the batch: the
    # batch halves for all colonies only when one of them needs it, and then
    # the colonies' steps differ from their steps alone by design.
    assert report.substeps == 1 and all(r.substeps == 1 for r in reports_alone)
    for k, (w, a, r) in enumerate(zip(batch.worlds, alone, reports_alone)):
        assert np.array_equal(w.ids, a.ids)
        spread = np.max(np.abs(w.geometry()[:, :3] - a.geometry()[:, :3]))
        print(f"colony {k}: substeps {report.substeps}/{r.substeps}, refinements "
              f"{report.refinements}/{r.refinements}, spread {spread:.3e}")
        if r.refinements == report.refinements:
            # The same rows as alone (a colony that needed fewer refinement
            # rounds than the batch keeps its rows and skips the rest).
            assert colonies["rows"][k] == r.max_rows, (k, colonies["rows"][k], r.max_rows)
        # A position spread at the solve's tolerance level (measured: 0).
        assert spread <= 4 * TOLERANCE, (k, spread)
        assert np.all(np.isfinite(w.geometry()))
        assert colonies["iterations"][k] > 0 or r.iterations == 0
        # Each colony's last solve converged to its own tolerance.
        assert colonies["status"][k] == 0


def test_each_colony_matches_the_reference_stepped_alone(reference):
    """Each colony of a batch against the reference CPU backend stepping that
    colony alone with the colony's own drag and contact stiffness
    (ContactDynamicsParameters, cpp/include/microsimulator/contact_dynamics.hpp:37-65),
    at the tight tolerance 2e-5 um: the same substep plan as the reference
    (here one substep for every colony and for the batch), the rows the
    reference's last solve had, and every position within 1e-4 capsule
    radius of the reference's."""
    tight = 2.0e-5
    worlds = settled_worlds()
    expected = []
    for k, w in enumerate(worlds):
        alone = w.copy()
        p = ContactDynamicsParameters(overlap_tolerance=tight, drag=DRAG[k], contact_stiffness=STIFFNESS[k])
        expected.append((alone, reference.advance_contact_dynamics(alone, None, DT, p).report))
    batch = sweep.ColonyBatch(worlds, DRAG, STIFFNESS)
    b = B200Backend(0)
    try:
        report, colonies = batch.step(b, DT, ContactDynamicsParameters(overlap_tolerance=tight))
    finally:
        b.close()
    print("batch", report, [(r.substeps, r.refinements, r.max_rows) for _, r in expected])
    assert all(r.substeps == report.substeps for _, r in expected), report
    for k, (w, (alone, r)) in enumerate(zip(batch.worlds, expected)):
        assert np.array_equal(w.ids, alone.ids)
        spread = float(np.max(np.abs(w.geometry()[:, :3] - alone.geometry()[:, :3])))
        print(f"colony {k}: {len(w)} cells, max |position - reference| {spread:.3e} um")
        assert spread <= 1e-4 * 0.5, (k, spread)
        assert colonies["status"][k] == 0
        assert abs(float(colonies["max_overlap"][k]) - r.max_overlap) <= 2 * tight


def SIZES_after(worlds):
    return [len(w) for w in worlds]


def test_colony_parameters_reach_their_colony(backend):
    """Two copies of one colony with different drag move differently; the
    same colony twice with the same parameters moves identically."""
    w = settled_worlds()[1]
    batch = sweep.ColonyBatch([w.copy(), w.copy(), w.copy()], [1.0, 1.0, 2.0], [1.0e4, 1.0e4, 1.0e4])
    b = B200Backend(0)
    try:
        batch.step(b, DT, ContactDynamicsParameters(overlap_tolerance=TOLERANCE))
    finally:
        b.close()
    a, same, slow = (x.geometry() for x in batch.worlds)
    assert np.array_equal(a, same)
    assert not np.array_equal(a, slow)


def test_colonies_in_the_same_place_never_touch(backend):
    """Colonies are laid out in the same region of space; a batch of a
    colony and a shifted copy steps each as alone."""
    w = settled_worlds()[2]
    shifted = w.copy()
    shifted.position_x = shifted.position_x + np.float32(1.3)
    alone = [w.copy(), shifted.copy()]
    reports = [backend.advance_contact_dynamics(a, None, DT, params(0)).report for a in alone]
    batch = sweep.ColonyBatch([w.copy(), shifted.copy()], [DRAG[0]] * 2, [STIFFNESS[0]] * 2)
    b = B200Backend(0)
    try:
        report, colonies = batch.step(b, DT, ContactDynamicsParameters(overlap_tolerance=TOLERANCE))
    finally:
        b.close()
    assert report.substeps == reports[0].substeps == reports[1].substeps == 1
    for k in range(2):
        if report.refinements == reports[k].refinements:
            assert colonies["rows"][k] == reports[k].max_rows
        spread = np.max(np.abs(batch.worlds[k].geometry()[:, :3] - alone[k].geometry()[:, :3]))
        assert spread <= 4 * TOLERANCE, (k, spread)


def test_device_batch_equals_host_batch(backend):
    worlds = settled_worlds()[:3]
    batch = sweep.ColonyBatch(worlds, DRAG[:3], STIFFNESS[:3])
    host = batch.concatenated()
    device = DeviceCells(host.copy())
    b = B200Backend(0)
    try:
        rh, ch = b.advance_contact_dynamics_batch(host, batch.counts(), batch.drag, batch.stiffness, DT,
                                                  ContactDynamicsParameters(overlap_tolerance=TOLERANCE))
        # The second call reuses the first call's tuning.
        fresh = batch.concatenated()
        device = DeviceCells(fresh)
        rd, cd = b.advance_contact_dynamics_batch(device, batch.counts(), batch.drag, batch.stiffness, DT,
                                                  ContactDynamicsParameters(overlap_tolerance=TOLERANCE))
    finally:
        b.close()
    out = batch.concatenated()
    device.download(out)
    assert rh == rd
    assert np.array_equal(ch, cd)
    assert np.array_equal(host.geometry(), out.geometry())


def test_batch_rejects_what_it_cannot_step(backend):
    w = settled_worlds()[3]
    batch = sweep.ColonyBatch([w], [1.0], [1.0e4])
    cells = batch.concatenated()
    p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    with pytest.raises(ValueError):
        backend.advance_contact_dynamics_batch(cells, [len(cells) - 1], [1.0], [1.0e4], DT, p)
    with pytest.raises(ValueError):
        backend.advance_contact_dynamics_batch(cells, [len(cells)], [0.0], [1.0e4], DT, p)
    bad = cells.copy()
    bad.position_x = bad.position_x.copy()
    bad.position_x[0] = np.nan
    before = bad.copy()
    with pytest.raises(ValueError):
        backend.advance_contact_dynamics_batch(bad, [len(cells)], [1.0], [1.0e4], DT, p)
    assert np.array_equal(before.geometry(), bad.geometry(), equal_nan=True)
    backend.set_warm_start(backend.WARM_START_GUESS)
    try:
        with pytest.raises(ValueError):
            backend.advance_contact_dynamics_batch(cells, [len(cells)], [1.0], [1.0e4], DT, p)
    finally:
        backend.set_warm_start(0)


def test_batch_with_empty_and_single_cell_colonies(backend):
    """Empty colonies, a single cell and a colony of two touching cells step
    together; the empty ones report nothing, the single cell grows freely."""
    from microsimulator_b200.world import WorldState

    w = settled_worlds()[3]  # 50 cells
    empty = WorldState()
    one = WorldState()
    one.add_cell(position=(3.0, 4.0, 0.0), length=2.0, growth_rate=0.5)
    pair = WorldState()
    pair.add_cell(position=(-1.4, 0.0, 0.0), length=2.0)
    pair.add_cell(position=(1.4, 0.0, 0.0), length=2.0)
    worlds = [empty, w.copy(), one, empty.copy(), pair]
    batch = sweep.ColonyBatch(worlds, [1.0] * 5, [1.0e4] * 5)
    b = B200Backend(0)
    try:
        report, colonies = batch.step(b, DT, ContactDynamicsParameters(overlap_tolerance=TOLERANCE))
    finally:
        b.close()
    assert list(colonies["cells"]) == [0, len(w), 1, 0, 2]
    assert colonies["iterations"][0] == 0 and colonies["rows"][0] == 0
    assert colonies["iterations"][3] == 0
    assert np.all(colonies["status"] == 0)
    grown = batch.worlds[2]
    assert abs(float(grown.lengths[0]) - 2.02) < 1e-5
    assert grown.position_x[0] == np.float32(3.0) and grown.position_y[0] == np.float32(4.0)
    # The overlapping pair pushed apart symmetrically.
    px = batch.worlds[4].position_x
    assert px[0] < -1.4 and px[1] > 1.4 and abs(float(px[0] + px[1])) < 1e-4


def test_colonies_with_interleaved_ids_step_as_with_grouped_ids():
    """Rows in first-id order are grouped by colony when each colony's ids
    are a block (as the sweep tags them), and interleaved when the colonies'
    ids alternate.  The per-colony deepest overlaps, flag counts and row
    counts are folded per warp where a warp's rows share a colony and added
    lane by lane where they do not; either way each colony's step is the
    same: with the same order of ids within every colony, the same bits."""
    worlds = settled_worlds()
    grouped = sweep.concatenate(worlds)
    interleaved = grouped.copy()
    colony = np.repeat(np.arange(len(worlds), dtype=np.uint64), [len(w) for w in worlds])
    local = np.concatenate([w.ids for w in worlds]).astype(np.uint64)
    interleaved.ids = local * np.uint64(len(worlds)) + colony
    interleaved.next_id = int(interleaved.ids.max()) + 1
    counts = np.array([len(w) for w in worlds], dtype=np.uint32)
    dyn = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    b = B200Backend(0)
    try:
        ra, ca = b.advance_contact_dynamics_batch(grouped, counts, DRAG, STIFFNESS, DT, dyn)
        rb, cb = b.advance_contact_dynamics_batch(interleaved, counts, DRAG, STIFFNESS, DT, dyn)
    finally:
        b.close()
    assert (ra.substeps, ra.refinements) == (rb.substeps, rb.refinements)
    assert np.array_equal(ca["rows"], cb["rows"])
    assert np.array_equal(ca["iterations"], cb["iterations"])
    assert np.array_equal(ca["max_overlap"], cb["max_overlap"])
    assert np.array_equal(grouped.geometry(), interleaved.geometry())
