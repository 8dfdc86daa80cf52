"""The two forms of the BB relaxation on the device (msb_set_relaxation): the
CUDA graph with a WHILE node and the fused cooperative kernel.  Both run the
same per-pass arithmetic; on one block they are the same computation bit for
bit, on several they reduce the BB products over different block counts and
converge to the same tolerance."""

import numpy as np
import pytest

from microsimulator_b200 import workloads
from microsimulator_b200.backend import B200Backend
from microsimulator_b200.types import ContactDynamicsParameters, ContactSolveParameters
from tests.golden.make_golden import chain_system

pytestmark = pytest.mark.gpu

GRAPH, FUSED = B200Backend.RELAXATION_GRAPH, B200Backend.RELAXATION_FUSED


@pytest.fixture
def forms(backend):
    yield backend
    backend.set_relaxation(B200Backend.RELAXATION_AUTOMATIC)


def solve_with(backend, form, system, parameters):
    backend.set_relaxation(form)
    return backend.solve_contact_forces(system, np.zeros(len(system.rows), np.float32), parameters)


@pytest.mark.parametrize("count,law", [(2, 0), (9, 1), (9, 2), (5, 1), (6, 2)])
def test_one_block_solves_are_identical(forms, count, law):
    system = chain_system(count, law)
    parameters = ContactSolveParameters(2.0e-6, 200000)
    graph = solve_with(forms, GRAPH, system, parameters)
    fused = solve_with(forms, FUSED, system, parameters)
    assert graph.report == fused.report
    assert np.array_equal(graph.multipliers, fused.multipliers)


def test_several_block_solve_converges_alike(forms):
    system = chain_system(300, 2)
    parameters = ContactSolveParameters(2.0e-6, 200000)
    graph = solve_with(forms, GRAPH, system, parameters)
    fused = solve_with(forms, FUSED, system, parameters)
    assert graph.report.status == fused.report.status == 0
    assert fused.report.residual <= 2.0e-6
    scale = max(1.0, float(np.max(np.abs(graph.multipliers))))
    assert np.max(np.abs(graph.multipliers - fused.multipliers)) <= 2e-3 * scale


def test_many_block_steps_agree(forms):
    world = workloads.jammed(60_000, seed=11)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    results = {}
    for form in (GRAPH, FUSED):
        forms.set_relaxation(form)
        w = world.copy()
        report = forms.advance_contact_dynamics(w, None, 0.02, p).report
        results[form] = (w, report)
    (wg, rg), (wf, rf) = results[GRAPH], results[FUSED]
    assert rg.substeps == rf.substeps and rg.halvings == rf.halvings
    assert rf.max_overlap <= 5e-4 * 1.0001 or rf.max_overlap <= rg.max_overlap * 1.0001
    # The same unique solutions up to the solve tolerance.
    assert np.max(np.abs(wg.geometry()[:, :3] - wf.geometry()[:, :3])) < 4 * 5e-4


def test_fused_steps_with_walls(forms, oracle):
    world, walls = workloads.trap_colony(n=800, seed=6, area_fraction=0.5)
    p = ContactDynamicsParameters(overlap_tolerance=5e-4)
    forms.set_relaxation(FUSED)
    a, b = world.copy(), world.copy()
    ra = forms.advance_contact_dynamics(a, walls, 0.02, p)
    rb = oracle.advance_contact_dynamics(b, walls, 0.02, p)
    assert ra.report.substeps == rb.report.substeps
    # Within a few solve tolerances of the reference-identical oracle.
    assert np.max(np.abs(a.geometry() - b.geometry())) <= 4 * p.overlap_tolerance


def test_invalid_form(forms):
    with pytest.raises(ValueError):
        forms.set_relaxation(3)
