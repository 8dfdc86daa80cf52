"""The reference's Python tests of the contact path
(python/tests/test_simulation.py), on this backend through its Simulation
mirror: the same scenarios, the same assertions."""

import math

import numpy as np
import pytest

from microsimulator_b200 import abi
from microsimulator_b200.simulation import Simulation
from microsimulator_b200.types import ContactDynamicsParameters

pytestmark = pytest.mark.gpu


@pytest.fixture
def sim(backend):
    return Simulation(backend=backend)


def test_contact_step_pushes_overlapping_cells_apart(sim):
    """test_simulation.py:274-299."""
    first_id = sim.add_cell(length=4.0, growth_rate=0.0)
    second_id = sim.add_cell(position=(0.0, 0.8, 0.0), length=4.0, growth_rate=0.0)
    parameters = ContactDynamicsParameters()
    result = sim.step(0.05, parameters)
    # One step recovers the overlap limit, shared equally by cells of equal drag.
    assert result.report.max_rows >= 1
    below, above = sim.cell(first_id), sim.cell(second_id)
    assert math.isclose(below["position"][1], -0.025, abs_tol=2.0e-3)
    assert math.isclose(above["position"][1], 0.825, abs_tol=2.0e-3)
    assert math.isclose(below["length"], 4.0)
    for _ in range(8):
        result = sim.step(0.05, parameters)
    assert result.report.max_overlap <= 2.0e-3
    assert sim.cell(second_id)["position"][1] - sim.cell(first_id)["position"][1] >= 0.998


def test_constraints_participate_in_the_contact_solve(sim):
    """test_simulation.py:367-385."""
    cell_id = sim.add_cell(position=(0.0, 0.4, 0.0), length=2.0, radius=0.5)
    sim.add_plane_constraint(inward_normal=(0.0, 1.0, 0.0))
    sim.step(0.05, ContactDynamicsParameters())
    assert sim.cell(cell_id)["position"][1] > 0.4


def test_box_constraints_participate_in_the_contact_solve(sim):
    """test_simulation.py:389-418."""
    cell_id = sim.add_cell(position=(1.4, 0.0, 0.0), direction=(0.0, 1.0, 0.0), length=2.0, radius=0.5)
    constraint_id = sim.add_box_constraint(half_extents=(1.0, 1.0, 1.0), allowed_region=abi.REGION_OUTSIDE)
    graph = sim.find_external_contacts()
    assert len(graph) == 2
    assert np.all(graph.contacts["constraint_id"] == constraint_id)
    assert np.all(graph.contacts["constraint_kind"] == abi.CONSTRAINT_BOX)
    assert np.allclose(graph.contacts["signed_separation"], -0.1, atol=1.0e-6)
    sim.step(0.05, ContactDynamicsParameters())
    assert sim.cell(cell_id)["position"][0] > 1.4


def test_finite_wall_detects_midspan_capsule_contact(sim):
    """test_simulation.py:422-451."""
    cell_id = sim.add_cell(position=(0.0, 0.75, 0.0), direction=(1.0, 0.0, 0.0), length=3.5, radius=0.5)
    constraint_id = sim.add_box_constraint(half_extents=(1.0, 1.0, 5.0))
    graph = sim.find_external_contacts()
    assert len(graph) == 1
    contact = graph.contacts[0]
    assert contact["constraint_id"] == constraint_id
    assert contact["constraint_kind"] == abi.CONSTRAINT_BOX
    assert contact["location"] == abi.ROD_INTERIOR
    assert math.isclose(contact["point_on_cell"][0], 0.0, abs_tol=2.0e-5)
    assert math.isclose(contact["point_on_cell"][1], 0.25, abs_tol=2.0e-5)
    assert math.isclose(contact["normal"][1], -1.0, abs_tol=2.0e-5)
    assert math.isclose(contact["signed_separation"], -0.75, abs_tol=2.0e-5)
    sim.step(0.05, ContactDynamicsParameters())
    assert sim.cell(cell_id)["position"][1] > 0.75


def spanning_pair(backend, tilt):
    """_spanning_pair of test_contact_dynamics.py:534-548: two cells end to
    end that exactly span a closed 4 by 4 chamber."""
    sim = Simulation(backend=backend)
    sim.add_box_constraint(half_extents=(2.0, 2.0, 0.6), allowed_region=abi.REGION_INSIDE)
    for sign in (-1.0, 1.0):
        sim.add_cell(position=(sign * 1.0, 0.0, 0.0), direction=(math.cos(sign * tilt), math.sin(sign * tilt), 0.0),
                     length=1.2, radius=0.4)
    return sim


def test_collinear_cells_spanning_a_chamber_buckle(backend):
    """test_contact_dynamics.py:551-573: growth that ignores load turns the
    pair out of line; a perfectly straight pair with a load response stalls."""
    from microsimulator_b200.types import GrowthLoadLaw, GrowthLoadResponse

    sim = spanning_pair(backend, 0.01)
    parameters = ContactDynamicsParameters()
    result = sim.step(0.0, parameters)
    for _ in range(12):
        result = sim.step(0.05, parameters)
    w = sim.world
    assert np.all(np.abs(w.direction_y) > 0.3)
    assert np.all(w.lengths > 1.2 * 1.6)
    assert result.report.max_overlap < 0.01
    assert np.all(np.abs(w.position_z) < 1e-3)

    straight = spanning_pair(backend, 0.0)
    stalling = ContactDynamicsParameters(growth=GrowthLoadResponse(GrowthLoadLaw.LINEAR, stall_load=4.0))
    stalling.wall_stiffness = stalling.contact_stiffness
    for _ in range(40):
        straight.step(0.05, stalling)
    w = straight.world
    assert np.all(w.direction_y == 0.0)
    assert np.all(np.abs(w.lengths - 1.2) <= 5e-3)
