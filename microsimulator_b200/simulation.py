"""``Simulation`` with the reference's contact-path surface
(cpp/include/microsimulator/simulation.hpp:16-119, the contact members):
cells and constraints held on the host, every contact computation on the B200
backend.

``step(dt, dynamics, contacts, constraints)`` advances growth and contact
together as Simulation::step does (cpp/core/simulation.cpp:387-488); a step
that fails leaves the cells unchanged and raises.
"""

from __future__ import annotations

import numpy as np

from .backend import B200Backend
from .graph import ContactGraph, ExternalContactGraph
from .types import (
    ConstraintContactParameters,
    ContactDynamicsParameters,
    ContactDynamicsResult,
    ContactParameters,
    ContactSolveParameters,
    ContactSolveResult,
    ContactSystem,
)
from .world import ConstraintSet, WorldState


class Simulation:
    def __init__(self, device_index: int = 0, backend: B200Backend | None = None):
        self.world = WorldState()
        self.constraints = ConstraintSet()
        self.backend = backend or B200Backend(device_index)
        self._time = 0.0

    # -- state ------------------------------------------------------------
    def time(self) -> float:
        return self._time

    def cell_count(self) -> int:
        return len(self.world)

    def add_cell(self, position=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0), length=3.5, radius=0.5,
                 growth_rate=1.0, fixed=False) -> int:
        return self.world.add_cell(position, direction, length, radius, growth_rate, fixed)

    def add_plane_constraint(self, **kwargs) -> int:
        return self.constraints.add_plane(**kwargs)

    def add_sphere_constraint(self, **kwargs) -> int:
        return self.constraints.add_sphere(**kwargs)

    def add_box_constraint(self, **kwargs) -> int:
        return self.constraints.add_box(**kwargs)

    def add_cylinder_constraint(self, **kwargs) -> int:
        return self.constraints.add_cylinder(**kwargs)

    def divide(self, parent_id: int, first_fraction: float) -> tuple[int, int]:
        return self.world.divide(parent_id, first_fraction)

    def divide_equal(self, parent_id: int) -> tuple[int, int]:
        return self.world.divide(parent_id, 0.5)

    def set_cell_geometry(self, cell_id: int, position, direction, length) -> None:
        self.world.set_cell_geometry(self.world.slot_of(cell_id), position, direction, length)

    def set_cell_fixed(self, cell_id: int, fixed: bool) -> None:
        self.world.set_cell_fixed(cell_id, fixed)

    def cell(self, cell_id: int) -> dict:
        w = self.world
        s = w.slot_of(cell_id)
        return {
            "id": int(w.ids[s]),
            "slot": s,
            "position": (float(w.position_x[s]), float(w.position_y[s]), float(w.position_z[s])),
            "direction": (float(w.direction_x[s]), float(w.direction_y[s]), float(w.direction_z[s])),
            "length": float(w.lengths[s]),
            "radius": float(w.radii[s]),
            "growth_rate": float(w.growth_rates[s]),
            "fixed": bool(w.fixed[s]),
        }

    # -- contact path ---------------------------------------------------------
    def step(self, dt: float, dynamics: ContactDynamicsParameters | None = None,
             contacts: ContactParameters | None = None,
             constraints: ConstraintContactParameters | None = None) -> ContactDynamicsResult:
        if not np.isfinite(dt) or dt < 0:
            raise ValueError("time step must be finite and non-negative")
        result = self.backend.advance_contact_dynamics(self.world, self.constraints, dt, dynamics, contacts,
                                                       constraints)
        self._time += float(dt)
        return result

    def find_cell_contacts(self, parameters: ContactParameters | None = None) -> ContactGraph:
        """Simulation::find_cell_contacts: the ContactGraph of the cells."""
        return self.backend.find_cell_contact_graph(self.world, parameters)

    def find_external_contacts(self, parameters: ConstraintContactParameters | None = None) -> ExternalContactGraph:
        """Simulation::find_external_contacts: the ExternalContactGraph of the
        cells against the constraints."""
        return self.backend.find_external_contact_graph(self.world, self.constraints, parameters)

    def solve_contact_system(self, system: ContactSystem, initial_multipliers,
                             parameters: ContactSolveParameters | None = None) -> ContactSolveResult:
        return self.backend.solve_contact_forces(system, initial_multipliers, parameters)
