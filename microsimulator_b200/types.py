"""Parameter and result types of the contact path, with the reference's names
and defaults, and their conversion to the C-ABI structs.

Defaults follow cpp/include/microsimulator/contact_graph.hpp:13-17,
constraints.hpp:141-144 and contact_dynamics.hpp:161-201 of the reference.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import abi


class GrowthLoadLaw:
    NONE = abi.GROWTH_LAW_NONE
    EXPONENTIAL = abi.GROWTH_LAW_EXPONENTIAL
    LINEAR = abi.GROWTH_LAW_LINEAR


class ContactSolveStatus:
    CONVERGED = abi.SOLVE_CONVERGED
    ITERATION_LIMIT = abi.SOLVE_ITERATION_LIMIT
    BREAKDOWN = abi.SOLVE_BREAKDOWN


class ConstraintRegion:
    OUTSIDE = abi.REGION_OUTSIDE
    INSIDE = abi.REGION_INSIDE


class RodContactLocation:
    NEGATIVE = abi.ROD_NEGATIVE
    POSITIVE = abi.ROD_POSITIVE
    INTERIOR = abi.ROD_INTERIOR


@dataclass
class ContactParameters:
    activation_margin: float = 0.01
    parallel_sine_threshold: float = 0.1
    degeneracy_epsilon: float = 1.0e-6

    def native(self) -> abi.ContactParameters:
        return abi.ContactParameters(
            self.activation_margin, self.parallel_sine_threshold, self.degeneracy_epsilon
        )


@dataclass
class ConstraintContactParameters:
    activation_margin: float = 0.0
    degeneracy_epsilon: float = 1.0e-6

    def native(self) -> abi.ConstraintContactParameters:
        return abi.ConstraintContactParameters(self.activation_margin, self.degeneracy_epsilon)


@dataclass
class GrowthLoadResponse:
    law: int = GrowthLoadLaw.NONE
    sensitivity: float = 0.0
    free_load: float = 0.0
    stall_load: float = 1.0

    def native(self) -> abi.GrowthLoadResponse:
        return abi.GrowthLoadResponse(self.law, self.sensitivity, self.free_load, self.stall_load)


@dataclass
class ContactDynamicsParameters:
    drag: float = 1.0
    contact_stiffness: float = 1.0e4
    wall_stiffness: float = 1.0e6
    overlap_tolerance: float = 1.0e-3
    candidate_margin: float = 0.1
    max_overlap_recovery: float = 0.05
    max_growth_fraction: float = 0.25
    max_iterations: int = 20000
    max_refinements: int = 10
    max_step_halvings: int = 12
    flow_drift: bool = False
    growth: GrowthLoadResponse = field(default_factory=GrowthLoadResponse)

    def native(self) -> abi.ContactDynamicsParameters:
        return abi.ContactDynamicsParameters(
            self.drag,
            self.contact_stiffness,
            self.wall_stiffness,
            self.overlap_tolerance,
            self.candidate_margin,
            self.max_overlap_recovery,
            self.max_growth_fraction,
            self.max_iterations,
            self.max_refinements,
            self.max_step_halvings,
            1 if self.flow_drift else 0,
            self.growth.native(),
        )


@dataclass
class ContactSolveParameters:
    tolerance: float = 2.5e-4
    max_iterations: int = 20000

    def native(self) -> abi.ContactSolveParameters:
        return abi.ContactSolveParameters(self.tolerance, self.max_iterations)


@dataclass
class ContactSolveReport:
    status: int = ContactSolveStatus.CONVERGED
    iterations: int = 0
    residual: float = 0.0


@dataclass
class ContactSolveResult:
    multipliers: np.ndarray
    report: ContactSolveReport


@dataclass
class ContactResponse:
    velocities: np.ndarray  # (bodies, 6)
    loads: np.ndarray
    length_rates: np.ndarray


@dataclass
class ContactDynamicsReport:
    substeps: int = 0
    halvings: int = 0
    refinements: int = 0
    iterations: int = 0
    max_rows: int = 0
    max_overlap: float = 0.0

    @classmethod
    def from_native(cls, report: abi.ContactDynamicsReport) -> "ContactDynamicsReport":
        return cls(
            report.substeps,
            report.halvings,
            report.refinements,
            report.iterations,
            report.max_rows,
            report.max_overlap,
        )


@dataclass
class ContactDynamicsResult:
    report: ContactDynamicsReport
    center_velocities: np.ndarray  # (cells, 3)
    axial_loads: np.ndarray
    length_increments: np.ndarray


@dataclass
class ContactSystem:
    """A substep's contact problem: rows and bodies as structured arrays
    (``abi.CONTACT_ROW_DTYPE`` / ``abi.CONTACT_BODY_DTYPE``)."""

    rows: np.ndarray
    bodies: np.ndarray
    dt: float
    growth: GrowthLoadResponse = field(default_factory=GrowthLoadResponse)

    def native(self) -> abi.ContactSystem:
        self.rows = np.ascontiguousarray(self.rows, dtype=abi.CONTACT_ROW_DTYPE)
        self.bodies = np.ascontiguousarray(self.bodies, dtype=abi.CONTACT_BODY_DTYPE)
        return abi.ContactSystem(
            abi.ptr(self.rows) if len(self.rows) else None,
            len(self.rows),
            abi.ptr(self.bodies) if len(self.bodies) else None,
            len(self.bodies),
            self.dt,
            self.growth.native(),
        )


def empty_rows(count: int) -> np.ndarray:
    rows = np.zeros(count, dtype=abi.CONTACT_ROW_DTYPE)
    rows["second_slot"] = abi.INVALID_SLOT
    return rows


def empty_bodies(count: int) -> np.ndarray:
    bodies = np.zeros(count, dtype=abi.CONTACT_BODY_DTYPE)
    bodies["axis"][:, 0] = 1.0
    return bodies


@dataclass
class FlowField:
    """A fluid velocity field on a lattice of sites, as the reference's
    SignalGridSpec (shape, origin, spacing, obstacles) with its
    SignalGridVelocityField: face velocities x-major,
    x_faces (sx + 1, sy, sz), y_faces (sx, sy + 1, sz), z_faces (sx, sy, sz + 1),
    obstacles (sx, sy, sz) nonzero for solid sites."""

    shape: tuple
    origin: tuple
    spacing: tuple
    x_faces: np.ndarray
    y_faces: np.ndarray
    z_faces: np.ndarray
    obstacles: np.ndarray | None = None

    def arrays(self):
        sx, sy, sz = self.shape
        xf = np.ascontiguousarray(self.x_faces, dtype=np.float32).reshape(-1)
        yf = np.ascontiguousarray(self.y_faces, dtype=np.float32).reshape(-1)
        zf = np.ascontiguousarray(self.z_faces, dtype=np.float32).reshape(-1)
        if xf.size != (sx + 1) * sy * sz or yf.size != sx * (sy + 1) * sz or zf.size != sx * sy * (sz + 1):
            raise ValueError("flow face arrays do not match the shape")
        ob = None
        if self.obstacles is not None:
            ob = np.ascontiguousarray(self.obstacles, dtype=np.uint8).reshape(-1)
            if ob.size != sx * sy * sz:
                raise ValueError("flow obstacles do not match the shape")
        return xf, yf, zf, ob

    def native(self) -> abi.FlowField:
        xf, yf, zf, ob = self.arrays()
        self._keep = (xf, yf, zf, ob)
        return abi.FlowField(self.shape[0], self.shape[1], self.shape[2], 0, abi.Vec3(*self.origin),
                             abi.Vec3(*self.spacing), abi.ptr(xf), abi.ptr(yf), abi.ptr(zf),
                             abi.ptr(ob) if ob is not None else None)
