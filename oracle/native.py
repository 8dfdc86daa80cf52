"""Test infrastructure: ctypes access to the two CPU checkers.

* ``Oracle``    - ``_build/liboracle.so``, the CPU restatement of the contact
  path in contact_oracle.cpp (``precision=32`` follows the reference's FP32
  arithmetic bit for bit; ``precision=64`` is the FP64 oracle).
* ``Reference`` - ``_ref/libmsref.so``, the reference MicroSimulator CPU
  backend itself, compiled from its sources by oracle/Makefile.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module; the product never does.  Both take the same inputs as the CUDA
backend (``microsimulator_b200.world`` containers, ``types`` parameters) and
return the same structured arrays.
"""

from __future__ import annotations

import ctypes
import subprocess
from ctypes import POINTER, c_char_p, c_float, c_int, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

from microsimulator_b200 import abi
from microsimulator_b200.types import (
    ConstraintContactParameters,
    ContactDynamicsParameters,
    ContactDynamicsReport,
    ContactDynamicsResult,
    ContactParameters,
    ContactResponse,
    ContactSolveParameters,
    ContactSolveReport,
    ContactSolveResult,
)

HERE = Path(__file__).resolve().parent
ORACLE_PATH = HERE / "_build" / "liboracle.so"
REFERENCE_PATH = HERE / "_ref" / "libmsref.so"


def build(reference: bool = True) -> None:
    """Builds the checkers (the reference only where its sources exist)."""
    targets = ["oracle"]
    if reference and Path("/root/reference/cpp").exists():
        targets.append("ref")
        # The reference's conformance tests against the B200 adapter need
        # libmsb200.so built first.
        if (HERE.parent / "microsimulator_b200" / "libmsb200.so").exists():
            targets.append("conformance")
    subprocess.run(["make", "-s", "-C", str(HERE), "-j8", *targets], check=True)


def _errcheck(library, last_error):
    def check(status: int) -> None:
        if status == abi.OK:
            return
        abi.raise_for_status(status, last_error().decode())

    return check


class _Checker:
    prefix = ""

    def __init__(self, path: Path):
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing; run oracle.native.build()")
        self.lib = ctypes.CDLL(str(path))

    def _call(self, name, *args) -> None:
        status = getattr(self.lib, self.prefix + name)(*args)
        if status != abi.OK:
            message = getattr(self.lib, self.prefix + "last_error")().decode()
            abi.raise_for_status(status, message)

    @staticmethod
    def _grow(call, dtype):
        """Calls ``call(buffer, capacity, count)`` until the buffer fits."""
        capacity = 1024
        while True:
            out = np.zeros(capacity, dtype=dtype)
            count = c_uint64(0)
            try:
                call(out, capacity, count)
                return out[: count.value].copy()
            except abi.NativeError as error:
                if error.status != abi.ERR_CAPACITY:
                    raise
                capacity = max(int(count.value), 2 * capacity)


class Oracle(_Checker):
    """The CPU restatement (FP32 bit-faithful, or FP64)."""

    prefix = "oracle_"

    def __init__(self, path: Path = ORACLE_PATH):
        super().__init__(path)
        self.lib.oracle_last_error.restype = c_char_p

    def find_cell_contacts(self, world, parameters=None, precision=32):
        parameters = parameters or ContactParameters()
        cells = world.arrays()
        native = parameters.native()
        flag = 0 if precision == 32 else 1
        return self._grow(
            lambda out, cap, count: self._call(
                "find_cell_contacts",
                c_uint32(flag),
                ctypes.byref(cells),
                ctypes.byref(native),
                c_void_p(abi.ptr(out)),
                c_uint64(cap),
                ctypes.byref(count),
            ),
            abi.CELL_CONTACT_DTYPE,
        )

    def find_cell_contact_candidates(self, world, margin=0.01):
        cells = world.arrays()
        pairs = self._grow(
            lambda out, cap, count: self._call(
                "find_cell_contact_candidates",
                ctypes.byref(cells),
                c_float(margin),
                c_void_p(abi.ptr(out)),
                c_uint64(cap),
                ctypes.byref(count),
            ),
            np.dtype([("first_slot", "<u4"), ("second_slot", "<u4")]),
        )
        return pairs

    def find_external_contacts(self, world, constraints, parameters=None, every_face=False, precision=32):
        parameters = parameters or ConstraintContactParameters()
        cells = world.arrays()
        native = parameters.native()
        flag = 0 if precision == 32 else 1
        return self._grow(
            lambda out, cap, count: self._call(
                "find_external_contacts",
                c_uint32(flag),
                ctypes.byref(cells),
                c_void_p(constraints.pointer()),
                c_uint64(len(constraints)),
                ctypes.byref(native),
                c_uint32(1 if every_face else 0),
                c_void_p(abi.ptr(out)),
                c_uint64(cap),
                ctypes.byref(count),
            ),
            abi.EXTERNAL_CONTACT_DTYPE,
        )

    def solve_contact_forces(self, system, initial, parameters=None, precision=32):
        parameters = parameters or ContactSolveParameters()
        native = system.native()
        initial = np.ascontiguousarray(initial, dtype=np.float32)
        out = np.zeros(len(system.rows), dtype=np.float32)
        report = abi.ContactSolveReport()
        prm = parameters.native()
        self._call(
            "solve_contact_forces",
            c_uint32(0 if precision == 32 else 1),
            ctypes.byref(native),
            c_void_p(abi.ptr(initial)),
            ctypes.byref(prm),
            c_void_p(abi.ptr(out)),
            ctypes.byref(report),
        )
        return ContactSolveResult(out, ContactSolveReport(report.status, report.iterations, report.residual))

    def evaluate_contact_response(self, system, multipliers, precision=32):
        native = system.native()
        multipliers = np.ascontiguousarray(multipliers, dtype=np.float32)
        n = len(system.bodies)
        velocities = np.zeros((n, 6), dtype=np.float32)
        loads = np.zeros(n, dtype=np.float32)
        rates = np.zeros(n, dtype=np.float32)
        self._call(
            "evaluate_contact_response",
            c_uint32(0 if precision == 32 else 1),
            ctypes.byref(native),
            c_void_p(abi.ptr(multipliers)),
            c_void_p(abi.ptr(velocities)),
            c_void_p(abi.ptr(loads)),
            c_void_p(abi.ptr(rates)),
        )
        return ContactResponse(velocities, loads, rates)

    def evaluate_contact_gaps(self, system, multipliers, precision=32):
        native = system.native()
        multipliers = np.ascontiguousarray(multipliers, dtype=np.float32)
        gaps = np.zeros(len(system.rows), dtype=np.float32)
        self._call(
            "evaluate_contact_gaps",
            c_uint32(0 if precision == 32 else 1),
            ctypes.byref(native),
            c_void_p(abi.ptr(multipliers)),
            c_void_p(abi.ptr(gaps)),
        )
        return gaps

    def contact_system_diagonal_bound(self, system, precision=32):
        native = system.native()
        bound = c_float(0)
        self._call(
            "contact_system_diagonal_bound",
            c_uint32(0 if precision == 32 else 1),
            ctypes.byref(native),
            ctypes.byref(bound),
        )
        return bound.value

    def advance_contact_dynamics(self, world, constraints, dt, dynamics=None, contacts=None,
                                 constraint_parameters=None, precision=32):
        """Steps ``world`` in place; returns a ContactDynamicsResult."""
        return _advance(
            self, "advance_contact_dynamics", (c_uint32(0 if precision == 32 else 1),),
            world, constraints, dt, dynamics, contacts, constraint_parameters,
        )


class Reference(_Checker):
    """The reference MicroSimulator CPU backend (compiled from its sources)."""

    prefix = "ref_"

    def __init__(self, path: Path = REFERENCE_PATH):
        super().__init__(path)
        self.lib.ref_last_error.restype = c_char_p
        self.lib.ref_thread_count.restype = c_uint64
        self.lib.ref_world_create.restype = c_void_p
        self.lib.ref_world_create.argtypes = [c_void_p, c_void_p, c_uint64]
        self.lib.ref_world_destroy.argtypes = [c_void_p]
        self.lib.ref_world_size.restype = c_uint64
        self.lib.ref_world_size.argtypes = [c_void_p]

    def thread_count(self) -> int:
        return int(self.lib.ref_thread_count())

    def find_cell_contacts(self, world, parameters=None, exhaustive=False):
        parameters = parameters or ContactParameters()
        cells = world.arrays()
        native = parameters.native()
        return self._grow(
            lambda out, cap, count: self._call(
                "find_cell_contacts",
                ctypes.byref(cells),
                ctypes.byref(native),
                c_uint32(1 if exhaustive else 0),
                c_void_p(abi.ptr(out)),
                c_uint64(cap),
                ctypes.byref(count),
                None,
                None,
            ),
            abi.CELL_CONTACT_DTYPE,
        )

    def incidence(self, world, parameters=None):
        """ContactGraph incidence: (offsets, contact indices) by slot."""
        parameters = parameters or ContactParameters()
        contacts = self.find_cell_contacts(world, parameters)
        cells = world.arrays()
        native = parameters.native()
        offsets = np.zeros(len(world) + 1, dtype=np.uint64)
        indices = np.zeros(max(1, 2 * len(contacts)), dtype=np.uint64)
        out = np.zeros(max(1, len(contacts)), dtype=abi.CELL_CONTACT_DTYPE)
        count = c_uint64(0)
        self._call(
            "find_cell_contacts",
            ctypes.byref(cells),
            ctypes.byref(native),
            c_uint32(0),
            c_void_p(abi.ptr(out)),
            c_uint64(len(out)),
            ctypes.byref(count),
            c_void_p(abi.ptr(offsets)),
            c_void_p(abi.ptr(indices)),
        )
        return offsets, indices[: int(offsets[-1])]

    def contact_graph(self, contacts, cell_count):
        """ContactGraph(cell_count, contacts): (incidence offsets, incidence
        contact indices, neighbour offsets, neighbour ids)."""
        records = np.ascontiguousarray(contacts, dtype=abi.CELL_CONTACT_DTYPE)
        entries = max(1, 2 * len(records))
        incidence_offsets = np.zeros(int(cell_count) + 1, dtype=np.uint64)
        incidence = np.zeros(entries, dtype=np.uint64)
        neighbor_offsets = np.zeros(int(cell_count) + 1, dtype=np.uint64)
        neighbors = np.zeros(entries, dtype=np.uint64)
        count = c_uint64(0)
        self._call("contact_graph", c_void_p(abi.ptr(records)), c_uint64(len(records)), c_uint64(cell_count),
                   c_void_p(abi.ptr(incidence_offsets)), c_void_p(abi.ptr(incidence)),
                   c_void_p(abi.ptr(neighbor_offsets)), c_void_p(abi.ptr(neighbors)), c_uint64(entries),
                   ctypes.byref(count))
        return incidence_offsets, incidence[: 2 * len(records)], neighbor_offsets, neighbors[: count.value]

    def external_contact_graph(self, contacts, cell_count):
        """ExternalContactGraph(cell_count, contacts): (incidence offsets,
        incidence contact indices)."""
        records = np.ascontiguousarray(contacts, dtype=abi.EXTERNAL_CONTACT_DTYPE)
        offsets = np.zeros(int(cell_count) + 1, dtype=np.uint64)
        indices = np.zeros(max(1, len(records)), dtype=np.uint64)
        self._call("external_contact_graph", c_void_p(abi.ptr(records)), c_uint64(len(records)),
                   c_uint64(cell_count), c_void_p(abi.ptr(offsets)), c_void_p(abi.ptr(indices)))
        return offsets, indices[: len(records)]

    def find_cell_contact_candidates(self, world, parameters=None):
        parameters = parameters or ContactParameters()
        cells = world.arrays()
        native = parameters.native()
        return self._grow(
            lambda out, cap, count: self._call(
                "find_cell_contact_candidates",
                ctypes.byref(cells),
                ctypes.byref(native),
                c_void_p(abi.ptr(out)),
                c_uint64(cap),
                ctypes.byref(count),
            ),
            np.dtype([("first_slot", "<u4"), ("second_slot", "<u4")]),
        )

    def find_external_contacts(self, world, constraints, parameters=None, every_face=False):
        parameters = parameters or ConstraintContactParameters()
        cells = world.arrays()
        native = parameters.native()
        return self._grow(
            lambda out, cap, count: self._call(
                "find_external_contacts",
                ctypes.byref(cells),
                c_void_p(constraints.pointer()),
                c_uint64(len(constraints)),
                ctypes.byref(native),
                c_uint32(1 if every_face else 0),
                c_void_p(abi.ptr(out)),
                c_uint64(cap),
                ctypes.byref(count),
            ),
            abi.EXTERNAL_CONTACT_DTYPE,
        )

    def solve_contact_forces(self, system, initial, parameters=None):
        parameters = parameters or ContactSolveParameters()
        native = system.native()
        initial = np.ascontiguousarray(initial, dtype=np.float32)
        out = np.zeros(len(system.rows), dtype=np.float32)
        report = abi.ContactSolveReport()
        prm = parameters.native()
        self._call(
            "solve_contact_forces",
            ctypes.byref(native),
            c_void_p(abi.ptr(initial)),
            ctypes.byref(prm),
            c_void_p(abi.ptr(out)),
            ctypes.byref(report),
        )
        return ContactSolveResult(out, ContactSolveReport(report.status, report.iterations, report.residual))

    def evaluate_contact_response(self, system, multipliers):
        native = system.native()
        multipliers = np.ascontiguousarray(multipliers, dtype=np.float32)
        n = len(system.bodies)
        velocities = np.zeros((n, 6), dtype=np.float32)
        loads = np.zeros(n, dtype=np.float32)
        rates = np.zeros(n, dtype=np.float32)
        self._call(
            "evaluate_contact_response",
            ctypes.byref(native),
            c_void_p(abi.ptr(multipliers)),
            c_void_p(abi.ptr(velocities)),
            c_void_p(abi.ptr(loads)),
            c_void_p(abi.ptr(rates)),
        )
        return ContactResponse(velocities, loads, rates)

    def evaluate_contact_gaps(self, system, multipliers):
        native = system.native()
        multipliers = np.ascontiguousarray(multipliers, dtype=np.float32)
        gaps = np.zeros(len(system.rows), dtype=np.float32)
        self._call("evaluate_contact_gaps", ctypes.byref(native), c_void_p(abi.ptr(multipliers)), c_void_p(abi.ptr(gaps)))
        return gaps

    def contact_system_diagonal_bound(self, system):
        native = system.native()
        bound = c_float(0)
        self._call("contact_system_diagonal_bound", ctypes.byref(native), ctypes.byref(bound))
        return bound.value

    def advance_contact_dynamics(self, world, constraints, dt, dynamics=None, contacts=None,
                                 constraint_parameters=None):
        return _advance(self, "advance_contact_dynamics", (), world, constraints, dt, dynamics,
                        contacts, constraint_parameters)

    def flow_step(self, world, field, dt, dynamics=None) -> ContactDynamicsReport:
        """One Simulation::step of the reference with flow drift in `field`
        (a microsimulator_b200.types.FlowField); `world` (ids 1..n in slot
        order) is updated in place."""
        dynamics = dynamics or ContactDynamicsParameters()
        cells = world.arrays()
        native = field.native()
        dyn = dynamics.native()
        report = abi.ContactDynamicsReport()
        self._call("flow_step", ctypes.byref(cells), ctypes.byref(native), c_float(dt), ctypes.byref(dyn),
                   ctypes.byref(report))
        return ContactDynamicsReport.from_native(report)

    # -- a world held across calls (bench) ------------------------------
    def world_create(self, world, constraints=None):
        cells = world.arrays()
        pointer = constraints.pointer() if constraints is not None else None
        count = len(constraints) if constraints is not None else 0
        handle = self.lib.ref_world_create(ctypes.byref(cells), pointer, count)
        if not handle:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return handle

    def world_destroy(self, handle) -> None:
        self.lib.ref_world_destroy(c_void_p(handle))

    def world_step(self, handle, dt, dynamics=None) -> ContactDynamicsReport:
        dynamics = dynamics or ContactDynamicsParameters()
        native = dynamics.native()
        report = abi.ContactDynamicsReport()
        self._call("world_step", c_void_p(handle), c_float(dt), ctypes.byref(native), ctypes.byref(report))
        return ContactDynamicsReport.from_native(report)

    def world_divide(self, handle, parents, rotations) -> None:
        parents = np.ascontiguousarray(parents, dtype=np.uint64)
        rotations = np.ascontiguousarray(rotations, dtype=np.float32)
        self._call("world_divide", c_void_p(handle), c_void_p(abi.ptr(parents)), c_uint64(len(parents)),
                   c_void_p(abi.ptr(rotations)))

    def world_read(self, handle, world) -> None:
        n = int(self.lib.ref_world_size(c_void_p(handle)))
        arrays = [np.zeros(n, dtype=np.uint64)] + [np.zeros(n, dtype=np.float32) for _ in range(7)]
        self._call("world_read", c_void_p(handle), *(c_void_p(abi.ptr(a)) for a in arrays))
        world.ids = arrays[0]
        (world.position_x, world.position_y, world.position_z, world.direction_x, world.direction_y,
         world.direction_z, world.lengths) = arrays[1:]


def _advance(checker, name, prefix_args, world, constraints, dt, dynamics, contacts, constraint_parameters):
    dynamics = dynamics or ContactDynamicsParameters()
    contacts = contacts or ContactParameters()
    constraint_parameters = constraint_parameters or ConstraintContactParameters()
    n = len(world)
    cells = world.arrays()
    velocities = np.zeros((n, 3), dtype=np.float32)
    loads = np.zeros(n, dtype=np.float32)
    increments = np.zeros(n, dtype=np.float32)
    outputs = abi.ContactDynamicsOutputs(abi.ptr(velocities), abi.ptr(loads), abi.ptr(increments))
    report = abi.ContactDynamicsReport()
    dyn = dynamics.native()
    cp = contacts.native()
    wp = constraint_parameters.native()
    pointer = constraints.pointer() if constraints is not None else None
    count = len(constraints) if constraints is not None else 0
    checker._call(
        name,
        *prefix_args,
        ctypes.byref(cells),
        c_void_p(pointer),
        c_uint64(count),
        c_float(dt),
        ctypes.byref(dyn),
        ctypes.byref(cp),
        ctypes.byref(wp),
        ctypes.byref(report),
        ctypes.byref(outputs),
    )
    return ContactDynamicsResult(ContactDynamicsReport.from_native(report), velocities, loads, increments)
