"""The B200 contact backend behind the reference's ComputeBackend contact
methods (cpp/include/microsimulator/backend.hpp:35-43), through the C-ABI of
``include/msb200.h``.

Every call runs on the GPU; there is no CPU path.  Errors come back as the
exceptions the reference raises: ``ValueError`` for std::invalid_argument,
``OverflowError`` for std::overflow_error, ``abi.NativeError`` (a
RuntimeError) for std::runtime_error and CUDA failures.

The native calls release the GIL (ctypes does), so, as the reference's
bindings do (cpp/python/native_call.hpp:19-84), a backend is marked busy for
the length of each call and a call from another thread meanwhile raises
RuntimeError("native object is in use by another thread") instead of racing
on the context.
"""

from __future__ import annotations

import ctypes
import functools
import threading
from ctypes import c_float, c_uint32, c_uint64, c_void_p

import numpy as np

from . import abi
from .graph import ContactGraph, ExternalContactGraph
from .types import (
    ConstraintContactParameters,
    ContactDynamicsParameters,
    ContactDynamicsReport,
    ContactDynamicsResult,
    ContactParameters,
    ContactResponse,
    ContactSolveParameters,
    ContactSolveReport,
    ContactSolveResult,
    ContactSystem,
)


def device_count() -> int:
    """cuda_backend_device_count()."""
    return int(abi.load_library().msb_device_count())


IN_USE = "native object is in use by another thread"


def _exclusive(method):
    """One call at a time per backend: the calling thread holds the
    backend's busy lock for the call (re-entered by its own nested calls);
    another thread's call raises RuntimeError, as BusyObjects::enter does."""

    @functools.wraps(method)
    def call(self, *args, **kwargs):
        busy = self.__dict__.get("_busy")
        if busy is None:
            return method(self, *args, **kwargs)
        if not busy.acquire(blocking=False):
            raise abi.NativeError(abi.ERR_RUNTIME, IN_USE)
        try:
            return method(self, *args, **kwargs)
        finally:
            busy.release()

    return call


def _calls_exclusive(cls):
    """Wraps every public method of `cls` in _exclusive."""
    for name, member in list(vars(cls).items()):
        if name.startswith("_") or isinstance(member, (staticmethod, classmethod)) or not callable(member):
            continue
        setattr(cls, name, _exclusive(member))
    return cls


@_calls_exclusive
class B200Backend:
    """make_cuda_backend(device_index): one context, one stream, its buffers."""

    def __init__(self, device_index: int = 0, library=None):
        """`library`: a path to load instead of libmsb200.so (the checked
        build, ``build.CHECKED_OUTPUT``)."""
        self._busy = threading.RLock()
        self._lib = abi.load_library(library)
        handle = c_void_p()
        status = self._lib.msb_context_create(device_index, ctypes.byref(handle))
        if status != abi.OK:
            raise abi.NativeError(status, f"could not create a B200 backend on device {device_index} (status {status})")
        self._handle = handle
        self.device_index = device_index
        self._capacity = 1024

    def close(self) -> None:
        if getattr(self, "_handle", None):
            self._lib.msb_context_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- helpers --------------------------------------------------------
    def _check(self, status: int) -> None:
        if status != abi.OK:
            abi.raise_for_status(status, self._lib.msb_last_error(self._handle).decode())

    def info(self) -> dict:
        buffer = ctypes.create_string_buffer(256)
        self._check(self._lib.msb_backend_info(self._handle, buffer, 256))
        return {"kind": "cuda", "name": "B200 contact backend", "device": buffer.value.decode(),
                "device_index": self.device_index, "native": True}

    def launch_count(self) -> int:
        return int(self._lib.msb_launch_count(self._handle))

    RELAXATION_AUTOMATIC = 0
    RELAXATION_GRAPH = 1
    RELAXATION_FUSED = 2

    def set_relaxation(self, form: int) -> None:
        """The BB relaxation's form on the device: 0 automatic, 1 a CUDA
        graph with a WHILE node (two kernels per iteration), 2 one persistent
        cooperative kernel with grid barriers."""
        self._check(self._lib.msb_set_relaxation(self._handle, form))

    WARM_START_ZERO = 0
    WARM_START_CARRY = 1
    WARM_START_GUESS = 2
    WARM_START_LEARNED = 4

    def set_warm_start(self, mode: int) -> None:
        """Flags: 0 the reference's semantics; 1 carry the previous step's
        final forces; 2 move the start multipliers toward the forces that a
        motion guess asks of each body; 4 let the warm-start network make
        that guess each step (see learned.py)."""
        self._check(self._lib.msb_set_warm_start(self._handle, mode))

    def set_motion_guess(self, guess, dt: float) -> None:
        """(cells, 3) float32 displacement guess (dx, dy, dtheta) over dt for
        the next step, or None to clear it."""
        if guess is None:
            self._check(self._lib.msb_set_motion_guess(self._handle, None, 0, c_float(dt)))
            return
        g = np.ascontiguousarray(guess, dtype=np.float32)
        if g.ndim != 2 or g.shape[1] != 3:
            raise ValueError("motion guess must have shape (cells, 3)")
        self._check(self._lib.msb_set_motion_guess(self._handle, c_void_p(abi.ptr(g)), g.shape[0], c_float(dt)))

    SOLVE_RECORD_DTYPE = np.dtype([("rows", "<u4"), ("iterations", "<u4"), ("status", "<u4"), ("residual", "<f4")])

    def last_step_solves(self) -> np.ndarray:
        """The solves of the last step in order: rows, iterations, status and
        residual of each."""
        count = ctypes.c_uint32(0)
        out = np.zeros(64, dtype=self.SOLVE_RECORD_DTYPE)
        status = self._lib.msb_last_step_solves(self._handle, c_void_p(abi.ptr(out)), len(out), ctypes.byref(count))
        if status == abi.ERR_CAPACITY:
            out = np.zeros(count.value, dtype=self.SOLVE_RECORD_DTYPE)
            status = self._lib.msb_last_step_solves(self._handle, c_void_p(abi.ptr(out)), len(out),
                                                    ctypes.byref(count))
        self._check(status)
        return out[: count.value].copy()

    def last_step_searches(self) -> dict:
        """The last step's overlap re-checks by how their candidates were
        found: a full search, the substep's kept candidates, or the kept
        candidates with a partial re-search of the cells that moved."""
        full, kept, partial = c_uint32(0), c_uint32(0), c_uint32(0)
        self._check(self._lib.msb_last_step_searches(self._handle, ctypes.byref(full), ctypes.byref(kept),
                                                     ctypes.byref(partial)))
        return {"full": full.value, "kept": kept.value, "partial": partial.value}

    def set_search_reuse(self, mode: int) -> None:
        """0: the re-checks use every kind of search (the default); 1: no
        partial re-search; 2: a full search each time."""
        self._check(self._lib.msb_set_search_reuse(self._handle, mode))

    PHASES = ("load", "search", "rows", "incidence", "solve", "move", "output", "guess")

    def last_step_phases(self) -> dict:
        """Device milliseconds of the last step by phase (CUDA events)."""
        out = np.zeros(len(self.PHASES), dtype=np.float64)
        self._check(self._lib.msb_last_step_phases(self._handle, c_void_p(abi.ptr(out)), len(out)))
        return dict(zip(self.PHASES, out.tolist()))

    def profile_iterations(self, iterations: int = 20) -> dict:
        """Mean device time of one BB iteration's body and row passes on the
        last solved system (CUDA events on the backend's stream)."""
        body, row = c_float(0), c_float(0)
        rows, bodies = c_uint64(0), c_uint64(0)
        self._check(self._lib.msb_profile_iterations(self._handle, iterations, ctypes.byref(body), ctypes.byref(row),
                                                     ctypes.byref(rows), ctypes.byref(bodies)))
        return {"body_ms": body.value, "row_ms": row.value, "rows": rows.value, "bodies": bodies.value}

    def _records(self, call, dtype, guess: int):
        capacity = max(self._capacity, guess)
        while True:
            out = np.zeros(capacity, dtype=dtype)
            count = c_uint64(0)
            status = call(out, capacity, count)
            if status == abi.ERR_CAPACITY:
                capacity = int(count.value) + 16
                continue
            self._check(status)
            self._capacity = max(self._capacity, int(count.value))
            return out[: count.value].copy()

    # -- ComputeBackend -------------------------------------------------
    def find_cell_contacts(self, world, parameters: ContactParameters | None = None) -> np.ndarray:
        """Contacts as ``abi.CELL_CONTACT_DTYPE`` records in (first id,
        second id, ordinal) order."""
        parameters = parameters or ContactParameters()
        cells = world.arrays()
        native = parameters.native()
        return self._records(
            lambda out, cap, count: self._lib.msb_find_cell_contacts(
                self._handle, ctypes.byref(cells), ctypes.byref(native), c_void_p(abi.ptr(out)), cap,
                ctypes.byref(count)),
            abi.CELL_CONTACT_DTYPE,
            8 * len(world),
        )

    def find_cell_contact_graph(self, world, parameters: ContactParameters | None = None) -> ContactGraph:
        """find_cell_contacts returning the whole ContactGraph: the contacts
        and their incidence and neighbour index, built on the device from the
        contacts as found."""
        parameters = parameters or ContactParameters()
        cells = world.arrays()
        native = parameters.native()
        n = len(world)
        capacity = max(self._capacity, 8 * n)
        while True:
            contacts = np.zeros(capacity, dtype=abi.CELL_CONTACT_DTYPE)
            index, arrays = self._index_arrays(n, 2 * capacity, True)
            count = c_uint64(0)
            status = self._lib.msb_find_cell_contact_graph(self._handle, ctypes.byref(cells), ctypes.byref(native),
                                                           c_void_p(abi.ptr(contacts)), capacity,
                                                           ctypes.byref(count), ctypes.byref(index))
            if status == abi.ERR_CAPACITY and count.value > capacity:
                capacity = int(count.value) + 16
                continue
            self._check(status)
            self._capacity = max(self._capacity, int(count.value))
            return self._graph(n, contacts[: count.value].copy(), index, arrays)

    def build_contact_graph(self, contacts: np.ndarray, cell_count: int) -> ContactGraph:
        """ContactGraph(cell_count, contacts) (contact_graph.cpp:302-349) on
        the device: validation, incidence and neighbours."""
        records = np.ascontiguousarray(contacts, dtype=abi.CELL_CONTACT_DTYPE)
        index, arrays = self._index_arrays(cell_count, 2 * len(records), True)
        self._check(self._lib.msb_build_contact_graph(self._handle, c_void_p(abi.ptr(records)), len(records),
                                                      cell_count, 0, ctypes.byref(index)))
        return self._graph(cell_count, records.copy(), index, arrays)

    def find_external_contact_graph(self, world, constraints,
                                    parameters: ConstraintContactParameters | None = None,
                                    every_face: bool = False) -> ExternalContactGraph:
        """find_external_contacts returning its whole ExternalContactGraph:
        the contacts and their incidence, built on the device from the
        contacts as found."""
        parameters = parameters or ConstraintContactParameters()
        cells = world.arrays()
        native = parameters.native()
        n = len(world)
        capacity = max(self._capacity, 4 * n + 16)
        while True:
            contacts = np.zeros(capacity, dtype=abi.EXTERNAL_CONTACT_DTYPE)
            offsets = np.zeros(n + 1, dtype=np.uint64)
            indices = np.zeros(capacity, dtype=np.uint64)
            count = c_uint64(0)
            status = self._lib.msb_find_external_contact_graph(
                self._handle, ctypes.byref(cells), c_void_p(constraints.pointer()), len(constraints),
                ctypes.byref(native), 1 if every_face else 0, c_void_p(abi.ptr(contacts)), capacity,
                ctypes.byref(count), c_void_p(abi.ptr(offsets)), c_void_p(abi.ptr(indices)))
            if status == abi.ERR_CAPACITY and count.value > capacity:
                capacity = int(count.value) + 16
                continue
            self._check(status)
            total = int(count.value)
            return ExternalContactGraph(n, contacts[:total].copy(), offsets, indices[:total].copy())

    def build_contact_graph_device(self, contacts_pointer: int, count: int, cell_count: int, index) -> int:
        """msb_build_contact_graph on device-resident contact records and
        index arrays (``graph.device_index``); returns the packed neighbour
        id count."""
        self._check(self._lib.msb_build_contact_graph(self._handle, c_void_p(contacts_pointer), count, cell_count, 1,
                                                      ctypes.byref(index)))
        return int(index.neighbor_count)

    def build_external_contact_graph(self, contacts: np.ndarray, cell_count: int) -> ExternalContactGraph:
        """ExternalContactGraph(cell_count, contacts) (constraints.cpp:288-307)."""
        records = np.ascontiguousarray(contacts, dtype=abi.EXTERNAL_CONTACT_DTYPE)
        offsets = np.zeros(int(cell_count) + 1, dtype=np.uint64)
        indices = np.zeros(max(1, len(records)), dtype=np.uint64)
        self._check(self._lib.msb_build_external_contact_graph(
            self._handle, c_void_p(abi.ptr(records)), len(records), cell_count, 0, c_void_p(abi.ptr(offsets)),
            c_void_p(abi.ptr(indices))))
        return ExternalContactGraph(cell_count, records.copy(), offsets, indices[: len(records)])

    @staticmethod
    def _index_arrays(cell_count: int, entries: int, neighbors: bool):
        arrays = {
            "incidence_offsets": np.zeros(int(cell_count) + 1, dtype=np.uint64),
            "incidence_contacts": np.zeros(max(1, entries), dtype=np.uint64),
        }
        if neighbors:
            arrays["neighbor_offsets"] = np.zeros(int(cell_count) + 1, dtype=np.uint64)
            arrays["neighbor_ids"] = np.zeros(max(1, entries), dtype=np.uint64)
        index = abi.ContactGraphIndex()
        for name, array in arrays.items():
            setattr(index, name, abi.ptr(array))
        index.neighbor_capacity = entries if neighbors else 0
        return index, arrays

    @staticmethod
    def _graph(cell_count, contacts, index, arrays) -> ContactGraph:
        return ContactGraph(cell_count, contacts, arrays["incidence_offsets"],
                            arrays["incidence_contacts"][: 2 * len(contacts)], arrays["neighbor_offsets"],
                            arrays["neighbor_ids"][: index.neighbor_count])

    def find_external_contacts(self, world, constraints, parameters: ConstraintContactParameters | None = None,
                               every_face: bool = False) -> np.ndarray:
        """find_external_contacts (nearest face) or, with ``every_face``,
        find_external_contact_faces; ``abi.EXTERNAL_CONTACT_DTYPE`` records."""
        parameters = parameters or ConstraintContactParameters()
        cells = world.arrays()
        native = parameters.native()
        return self._records(
            lambda out, cap, count: self._lib.msb_find_external_contacts(
                self._handle, ctypes.byref(cells), c_void_p(constraints.pointer()), len(constraints),
                ctypes.byref(native), 1 if every_face else 0, c_void_p(abi.ptr(out)), cap, ctypes.byref(count)),
            abi.EXTERNAL_CONTACT_DTYPE,
            4 * len(world) + 16,
        )

    def solve_contact_forces(self, system: ContactSystem, initial_multipliers,
                             parameters: ContactSolveParameters | None = None) -> ContactSolveResult:
        parameters = parameters or ContactSolveParameters()
        native = system.native()
        initial = np.ascontiguousarray(initial_multipliers, dtype=np.float32)
        if initial.shape[0] != len(system.rows):
            raise ValueError("contact multiplier count does not match the contact rows")
        out = np.zeros(len(system.rows), dtype=np.float32)
        report = abi.ContactSolveReport()
        prm = parameters.native()
        self._check(self._lib.msb_solve_contact_forces(
            self._handle, ctypes.byref(native), c_void_p(abi.ptr(initial) if len(initial) else None),
            ctypes.byref(prm), c_void_p(abi.ptr(out) if len(out) else None), ctypes.byref(report)))
        if len(system.rows) == 0:
            out = initial.copy()
        return ContactSolveResult(out, ContactSolveReport(report.status, report.iterations, report.residual))

    def evaluate_contact_response(self, system: ContactSystem, multipliers) -> ContactResponse:
        native = system.native()
        multipliers = np.ascontiguousarray(multipliers, dtype=np.float32)
        if multipliers.shape[0] != len(system.rows):
            raise ValueError("contact multiplier count does not match the contact rows")
        n = len(system.bodies)
        velocities = np.zeros((n, 6), dtype=np.float32)
        loads = np.zeros(n, dtype=np.float32)
        rates = np.zeros(n, dtype=np.float32)
        self._check(self._lib.msb_evaluate_contact_response(
            self._handle, ctypes.byref(native), c_void_p(abi.ptr(multipliers) if len(multipliers) else None),
            c_void_p(abi.ptr(velocities)), c_void_p(abi.ptr(loads)), c_void_p(abi.ptr(rates))))
        return ContactResponse(velocities, loads, rates)

    def evaluate_contact_gaps(self, system: ContactSystem, multipliers) -> np.ndarray:
        native = system.native()
        multipliers = np.ascontiguousarray(multipliers, dtype=np.float32)
        if multipliers.shape[0] != len(system.rows):
            raise ValueError("contact multiplier count does not match the contact rows")
        gaps = np.zeros(len(system.rows), dtype=np.float32)
        self._check(self._lib.msb_evaluate_contact_gaps(
            self._handle, ctypes.byref(native), c_void_p(abi.ptr(multipliers) if len(multipliers) else None),
            c_void_p(abi.ptr(gaps) if len(gaps) else None)))
        return gaps

    def contact_system_diagonal_bound(self, system: ContactSystem) -> float:
        native = system.native()
        bound = c_float(0.0)
        self._check(self._lib.msb_contact_system_diagonal_bound(self._handle, ctypes.byref(native),
                                                               ctypes.byref(bound)))
        return bound.value

    def advance_contact_dynamics(self, world, constraints, dt: float,
                                 dynamics: ContactDynamicsParameters | None = None,
                                 contacts: ContactParameters | None = None,
                                 constraint_parameters: ConstraintContactParameters | None = None,
                                 outputs=None) -> ContactDynamicsResult:
        """One contact-dynamics step of ``world`` (updated in place) with
        host buffers: the upload, the step and the download in one call.
        ``world`` is a WorldState or any object with its arrays (such as
        PinnedCells, whose page-locked arrays the library copies without
        staging).  ``outputs`` (velocities n x 3, loads n, increments n,
        float32) receives the step's outputs; new arrays without it."""
        dynamics = dynamics or ContactDynamicsParameters()
        contacts = contacts or ContactParameters()
        constraint_parameters = constraint_parameters or ConstraintContactParameters()
        n = len(world)
        cells = world.arrays()
        if outputs is None:
            velocities = np.zeros((n, 3), dtype=np.float32)
            loads = np.zeros(n, dtype=np.float32)
            increments = np.zeros(n, dtype=np.float32)
        else:
            velocities, loads, increments = outputs
            for array, shape in ((velocities, (n, 3)), (loads, (n,)), (increments, (n,))):
                if array.dtype != np.float32 or array.shape != shape or not array.flags.c_contiguous:
                    raise ValueError("outputs must be C-contiguous float32 arrays of shapes (n, 3), (n,), (n,)")
        outputs = abi.ContactDynamicsOutputs(abi.ptr(velocities), abi.ptr(loads), abi.ptr(increments))
        report = abi.ContactDynamicsReport()
        dyn, cp, wp = dynamics.native(), contacts.native(), constraint_parameters.native()
        pointer = constraints.pointer() if constraints is not None else None
        count = len(constraints) if constraints is not None else 0
        self._check(self._lib.msb_advance_contact_dynamics(
            self._handle, ctypes.byref(cells), c_void_p(pointer), count, c_float(dt), ctypes.byref(dyn),
            ctypes.byref(cp), ctypes.byref(wp), ctypes.byref(report), ctypes.byref(outputs)))
        return ContactDynamicsResult(ContactDynamicsReport.from_native(report), velocities, loads, increments)

    def advance_contact_dynamics_batch(self, cells, colony_cells, drag, stiffness, dt: float,
                                       dynamics: ContactDynamicsParameters | None = None,
                                       contacts: ContactParameters | None = None, outputs=None):
        """One step of a batch of independent colonies laid out colony after
        colony in ``cells`` (a WorldState, updated in place, or DeviceCells),
        each with its own drag and contact stiffness.  Returns the batch's
        report and one ``abi.COLONY_REPORT_DTYPE`` record per colony."""
        dynamics = dynamics or ContactDynamicsParameters()
        contacts = contacts or ContactParameters()
        counts = np.ascontiguousarray(colony_cells, dtype=np.uint32)
        k = counts.shape[0]
        params = (abi.ColonyParameters * k)()
        for i, (d, s) in enumerate(zip(np.asarray(drag, np.float32), np.asarray(stiffness, np.float32))):
            params[i] = abi.ColonyParameters(float(d), float(s))
        reports = np.zeros(k, dtype=abi.COLONY_REPORT_DTYPE)
        report = abi.ContactDynamicsReport()
        dyn, cp = dynamics.native(), contacts.native()
        device = isinstance(cells, DeviceCells)
        arrays = cells.arrays()
        native_outputs = outputs.native() if outputs is not None else None
        self._check(self._lib.msb_advance_contact_dynamics_batch(
            self._handle, ctypes.byref(arrays), c_void_p(abi.ptr(counts)), k, ctypes.byref(params), c_float(dt),
            ctypes.byref(dyn), ctypes.byref(cp), ctypes.byref(report), c_void_p(abi.ptr(reports)),
            ctypes.byref(native_outputs) if native_outputs is not None else None, 1 if device else 0))
        return ContactDynamicsReport.from_native(report), reports

    def set_flow_field(self, field) -> None:
        """Gives the backend a flow field (a ``FlowField``) for steps with
        ``flow_drift``; None removes it."""
        if field is None:
            self._check(self._lib.msb_set_flow_field(self._handle, None))
            return
        native = field.native()
        self._check(self._lib.msb_set_flow_field(self._handle, ctypes.byref(native)))

    def tune_batch(self) -> None:
        """Ask for a new tuning of the batched launch at the next batch call."""
        self._check(self._lib.msb_tune_batch(self._handle))

    def batch_tuning(self) -> dict:
        cluster, threads, lean, scale = ctypes.c_uint32(0), ctypes.c_uint32(0), ctypes.c_uint32(0), c_float(0)
        self._check(self._lib.msb_batch_tuning(self._handle, ctypes.byref(cluster), ctypes.byref(threads),
                                               ctypes.byref(lean), ctypes.byref(scale)))
        return {"cluster": cluster.value, "threads": threads.value, "lean": bool(lean.value),
                "box_scale": scale.value}

    def advance_contact_dynamics_device(self, cells: "DeviceCells", constraints, dt: float,
                                        dynamics: ContactDynamicsParameters | None = None,
                                        contacts: ContactParameters | None = None,
                                        constraint_parameters: ConstraintContactParameters | None = None,
                                        outputs: "DeviceOutputs | None" = None) -> ContactDynamicsReport:
        """The same step on cells held in device memory (``DeviceCells``)."""
        dynamics = dynamics or ContactDynamicsParameters()
        contacts = contacts or ContactParameters()
        constraint_parameters = constraint_parameters or ConstraintContactParameters()
        native_cells = cells.arrays()
        native_outputs = outputs.native() if outputs is not None else None
        report = abi.ContactDynamicsReport()
        dyn, cp, wp = dynamics.native(), contacts.native(), constraint_parameters.native()
        pointer = constraints.pointer() if constraints is not None else None
        count = len(constraints) if constraints is not None else 0
        self._check(self._lib.msb_advance_contact_dynamics_device(
            self._handle, ctypes.byref(native_cells), c_void_p(pointer), count, c_float(dt), ctypes.byref(dyn),
            ctypes.byref(cp), ctypes.byref(wp), ctypes.byref(report),
            ctypes.byref(native_outputs) if native_outputs is not None else None))
        return ContactDynamicsReport.from_native(report)


class DeviceCells:
    """A world's arrays resident in GPU memory (torch tensors used as
    allocations only), for ``advance_contact_dynamics_device``."""

    def __init__(self, world, device: str = "cuda:0"):
        import torch

        def up(array, dtype):
            return torch.from_numpy(np.array(array)).to(device=device, dtype=dtype)

        self.count = len(world)
        self.ids = up(world.ids.view(np.int64), torch.int64)
        self.fields = {name: up(getattr(world, name), torch.float32) for name in world.FIELDS}
        self.fixed = up(world.fixed, torch.uint8)

    def arrays(self) -> abi.CellArrays:
        f = self.fields
        return abi.CellArrays(
            self.count, self.ids.data_ptr(), f["position_x"].data_ptr(), f["position_y"].data_ptr(),
            f["position_z"].data_ptr(), f["direction_x"].data_ptr(), f["direction_y"].data_ptr(),
            f["direction_z"].data_ptr(), f["lengths"].data_ptr(), f["radii"].data_ptr(),
            f["growth_rates"].data_ptr(), self.fixed.data_ptr())

    def download(self, world) -> None:
        for name in ("position_x", "position_y", "position_z", "direction_x", "direction_y", "direction_z",
                     "lengths"):
            setattr(world, name, self.fields[name].cpu().numpy().copy())


class PinnedCells:
    """A world's arrays in page-locked host memory (pinned torch tensors
    viewed as numpy arrays), which the host-buffer calls copy to and from the
    device directly.  ``load`` copies a WorldState in, ``store`` copies the
    stepped geometry back; ``outputs`` are pinned output arrays for
    ``advance_contact_dynamics(..., outputs=...)``."""

    FIELDS = ("position_x", "position_y", "position_z", "direction_x", "direction_y", "direction_z", "lengths",
              "radii", "growth_rates")

    def __init__(self, capacity: int):
        import torch

        def pinned(count, dtype):
            return torch.empty(count, dtype=dtype, pin_memory=True).numpy()

        self.capacity = int(capacity)
        self.count = 0
        self._ids = pinned(self.capacity, torch.int64).view(np.uint64)
        self._fields = {name: pinned(self.capacity, torch.float32) for name in self.FIELDS}
        self._fixed = pinned(self.capacity, torch.uint8)
        self._velocities = pinned(3 * self.capacity, torch.float32)
        self._loads = pinned(self.capacity, torch.float32)
        self._increments = pinned(self.capacity, torch.float32)

    def __len__(self) -> int:
        return self.count

    def load(self, world) -> None:
        n = len(world)
        if n > self.capacity:
            raise ValueError(f"{n} cells exceed the pinned capacity {self.capacity}")
        self.count = n
        self._ids[:n] = world.ids
        for name in self.FIELDS:
            self._fields[name][:n] = getattr(world, name)
        self._fixed[:n] = world.fixed

    def store(self, world) -> None:
        n = self.count
        for name in ("position_x", "position_y", "position_z", "direction_x", "direction_y", "direction_z",
                     "lengths"):
            setattr(world, name, self._fields[name][:n].copy())

    def outputs(self):
        n = self.count
        return self._velocities[:3 * n].reshape(n, 3), self._loads[:n], self._increments[:n]

    def arrays(self) -> abi.CellArrays:
        f = self._fields
        return abi.CellArrays(
            self.count, abi.ptr(self._ids), abi.ptr(f["position_x"]), abi.ptr(f["position_y"]),
            abi.ptr(f["position_z"]), abi.ptr(f["direction_x"]), abi.ptr(f["direction_y"]),
            abi.ptr(f["direction_z"]), abi.ptr(f["lengths"]), abi.ptr(f["radii"]), abi.ptr(f["growth_rates"]),
            abi.ptr(self._fixed))


class DeviceOutputs:
    def __init__(self, count: int, device: str = "cuda:0"):
        import torch

        self.velocities = torch.zeros((count, 3), dtype=torch.float32, device=device)
        self.loads = torch.zeros(count, dtype=torch.float32, device=device)
        self.increments = torch.zeros(count, dtype=torch.float32, device=device)

    def native(self) -> abi.ContactDynamicsOutputs:
        return abi.ContactDynamicsOutputs(self.velocities.data_ptr(), self.loads.data_ptr(),
                                          self.increments.data_ptr())
