"""ctypes mirror of ``include/msb200.h``, the backend's C-ABI.

The struct layouts here and in the header are one contract; a test checks
their sizes against the header's.  ``load_library()`` loads the in-tree
``libmsb200.so`` and raises when it is missing: there is no fallback.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int, c_size_t, c_uint8, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

PACKAGE_DIR = Path(__file__).resolve().parent
LIBRARY_PATH = PACKAGE_DIR / "libmsb200.so"

INVALID_SLOT = 0xFFFFFFFF

# msb_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OVERFLOW = 2
ERR_RUNTIME = 3
ERR_CUDA = 4
ERR_CAPACITY = 5
ERR_DEVICE_CHECK = 6
ERR_NO_DEVICE = 7

# msb_solve_status (ContactSolveStatus)
SOLVE_CONVERGED = 0
SOLVE_ITERATION_LIMIT = 1
SOLVE_BREAKDOWN = 2

# msb_growth_load_law (GrowthLoadLaw)
GROWTH_LAW_NONE = 0
GROWTH_LAW_EXPONENTIAL = 1
GROWTH_LAW_LINEAR = 2

# msb_constraint_kind / region / rod location
CONSTRAINT_PLANE = 0
CONSTRAINT_SPHERE = 1
CONSTRAINT_BOX = 2
CONSTRAINT_CYLINDER = 3
REGION_OUTSIDE = 0
REGION_INSIDE = 1
ROD_NEGATIVE = 0
ROD_POSITIVE = 1
ROD_INTERIOR = 2


class Vec3(ctypes.Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float)]


class CellArrays(ctypes.Structure):
    _fields_ = [
        ("count", c_uint64),
        ("ids", c_void_p),
        ("position_x", c_void_p),
        ("position_y", c_void_p),
        ("position_z", c_void_p),
        ("direction_x", c_void_p),
        ("direction_y", c_void_p),
        ("direction_z", c_void_p),
        ("lengths", c_void_p),
        ("radii", c_void_p),
        ("growth_rates", c_void_p),
        ("fixed", c_void_p),
    ]


class ContactParameters(ctypes.Structure):
    _fields_ = [
        ("activation_margin", c_float),
        ("parallel_sine_threshold", c_float),
        ("degeneracy_epsilon", c_float),
    ]


class CellContact(ctypes.Structure):
    _fields_ = [
        ("first_id", c_uint64),
        ("second_id", c_uint64),
        ("first_slot", c_uint32),
        ("second_slot", c_uint32),
        ("ordinal", c_uint32),
        ("point_on_first", Vec3),
        ("normal", Vec3),
        ("signed_separation", c_float),
        ("weight", c_float),
        ("reserved", c_uint32),
    ]


class Constraint(ctypes.Structure):
    _fields_ = [
        ("id", c_uint64),
        ("kind", c_uint32),
        ("allowed_region", c_uint32),
        ("a", Vec3),
        ("b", Vec3),
        ("radius", c_float),
        ("half_height", c_float),
        ("coefficient", c_float),
        ("reserved", c_uint32),
    ]


class ConstraintContactParameters(ctypes.Structure):
    _fields_ = [("activation_margin", c_float), ("degeneracy_epsilon", c_float)]


class ExternalContact(ctypes.Structure):
    _fields_ = [
        ("cell_id", c_uint64),
        ("constraint_id", c_uint64),
        ("cell_slot", c_uint32),
        ("constraint_kind", c_uint32),
        ("location", c_uint32),
        ("point_on_cell", Vec3),
        ("normal", Vec3),
        ("signed_separation", c_float),
        ("weight", c_float),
        ("reserved", c_uint32),
    ]


class GrowthLoadResponse(ctypes.Structure):
    _fields_ = [
        ("law", c_uint32),
        ("sensitivity", c_float),
        ("free_load", c_float),
        ("stall_load", c_float),
    ]


class ContactRow(ctypes.Structure):
    _fields_ = [
        ("first_slot", c_uint32),
        ("second_slot", c_uint32),
        ("first_jacobian", c_float * 6),
        ("second_jacobian", c_float * 6),
        ("first_length_lever", c_float),
        ("second_length_lever", c_float),
        ("offset", c_float),
        ("compliance", c_float),
    ]


class ContactBody(ctypes.Structure):
    _fields_ = [
        ("axis", Vec3),
        ("translational_mobility", c_float),
        ("transverse_mobility", c_float),
        ("axial_mobility", c_float),
        ("length_rate", c_float),
        ("drift", c_float * 6),
    ]


class ContactSystem(ctypes.Structure):
    _fields_ = [
        ("rows", c_void_p),
        ("row_count", c_uint64),
        ("bodies", c_void_p),
        ("body_count", c_uint64),
        ("dt", c_float),
        ("growth", GrowthLoadResponse),
    ]


class ContactSolveParameters(ctypes.Structure):
    _fields_ = [("tolerance", c_float), ("max_iterations", c_uint32)]


class ContactSolveReport(ctypes.Structure):
    _fields_ = [("status", c_uint32), ("iterations", c_uint32), ("residual", c_float)]


class ContactDynamicsParameters(ctypes.Structure):
    _fields_ = [
        ("drag", c_float),
        ("contact_stiffness", c_float),
        ("wall_stiffness", c_float),
        ("overlap_tolerance", c_float),
        ("candidate_margin", c_float),
        ("max_overlap_recovery", c_float),
        ("max_growth_fraction", c_float),
        ("max_iterations", c_uint32),
        ("max_refinements", c_uint32),
        ("max_step_halvings", c_uint32),
        ("flow_drift", c_uint32),
        ("growth", GrowthLoadResponse),
    ]


class ContactDynamicsReport(ctypes.Structure):
    _fields_ = [
        ("substeps", c_uint32),
        ("halvings", c_uint32),
        ("refinements", c_uint32),
        ("reserved", c_uint32),
        ("iterations", c_uint64),
        ("max_rows", c_uint64),
        ("max_overlap", c_float),
        ("reserved2", c_uint32),
    ]


class ContactDynamicsOutputs(ctypes.Structure):
    _fields_ = [
        ("center_velocities", c_void_p),
        ("axial_loads", c_void_p),
        ("length_increments", c_void_p),
    ]


class FlowField(ctypes.Structure):
    _fields_ = [
        ("shape_x", c_uint32),
        ("shape_y", c_uint32),
        ("shape_z", c_uint32),
        ("reserved", c_uint32),
        ("origin", Vec3),
        ("spacing", Vec3),
        ("x_faces", c_void_p),
        ("y_faces", c_void_p),
        ("z_faces", c_void_p),
        ("obstacles", c_void_p),
    ]


class ContactGraphIndex(ctypes.Structure):
    _fields_ = [
        ("incidence_offsets", c_void_p),
        ("incidence_contacts", c_void_p),
        ("neighbor_offsets", c_void_p),
        ("neighbor_ids", c_void_p),
        ("neighbor_capacity", c_uint64),
        ("neighbor_count", c_uint64),
    ]


class ColonyParameters(ctypes.Structure):
    _fields_ = [("drag", c_float), ("contact_stiffness", c_float)]


# numpy views of the record types, for bulk conversion.
COLONY_REPORT_DTYPE = np.dtype([("iterations", "<u8"), ("max_overlap", "<f4"), ("rows", "<u4"), ("cells", "<u4"),
                                ("status", "<u4")])

CELL_CONTACT_DTYPE = np.dtype(
    [
        ("first_id", "<u8"),
        ("second_id", "<u8"),
        ("first_slot", "<u4"),
        ("second_slot", "<u4"),
        ("ordinal", "<u4"),
        ("point_on_first", "<f4", 3),
        ("normal", "<f4", 3),
        ("signed_separation", "<f4"),
        ("weight", "<f4"),
        ("reserved", "<u4"),
    ]
)
EXTERNAL_CONTACT_DTYPE = np.dtype(
    [
        ("cell_id", "<u8"),
        ("constraint_id", "<u8"),
        ("cell_slot", "<u4"),
        ("constraint_kind", "<u4"),
        ("location", "<u4"),
        ("point_on_cell", "<f4", 3),
        ("normal", "<f4", 3),
        ("signed_separation", "<f4"),
        ("weight", "<f4"),
        ("reserved", "<u4"),
    ]
)
CONTACT_ROW_DTYPE = np.dtype(
    [
        ("first_slot", "<u4"),
        ("second_slot", "<u4"),
        ("first_jacobian", "<f4", 6),
        ("second_jacobian", "<f4", 6),
        ("first_length_lever", "<f4"),
        ("second_length_lever", "<f4"),
        ("offset", "<f4"),
        ("compliance", "<f4"),
    ]
)
CONTACT_BODY_DTYPE = np.dtype(
    [
        ("axis", "<f4", 3),
        ("translational_mobility", "<f4"),
        ("transverse_mobility", "<f4"),
        ("axial_mobility", "<f4"),
        ("length_rate", "<f4"),
        ("drift", "<f4", 6),
    ]
)
CONSTRAINT_DTYPE = np.dtype(
    [
        ("id", "<u8"),
        ("kind", "<u4"),
        ("allowed_region", "<u4"),
        ("a", "<f4", 3),
        ("b", "<f4", 3),
        ("radius", "<f4"),
        ("half_height", "<f4"),
        ("coefficient", "<f4"),
        ("reserved", "<u4"),
    ]
)

assert CELL_CONTACT_DTYPE.itemsize == ctypes.sizeof(CellContact) == 64
assert EXTERNAL_CONTACT_DTYPE.itemsize == ctypes.sizeof(ExternalContact)
assert CONTACT_ROW_DTYPE.itemsize == ctypes.sizeof(ContactRow) == 72
assert CONTACT_BODY_DTYPE.itemsize == ctypes.sizeof(ContactBody) == 52
assert CONSTRAINT_DTYPE.itemsize == ctypes.sizeof(Constraint)


def ptr(array) -> int | None:
    """Address of a numpy array's data (or a torch tensor's), None for None."""
    if array is None:
        return None
    if hasattr(array, "data_ptr"):
        return array.data_ptr()
    return array.ctypes.data


# The entry points of include/msb200.h and their ctypes signatures.
SIGNATURES = {
    "msb_device_count": (c_size_t, []),
    "msb_context_create": (c_int, [c_uint32, POINTER(c_void_p)]),
    "msb_context_destroy": (None, [c_void_p]),
    "msb_last_error": (c_char_p, [c_void_p]),
    "msb_backend_info": (c_int, [c_void_p, c_char_p, c_size_t]),
    "msb_find_cell_contacts": (
        c_int,
        [c_void_p, POINTER(CellArrays), POINTER(ContactParameters), c_void_p, c_uint64, POINTER(c_uint64)],
    ),
    "msb_set_relaxation": (c_int, [c_void_p, c_uint32]),
    "msb_find_cell_contact_graph": (
        c_int,
        [c_void_p, POINTER(CellArrays), POINTER(ContactParameters), c_void_p, c_uint64, POINTER(c_uint64),
         c_void_p],
    ),
    "msb_build_contact_graph": (c_int, [c_void_p, c_void_p, c_uint64, c_uint64, c_uint32, c_void_p]),
    "msb_find_external_contact_graph": (
        c_int,
        [c_void_p, POINTER(CellArrays), c_void_p, c_uint64, POINTER(ConstraintContactParameters), c_uint32,
         c_void_p, c_uint64, POINTER(c_uint64), c_void_p, c_void_p],
    ),
    "msb_build_external_contact_graph": (
        c_int, [c_void_p, c_void_p, c_uint64, c_uint64, c_uint32, c_void_p, c_void_p]),
    "msb_find_external_contacts": (
        c_int,
        [
            c_void_p,
            POINTER(CellArrays),
            c_void_p,
            c_uint64,
            POINTER(ConstraintContactParameters),
            c_uint32,
            c_void_p,
            c_uint64,
            POINTER(c_uint64),
        ],
    ),
    "msb_solve_contact_forces": (
        c_int,
        [
            c_void_p,
            POINTER(ContactSystem),
            c_void_p,
            POINTER(ContactSolveParameters),
            c_void_p,
            POINTER(ContactSolveReport),
        ],
    ),
    "msb_evaluate_contact_response": (
        c_int,
        [c_void_p, POINTER(ContactSystem), c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "msb_evaluate_contact_gaps": (c_int, [c_void_p, POINTER(ContactSystem), c_void_p, c_void_p]),
    "msb_contact_system_diagonal_bound": (c_int, [c_void_p, POINTER(ContactSystem), POINTER(c_float)]),
    "msb_advance_contact_dynamics": (
        c_int,
        [
            c_void_p,
            POINTER(CellArrays),
            c_void_p,
            c_uint64,
            c_float,
            POINTER(ContactDynamicsParameters),
            POINTER(ContactParameters),
            POINTER(ConstraintContactParameters),
            POINTER(ContactDynamicsReport),
            POINTER(ContactDynamicsOutputs),
        ],
    ),
    "msb_advance_contact_dynamics_device": (
        c_int,
        [
            c_void_p,
            POINTER(CellArrays),
            c_void_p,
            c_uint64,
            c_float,
            POINTER(ContactDynamicsParameters),
            POINTER(ContactParameters),
            POINTER(ConstraintContactParameters),
            POINTER(ContactDynamicsReport),
            POINTER(ContactDynamicsOutputs),
        ],
    ),
    "msb_launch_count": (c_uint64, [c_void_p]),
    "msb_last_step_phases": (c_int, [c_void_p, c_void_p, c_uint32]),
    "msb_set_warm_start": (c_int, [c_void_p, c_uint32]),
    "msb_set_flow_field": (c_int, [c_void_p, c_void_p]),
    "msb_advance_contact_dynamics_batch": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_float, c_void_p,
                                                   c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "msb_tune_batch": (c_int, [c_void_p]),
    "msb_batch_tuning": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "msb_cell_features": (c_int, [c_void_p, c_void_p, c_void_p]),
    "msb_mlp_activation_bytes": (c_uint64, [c_uint64]),
    "msb_mlp_backward_scratch_bytes": (c_uint64, [c_uint64]),
    "msb_mlp_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_void_p, c_void_p, c_void_p]),
    "msb_mlp_backward": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "msb_mlp_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint32, c_float, c_float, c_float, c_float,
                             c_void_p, c_void_p, c_void_p]),
    "msb_set_warm_start_network": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "msb_set_motion_guess": (c_int, [c_void_p, c_void_p, c_uint64, c_float]),
    "msb_last_step_solves": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p]),
    "msb_last_step_searches": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "msb_set_search_reuse": (c_int, [c_void_p, c_uint32]),
    "msb_solve_contact_forces_no_alloc": (
        c_int,
        [
            POINTER(ContactSystem),
            c_void_p,
            POINTER(ContactSolveParameters),
            c_void_p,
            POINTER(ContactSolveReport),
            c_void_p,
        ],
    ),
    "msb_profile_iterations": (
        c_int,
        [c_void_p, c_uint32, POINTER(c_float), POINTER(c_float), POINTER(c_uint64), POINTER(c_uint64)],
    ),
}

_library = None


def load_library(path: str | os.PathLike | None = None):
    """Load libmsb200.so (built in-tree by ``__graft_entry__.build()``).

    Raises FileNotFoundError when the library has not been built: the CUDA
    path is the only path.
    """
    global _library
    if _library is not None and path is None:
        return _library
    target = Path(path) if path is not None else LIBRARY_PATH
    if not target.exists():
        raise FileNotFoundError(
            f"{target} is missing: build the CUDA extension with __graft_entry__.build()"
        )
    library = ctypes.CDLL(str(target))
    for name, (restype, argtypes) in SIGNATURES.items():
        function = getattr(library, name)
        function.restype = restype
        function.argtypes = argtypes
    if path is None:
        _library = library
    return library


class NativeError(RuntimeError):
    """A failure reported by the native library, with its status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def raise_for_status(status: int, message: str) -> None:
    """Map a C-ABI status to the exception the reference would raise."""
    if status == OK:
        return
    if status == ERR_INVALID_ARGUMENT:
        raise ValueError(message)
    if status == ERR_OVERFLOW:
        raise OverflowError(message)
    raise NativeError(status, message)
