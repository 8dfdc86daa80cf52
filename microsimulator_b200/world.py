"""Host-side cell and constraint containers for the contact path.

``WorldState`` keeps the cells as structure-of-arrays numpy buffers by slot,
with the reference WorldState's identity and division rules
(cpp/core/world_state.cpp:176-276, 405-430): stable increasing ids, a divided
parent's slot taken by its first daughter and the second daughter appended,
directions stored normalized.  All arithmetic is FP32, in the reference's
operation order, so that a world built here holds the same bits as one built
by the reference.  ``ConstraintSet`` mirrors cpp/core/constraints.cpp: ids are
allocated in insertion order across kinds.
"""

from __future__ import annotations

import numpy as np

from . import abi

f32 = np.float32


def normalized(x, y, z):
    """``normalized`` of types.hpp:58-64 in FP32: v * (1 / |v|)."""
    x, y, z = f32(x), f32(y), f32(z)
    magnitude = np.sqrt(f32(f32(x * x) + f32(y * y)) + f32(z * z), dtype=f32)
    if not np.isfinite(magnitude) or magnitude <= 0:
        raise ValueError("cell direction must be finite and non-zero")
    scale = f32(f32(1.0) / magnitude)
    return f32(x * scale), f32(y * scale), f32(z * scale)


def normalized_arrays(x, y, z):
    """Vectorized ``normalized`` over FP32 arrays."""
    x = np.asarray(x, dtype=f32)
    y = np.asarray(y, dtype=f32)
    z = np.asarray(z, dtype=f32)
    magnitude = np.sqrt((x * x + y * y) + z * z).astype(f32)
    if not np.all(np.isfinite(magnitude)) or np.any(magnitude <= 0):
        raise ValueError("cell direction must be finite and non-zero")
    scale = (f32(1.0) / magnitude).astype(f32)
    return x * scale, y * scale, z * scale


class WorldState:
    FIELDS = (
        "position_x",
        "position_y",
        "position_z",
        "direction_x",
        "direction_y",
        "direction_z",
        "lengths",
        "radii",
        "growth_rates",
    )

    def __init__(self, capacity: int = 0):
        self.ids = np.zeros(0, dtype=np.uint64)
        for name in self.FIELDS:
            setattr(self, name, np.zeros(0, dtype=f32))
        self.fixed = np.zeros(0, dtype=np.uint8)
        self.next_id = 1
        self._slot_of: dict[int, int] = {}

    # -- construction ---------------------------------------------------
    @classmethod
    def from_arrays(
        cls,
        positions,
        directions,
        lengths,
        radii,
        growth_rates=None,
        fixed=None,
        ids=None,
    ) -> "WorldState":
        """Cells from (n, 3) positions and directions; directions are
        normalized as WorldState::append does."""
        world = cls()
        positions = np.asarray(positions, dtype=f32).reshape(-1, 3)
        directions = np.asarray(directions, dtype=f32).reshape(-1, 3)
        n = positions.shape[0]
        dx, dy, dz = normalized_arrays(directions[:, 0], directions[:, 1], directions[:, 2])
        world.position_x = np.array(positions[:, 0])
        world.position_y = np.array(positions[:, 1])
        world.position_z = np.array(positions[:, 2])
        world.direction_x, world.direction_y, world.direction_z = dx.copy(), dy.copy(), dz.copy()
        world.lengths = np.array(np.broadcast_to(np.asarray(lengths, dtype=f32), (n,)))
        world.radii = np.array(np.broadcast_to(np.asarray(radii, dtype=f32), (n,)))
        rates = 1.0 if growth_rates is None else growth_rates
        world.growth_rates = np.array(np.broadcast_to(np.asarray(rates, dtype=f32), (n,)))
        fixed = 0 if fixed is None else fixed
        world.fixed = np.array(np.broadcast_to(np.asarray(fixed, dtype=np.uint8), (n,)))
        if ids is None:
            world.ids = np.arange(1, n + 1, dtype=np.uint64)
        else:
            world.ids = np.ascontiguousarray(np.asarray(ids, dtype=np.uint64))
        world.next_id = int(world.ids.max()) + 1 if n else 1
        world._slot_of = {}
        if np.any(world.lengths < 0) or np.any(world.radii <= 0):
            raise ValueError("cell length must be non-negative and radius positive")
        return world

    def __len__(self) -> int:
        return int(self.ids.shape[0])

    @property
    def size(self) -> int:
        return len(self)

    def slot_of(self, cell_id: int) -> int:
        if len(self._slot_of) != len(self):
            self._slot_of = {int(i): s for s, i in enumerate(self.ids.tolist())}
        try:
            return self._slot_of[int(cell_id)]
        except KeyError:
            raise KeyError(f"unknown cell id {cell_id}") from None

    def add_cell(
        self,
        position=(0.0, 0.0, 0.0),
        direction=(1.0, 0.0, 0.0),
        length=3.5,
        radius=0.5,
        growth_rate=1.0,
        fixed=False,
    ) -> int:
        """WorldState::add_cell with CellInit's defaults (world_state.hpp:15-24)."""
        if length < 0 or radius <= 0:
            raise ValueError("cell length must be non-negative and radius positive")
        dx, dy, dz = normalized(*direction)
        cell_id = self.next_id
        self.next_id += 1
        self._append(cell_id, position, (dx, dy, dz), length, radius, growth_rate, fixed)
        return cell_id

    def _append(self, cell_id, position, direction, length, radius, growth_rate, fixed):
        self.ids = np.append(self.ids, np.uint64(cell_id))
        values = (*position, *direction, length, radius, growth_rate)
        for name, value in zip(self.FIELDS, values):
            setattr(self, name, np.append(getattr(self, name), f32(value)))
        self.fixed = np.append(self.fixed, np.uint8(1 if fixed else 0))
        self._slot_of[int(cell_id)] = len(self) - 1

    def set_cell_geometry(self, slot: int, position, direction, length) -> None:
        """WorldState::set_cell_geometry: stores the normalized direction."""
        dx, dy, dz = normalized(*direction)
        self.position_x[slot], self.position_y[slot], self.position_z[slot] = (f32(v) for v in position)
        self.direction_x[slot], self.direction_y[slot], self.direction_z[slot] = dx, dy, dz
        self.lengths[slot] = f32(length)

    def set_cell_fixed(self, cell_id: int, fixed: bool) -> None:
        self.fixed[self.slot_of(cell_id)] = 1 if fixed else 0

    def divide(self, parent_id: int, first_fraction: float = 0.5) -> tuple[int, int]:
        """WorldState::divide (world_state.cpp:238-276) in FP32."""
        self.divide_many(np.array([parent_id], dtype=np.uint64), first_fraction)
        return self.next_id - 2, self.next_id - 1

    def divide_many(self, parent_ids, first_fraction: float = 0.5, rotations=None) -> None:
        """Divides each parent in turn, as repeated WorldState::divide calls
        do, then turns each daughter in the xy plane by the (cos, sin) pairs in
        ``rotations`` (shape (k, 4): first daughter's cos, sin, second's)."""
        parent_ids = np.asarray(parent_ids, dtype=np.uint64)
        k = parent_ids.shape[0]
        if k == 0:
            return
        if len(np.unique(parent_ids)) != k:
            raise ValueError("a parent is listed twice")
        fraction = f32(first_fraction)
        if not (0 < fraction < 1):
            raise ValueError("first daughter fraction must be between zero and one")
        order = np.argsort(self.ids, kind="stable")
        where = np.searchsorted(self.ids[order], parent_ids)
        if np.any(where >= len(self)) or np.any(self.ids[order[np.minimum(where, len(self) - 1)]] != parent_ids):
            raise KeyError("unknown parent id")
        slots = order[where].astype(np.int64)
        length = self.lengths[slots]
        radius = self.radii[slots]
        available = (length - (f32(2.0) * radius)).astype(f32)
        if np.any(~(available >= 0)):
            raise ValueError("parent is too short to divide into valid daughters")
        first_length = (available * fraction).astype(f32)
        second_length = (available - first_length).astype(f32)
        px, py, pz = self.position_x[slots], self.position_y[slots], self.position_z[slots]
        dx, dy, dz = self.direction_x[slots], self.direction_y[slots], self.direction_z[slots]
        first_half = ((length - first_length) * f32(0.5)).astype(f32)
        second_half = ((length - second_length) * f32(0.5)).astype(f32)
        # CellInit direction goes through normalized() in append/replace.
        ndx, ndy, ndz = normalized_arrays(dx, dy, dz)
        first_pos = (px - dx * first_half, py - dy * first_half, pz - dz * first_half)
        second_pos = (px + dx * second_half, py + dy * second_half, pz + dz * second_half)
        first_ids = (self.next_id + 2 * np.arange(k)).astype(np.uint64)
        second_ids = first_ids + np.uint64(1)
        self.next_id += 2 * k
        n = len(self)
        # first daughter replaces the parent's slot
        self.ids[slots] = first_ids
        self.position_x[slots], self.position_y[slots], self.position_z[slots] = first_pos
        self.direction_x[slots], self.direction_y[slots], self.direction_z[slots] = ndx, ndy, ndz
        self.lengths[slots] = first_length
        # second daughter appended
        self.ids = np.concatenate([self.ids, second_ids])
        self.position_x = np.concatenate([self.position_x, second_pos[0]])
        self.position_y = np.concatenate([self.position_y, second_pos[1]])
        self.position_z = np.concatenate([self.position_z, second_pos[2]])
        self.direction_x = np.concatenate([self.direction_x, ndx])
        self.direction_y = np.concatenate([self.direction_y, ndy])
        self.direction_z = np.concatenate([self.direction_z, ndz])
        self.lengths = np.concatenate([self.lengths, second_length])
        self.radii = np.concatenate([self.radii, radius])
        self.growth_rates = np.concatenate([self.growth_rates, self.growth_rates[slots]])
        self.fixed = np.concatenate([self.fixed, self.fixed[slots]])
        self._slot_of = {}
        if rotations is not None:
            rotations = np.asarray(rotations, dtype=f32).reshape(k, 4)
            for daughter, where in ((0, slots), (1, n + np.arange(k))):
                c = rotations[:, 2 * daughter]
                s = rotations[:, 2 * daughter + 1]
                ox, oy, oz = self.direction_x[where], self.direction_y[where], self.direction_z[where]
                rx = (ox * c - oy * s).astype(f32)
                ry = (ox * s + oy * c).astype(f32)
                nx, ny, nz = normalized_arrays(rx, ry, oz)
                self.direction_x[where], self.direction_y[where], self.direction_z[where] = nx, ny, nz

    # -- C-ABI view -------------------------------------------------------
    def arrays(self) -> abi.CellArrays:
        """The C-ABI view of this world's buffers (valid while they live)."""
        for name in ("ids", *self.FIELDS, "fixed"):
            value = getattr(self, name)
            if not value.flags.c_contiguous or not value.flags.writeable:
                setattr(self, name, np.ascontiguousarray(value).copy())
        return abi.CellArrays(
            len(self),
            abi.ptr(self.ids),
            abi.ptr(self.position_x),
            abi.ptr(self.position_y),
            abi.ptr(self.position_z),
            abi.ptr(self.direction_x),
            abi.ptr(self.direction_y),
            abi.ptr(self.direction_z),
            abi.ptr(self.lengths),
            abi.ptr(self.radii),
            abi.ptr(self.growth_rates),
            abi.ptr(self.fixed),
        )

    def copy(self) -> "WorldState":
        other = WorldState()
        other.ids = self.ids.copy()
        for name in (*self.FIELDS, "fixed"):
            setattr(other, name, getattr(self, name).copy())
        other.next_id = self.next_id
        return other

    def geometry(self) -> np.ndarray:
        """(n, 7) positions, directions and lengths, for comparisons."""
        return np.stack(
            [
                self.position_x,
                self.position_y,
                self.position_z,
                self.direction_x,
                self.direction_y,
                self.direction_z,
                self.lengths,
            ],
            axis=1,
        )


class ConstraintSet:
    """ConstraintSet (cpp/core/constraints.cpp): planes, spheres, boxes and
    cylinders with ids allocated in insertion order."""

    def __init__(self):
        self.records = np.zeros(0, dtype=abi.CONSTRAINT_DTYPE)
        self.next_id = 1

    def __len__(self) -> int:
        return int(self.records.shape[0])

    def _add(self, kind, region, a, b=(0.0, 0.0, 0.0), radius=0.0, half_height=0.0, coefficient=1.0):
        record = np.zeros(1, dtype=abi.CONSTRAINT_DTYPE)
        record["id"] = self.next_id
        record["kind"] = kind
        record["allowed_region"] = region
        record["a"] = a
        record["b"] = b
        record["radius"] = radius
        record["half_height"] = half_height
        record["coefficient"] = coefficient
        self.records = np.concatenate([self.records, record])
        self.next_id += 1
        return self.next_id - 1

    @staticmethod
    def _finite(*values) -> bool:
        return all(np.isfinite(f32(v)) for v in values)

    @staticmethod
    def _check_coefficient(coefficient) -> None:
        if not np.isfinite(f32(coefficient)) or f32(coefficient) <= 0:
            raise ValueError("constraint coefficient must be finite and positive")

    def add_plane(self, point=(0.0, 0.0, 0.0), inward_normal=(0.0, 1.0, 0.0), coefficient=1.0) -> int:
        """ConstraintSet::add_plane (constraints.cpp:169-186): the inward
        normal is stored normalized, inward_normal * (1 / |inward_normal|) in
        FP32."""
        if not self._finite(*point, *inward_normal):
            raise ValueError("plane fields must be finite")
        x, y, z = (f32(c) for c in inward_normal)
        magnitude = np.sqrt(f32(f32(x * x) + f32(y * y)) + f32(z * z), dtype=f32)
        if not np.isfinite(magnitude) or magnitude <= 0:
            raise ValueError("plane inward normal must be non-zero")
        self._check_coefficient(coefficient)
        scale = f32(f32(1.0) / magnitude)
        normal = (f32(x * scale), f32(y * scale), f32(z * scale))
        return self._add(abi.CONSTRAINT_PLANE, abi.REGION_OUTSIDE, point, normal, coefficient=coefficient)

    def add_sphere(self, center=(0.0, 0.0, 0.0), radius=1.0, coefficient=1.0, allowed_region=abi.REGION_OUTSIDE) -> int:
        """ConstraintSet::add_sphere (constraints.cpp:188-201)."""
        if not self._finite(*center, radius) or f32(radius) <= 0:
            raise ValueError("sphere geometry must be finite with a positive radius")
        self._check_coefficient(coefficient)
        return self._add(abi.CONSTRAINT_SPHERE, allowed_region, center, radius=radius, coefficient=coefficient)

    def add_box(self, center=(0.0, 0.0, 0.0), half_extents=(1.0, 1.0, 1.0), coefficient=1.0, allowed_region=abi.REGION_OUTSIDE) -> int:
        """ConstraintSet::add_box (constraints.cpp:203-216)."""
        if not self._finite(*center, *half_extents) or any(f32(h) <= 0 for h in half_extents):
            raise ValueError("box geometry must be finite with positive half extents")
        self._check_coefficient(coefficient)
        return self._add(abi.CONSTRAINT_BOX, allowed_region, center, half_extents, coefficient=coefficient)

    def add_cylinder(
        self, center=(0.0, 0.0, 0.0), radius=1.0, half_height=1.0, coefficient=1.0, allowed_region=abi.REGION_OUTSIDE
    ) -> int:
        """ConstraintSet::add_cylinder (constraints.cpp:218-234)."""
        if not self._finite(*center, radius, half_height) or f32(radius) <= 0 or f32(half_height) <= 0:
            raise ValueError("cylinder geometry must be finite with a positive radius and half height")
        self._check_coefficient(coefficient)
        return self._add(
            abi.CONSTRAINT_CYLINDER, allowed_region, center, radius=radius, half_height=half_height, coefficient=coefficient
        )

    def pointer(self):
        self.records = np.ascontiguousarray(self.records)
        return abi.ptr(self.records) if len(self) else None
