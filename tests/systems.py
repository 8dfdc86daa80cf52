"""Random contact systems for the parity tests: pair and constraint rows
mixed, signed-zero offsets and multipliers, zero jacobians and levers, fixed
bodies, drift, and the three growth-load laws."""

import numpy as np

from microsimulator_b200 import abi
from microsimulator_b200.types import ContactSystem, GrowthLoadResponse

LAWS = [
    GrowthLoadResponse(0, 0.0, 0.0, 1.0),
    GrowthLoadResponse(1, 0.4, 0.0, 1.0),
    GrowthLoadResponse(2, 0.0, 0.2, 3.0),
]


def mixed_system(seed: int, bodies: int, rows: int, law: GrowthLoadResponse, walls: float = 0.3) -> ContactSystem:
    rng = np.random.default_rng(seed)
    r = np.zeros(rows, dtype=abi.CONTACT_ROW_DTYPE)
    first = rng.integers(0, bodies, rows)
    second = (first + rng.integers(1, bodies, rows)) % bodies
    wall = rng.random(rows) < walls
    r["first_slot"] = first
    r["second_slot"] = np.where(wall, abi.INVALID_SLOT, second)
    r["first_jacobian"] = rng.normal(0.0, 1.0, (rows, 6)).astype(np.float32)
    r["second_jacobian"] = np.where(wall[:, None], 0.0, rng.normal(0.0, 1.0, (rows, 6))).astype(np.float32)
    r["first_length_lever"] = rng.uniform(0.0, 0.5, rows).astype(np.float32)
    r["second_length_lever"] = np.where(wall, 0.0, rng.uniform(0.0, 0.5, rows)).astype(np.float32)
    r["offset"] = rng.normal(0.0, 0.05, rows).astype(np.float32)
    r["compliance"] = rng.uniform(0.0, 0.2, rows).astype(np.float32)
    # Edge values: signed-zero offsets, rows with zero compliance, a zero
    # first jacobian and lever (the first side term is then +0.0f).
    r["offset"][::7] = np.float32(-0.0)
    r["offset"][3::7] = np.float32(0.0)
    r["compliance"][::5] = 0.0
    r["first_jacobian"][::11] = 0.0
    r["first_length_lever"][::11] = 0.0
    b = np.zeros(bodies, dtype=abi.CONTACT_BODY_DTYPE)
    axis = rng.normal(0.0, 1.0, (bodies, 3))
    b["axis"] = (axis / np.linalg.norm(axis, axis=1, keepdims=True)).astype(np.float32)
    b["translational_mobility"] = rng.uniform(0.2, 1.0, bodies).astype(np.float32)
    b["transverse_mobility"] = rng.uniform(0.1, 2.0, bodies).astype(np.float32)
    b["axial_mobility"] = rng.uniform(0.1, 2.0, bodies).astype(np.float32)
    b["length_rate"] = rng.choice(np.array([0.0, 0.5, 1.5, -0.25], np.float32), bodies)
    fixed = rng.random(bodies) < 0.05
    for name in ("translational_mobility", "transverse_mobility", "axial_mobility"):
        b[name][fixed] = 0.0
    b["drift"] = np.where(rng.random((bodies, 1)) < 0.3, rng.normal(0.0, 0.1, (bodies, 6)), 0.0).astype(np.float32)
    return ContactSystem(r, b, 0.02, law)


def multipliers_for(system: ContactSystem, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    m = rng.uniform(0.0, 2.0, len(system.rows)).astype(np.float32)
    m[::3] = 0.0
    m[1::9] = np.float32(-0.0)
    return m


def bits(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
