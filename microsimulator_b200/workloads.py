"""Seeded synthetic colonies of the contact workloads.

All draws use numpy's PCG64 with the stated seed, so every path (the CUDA
backend, the reference CPU backend, the oracle) starts from the same bits.
Capsules lie in the xy plane at z = 0 with radius 0.5 um, as the reference's
planar colonies do.  Where a workload names a cell count and an area fraction
whose stated box cannot hold them, the box is derived from the count and the
fraction: side = sqrt(N * mean capsule area / fraction).

  colony_1k     1,000 capsules, lengths U[2, 4] um, 40 x 40 um box (overlapping)
  trap_colony   capsules at area fraction 0.7 in a trap with wall boxes
  jammed        N capsules (1,000,000 by default), lengths log-normal
                (mu = ln 3 um, sigma 0.2), area fraction 0.85, open domain
  sweep         colonies of log-uniform size for the batched sweep
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .world import ConstraintSet, WorldState

RADIUS = 0.5


def mean_capsule_area(mean_length: float, radius: float = RADIUS) -> float:
    return math.pi * radius * radius + 2.0 * radius * mean_length


def _planar(rng, n, low, high, lengths, growth_rate):
    positions = np.zeros((n, 3), dtype=np.float64)
    positions[:, 0] = rng.uniform(low[0], high[0], n)
    positions[:, 1] = rng.uniform(low[1], high[1], n)
    theta = rng.uniform(0.0, math.pi, n)
    directions = np.stack([np.cos(theta), np.sin(theta), np.zeros(n)], axis=1)
    return WorldState.from_arrays(positions, directions, lengths, RADIUS, growth_rates=growth_rate)


def colony_1k(seed: int = 42, n: int = 1000, side: float = 40.0, growth_rate: float = 0.0) -> WorldState:
    """1,000 capsules, lengths U[2, 4] um, centres uniform in a 40 x 40 um box."""
    rng = np.random.default_rng(seed)
    lengths = rng.uniform(2.0, 4.0, n)
    return _planar(rng, n, (0.0, 0.0), (side, side), lengths, growth_rate)


def jammed(n: int = 1_000_000, area_fraction: float = 0.85, seed: int = 42, growth_rate: float = 0.5) -> WorldState:
    """N capsules near jamming in an open square domain derived from N and the
    area fraction; lengths log-normal (mu = ln 3 um, sigma = 0.2)."""
    rng = np.random.default_rng(seed)
    lengths = np.exp(rng.normal(math.log(3.0), 0.2, n))
    side = math.sqrt(n * mean_capsule_area(float(np.mean(lengths))) / area_fraction)
    return _planar(rng, n, (0.0, 0.0), (side, side), lengths, growth_rate)


def sweep_colony(n: int, seed: int = 42, area_fraction: float = 0.7, growth_rate: float = 0.5) -> WorldState:
    """One colony of a parameter sweep: N capsules with the shapes of the
    trap workload (radius 0.5 um, lengths U[2, 4] um) packed at the area
    fraction in an open square domain."""
    rng = np.random.default_rng(seed)
    lengths = rng.uniform(2.0, 4.0, n)
    side = math.sqrt(n * mean_capsule_area(float(np.mean(lengths))) / area_fraction)
    return _planar(rng, n, (0.0, 0.0), (side, side), lengths, growth_rate)


def jammed_side(n: int, area_fraction: float = 0.85) -> float:
    return math.sqrt(n * mean_capsule_area(3.0 * math.exp(0.02)) / area_fraction)


def trap_colony(n: int = 100_000, area_fraction: float = 0.7, seed: int = 42,
                growth_rate: float = 0.5) -> tuple[WorldState, ConstraintSet]:
    """Capsules packed at the area fraction in a trap opening onto a channel,
    with the wall boxes of the reference's TrapChannelDevice recipe
    (python/src/microsimulator/microfluidics.py:285-340).  The trap keeps the
    stated 100 x 40 um aspect and is scaled so that it holds N capsules at
    the fraction; the channel scales with it."""
    rng = np.random.default_rng(seed)
    lengths = rng.uniform(2.0, 4.0, n)
    area = n * mean_capsule_area(float(np.mean(lengths))) / area_fraction
    scale = math.sqrt(area / (100.0 * 40.0))
    trap_depth, trap_half_y = 100.0 * scale, 20.0 * scale
    channel_width, channel_half_length = 100.0 * scale, 300.0 * scale
    wall, half_z = 2.0, 3.0
    # The trap spans x in [0, depth], y in [-half_y, half_y]; the channel
    # runs along y at x in [-channel_width, 0].
    constraints = ConstraintSet()
    top = half_z + wall
    blocks = (
        ((0.0, trap_half_y, -top), (trap_depth + wall, channel_half_length, top)),
        ((0.0, -channel_half_length, -top), (trap_depth + wall, -trap_half_y, top)),
        ((trap_depth, -trap_half_y - wall, -top), (trap_depth + wall, trap_half_y + wall, top)),
    )
    for low, high in blocks:
        center = tuple((l + h) * 0.5 for l, h in zip(low, high))
        half = tuple((h - l) * 0.5 for l, h in zip(low, high))
        constraints.add_box(center=center, half_extents=half, allowed_region=0)
    constraints.add_box(
        center=((trap_depth + wall - channel_width) * 0.5, 0.0, 0.0),
        half_extents=((trap_depth + wall + channel_width) * 0.5, channel_half_length, half_z),
        allowed_region=1,
    )
    margin = 2.5
    world = _planar(rng, n, (margin, -trap_half_y + margin), (trap_depth - margin, trap_half_y - margin), lengths,
                    growth_rate)
    return world, constraints


@dataclass
class Divisions:
    parents: np.ndarray  # ids
    rotations: np.ndarray  # (k, 4) cos, sin of each daughter's turn


def plan_divisions(world: WorldState, fraction: float, seed: int, jitter: float = 0.02,
                   minimum_length: float | None = None) -> Divisions:
    """Picks round(fraction * N) parents at random among cells long enough to
    divide, and a turn of each daughter uniform in (-jitter, jitter)."""
    rng = np.random.default_rng(seed)
    long_enough = minimum_length if minimum_length is not None else 2.0 * RADIUS
    eligible = np.flatnonzero(world.lengths >= long_enough)
    k = min(len(eligible), int(round(fraction * len(world))))
    chosen = np.sort(rng.choice(eligible, size=k, replace=False)) if k > 0 else np.zeros(0, dtype=np.int64)
    angles = rng.uniform(-jitter, jitter, (k, 2))
    rotations = np.zeros((k, 4), dtype=np.float32)
    rotations[:, 0] = np.cos(angles[:, 0]).astype(np.float32)
    rotations[:, 1] = np.sin(angles[:, 0]).astype(np.float32)
    rotations[:, 2] = np.cos(angles[:, 1]).astype(np.float32)
    rotations[:, 3] = np.sin(angles[:, 1]).astype(np.float32)
    return Divisions(world.ids[chosen].copy(), rotations)


def sweep_sizes(count: int = 256, low: int = 500, high: int = 50_000, seed: int = 42):
    """Colony sizes log-uniform in [low, high] with per-colony contact
    stiffness and drag uniform in [0.5, 2]."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(low), math.log(high), count)).astype(np.int64)
    stiffness = rng.uniform(0.5, 2.0, count)
    drag = rng.uniform(0.5, 2.0, count)
    return sizes, stiffness, drag
