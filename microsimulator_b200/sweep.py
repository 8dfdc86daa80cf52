"""Parameter sweeps: many independent colonies stepped together through
msb_advance_contact_dynamics_batch, each with its own drag and contact
stiffness and its own convergence (one persistent launch of the batched
solve per solve of the step).

A ``ColonyBatch`` keeps one WorldState per colony (divisions append
daughters to their own colony) and lays the colonies out colony after colony
for each step, with ids made unique across the batch by the colony's index
in their top bits.
"""

from __future__ import annotations

import numpy as np

from . import workloads
from .types import ContactDynamicsParameters
from .world import WorldState

ID_SHIFT = 40


def concatenate(worlds) -> WorldState:
    """The colonies' cells colony after colony, ids tagged by colony."""
    out = WorldState()
    for name in (*WorldState.FIELDS, "fixed"):
        setattr(out, name, np.concatenate([getattr(w, name) for w in worlds]))
    tagged = []
    for k, w in enumerate(worlds):
        if len(w) and int(w.ids.max()) >= (1 << ID_SHIFT):
            raise ValueError("colony ids must stay below 2**40")
        tagged.append(w.ids + np.uint64(k << ID_SHIFT))
    out.ids = np.concatenate(tagged).astype(np.uint64)
    out.next_id = int(out.ids.max()) + 1 if len(out.ids) else 1
    return out


def split_into(batch: WorldState, worlds) -> None:
    """Copies the stepped geometry of a concatenated batch back into its colonies."""
    at = 0
    for w in worlds:
        n = len(w)
        for name in ("position_x", "position_y", "position_z", "direction_x", "direction_y", "direction_z",
                     "lengths"):
            setattr(w, name, getattr(batch, name)[at:at + n].copy())
        at += n


class ColonyBatch:
    def __init__(self, worlds, drag, stiffness):
        self.worlds = list(worlds)
        self.drag = np.asarray(drag, dtype=np.float32)
        self.stiffness = np.asarray(stiffness, dtype=np.float32)
        if len(self.drag) != len(self.worlds) or len(self.stiffness) != len(self.worlds):
            raise ValueError("one drag and one stiffness per colony")

    def __len__(self) -> int:
        return len(self.worlds)

    def cells(self) -> int:
        return sum(len(w) for w in self.worlds)

    def counts(self) -> np.ndarray:
        return np.array([len(w) for w in self.worlds], dtype=np.uint32)

    def concatenated(self) -> WorldState:
        return concatenate(self.worlds)

    def step(self, backend, dt: float, dynamics: ContactDynamicsParameters | None = None):
        """One step of every colony with host buffers; returns the batch report
        and the per-colony reports."""
        batch = self.concatenated()
        report, colonies = backend.advance_contact_dynamics_batch(batch, self.counts(), self.drag, self.stiffness, dt,
                                                                  dynamics)
        split_into(batch, self.worlds)
        for w in self.worlds:
            if len(w):
                w.next_id = int(w.ids.max()) + 1
        return report, colonies

    def divide(self, fraction: float, seed: int) -> None:
        """Divides `fraction` of each colony's cells (daughters turned by
        +-0.02 rad), as the workloads' division plan does."""
        for k, w in enumerate(self.worlds):
            plan = workloads.plan_divisions(w, fraction, seed=seed * 7919 + k)
            w.divide_many(plan.parents, 0.5, plan.rotations)


def sweep_batch(count: int = 256, low: int = 500, high: int = 50_000, seed: int = 42) -> ColonyBatch:
    """The sweep workload: `count` colonies with log-uniform sizes in
    [low, high]; contact stiffness and drag each the default's value times a
    factor uniform in [0.5, 2]; capsule shapes of the trap workload packed at
    area fraction 0.7."""
    sizes, stiffness, drag = workloads.sweep_sizes(count, low, high, seed)
    defaults = ContactDynamicsParameters()
    worlds = [workloads.sweep_colony(int(n), seed=seed * 1000 + k) for k, n in enumerate(sizes)]
    return ColonyBatch(worlds, defaults.drag * drag, defaults.contact_stiffness * stiffness)
