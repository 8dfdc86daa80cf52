"""A profiling case for the BB iteration kernels.

Relaxes a jammed colony for a few contact-dynamics steps, then times extra
projected iterations of the last solved system with the timing hook
(msb_profile_iterations), whose launches carry their own kernel instance
names (``body_pass_kernel<1>`` / ``row_pass_kernel<1>``) so that a profiler
can select them apart from the solve graph's launches:

  python -m microsimulator_b200.profile_case --cells 500000 --steps 2 --iterations 3
"""

from __future__ import annotations

import argparse
import json


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--cells", type=int, default=500_000)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--iterations", type=int, default=3)
    p.add_argument("--seed", type=int, default=42)
    args = p.parse_args()

    from . import workloads
    from .backend import B200Backend
    from .types import ContactDynamicsParameters

    backend = B200Backend(0)
    world = workloads.jammed(n=args.cells, seed=args.seed)
    dyn = ContactDynamicsParameters(overlap_tolerance=5e-4)
    reports = []
    for step in range(args.steps):
        plan = workloads.plan_divisions(world, 0.02, seed=args.seed * 100003 + step)
        world.divide_many(plan.parents, 0.5, plan.rotations)
        result = backend.advance_contact_dynamics(world, None, 0.02, dyn)
        world.next_id = int(world.ids.max()) + 1
        reports.append(result.report.iterations)
    timing = backend.profile_iterations(args.iterations)
    timing["algorithmic_bytes"] = timing["rows"] * 96 + timing["bodies"] * 128
    timing["iterations_per_step"] = reports
    print(json.dumps(timing))
    backend.close()


if __name__ == "__main__":
    main()
