"""Profiling cases.

--case bb (default): relaxes a jammed colony for a few contact-dynamics
steps, then times extra projected iterations of the last solved system with
the timing hook (msb_profile_iterations), whose launches carry their own
kernel instance names (``body_pass_kernel<1>`` / ``row_pass_kernel<1>``) so
that a profiler can select them apart from the solve graph's launches:

  python -m microsimulator_b200.profile_case --cells 500000 --steps 2 --iterations 3

--case mlp: the warm-start network's features and forward pass over a jammed
colony (``features_kernel``, ``forward_kernel``), timed with CUDA events:

  python -m microsimulator_b200.profile_case --case mlp --cells 1000000

--case batch: one step of a batch of sweep colonies (``batch_solve_kernel``;
the first call's autotuner launches the kernel once per launch shape first):

  python -m microsimulator_b200.profile_case --case batch --colonies 64
"""

from __future__ import annotations

import argparse
import json


def mlp_case(args) -> None:
    import torch

    from . import learned, workloads
    from .backend import B200Backend, DeviceCells

    backend = B200Backend(0)
    world = workloads.jammed(n=args.cells, seed=args.seed)
    cells = DeviceCells(world)
    net = learned.WarmStartNetwork("cuda:0", seed=args.seed, library=backend._lib)
    times = {"features_ms": [], "forward_ms": []}
    for _ in range(args.iterations):
        s0, s1, s2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        s0.record()
        x = learned.cell_features(backend, cells)
        s1.record()
        net.forward(x)
        s2.record()
        torch.cuda.synchronize()
        times["features_ms"].append(s0.elapsed_time(s1))
        times["forward_ms"].append(s1.elapsed_time(s2))
    flops = 2.0 * args.cells * (96 * 128 + 2 * 128 * 128 + 8 * 128)
    best = min(times["forward_ms"])
    print(json.dumps({**times, "cells": args.cells, "forward_flops": flops,
                      "forward_tflops": flops / (best * 1e-3) / 1e12}))
    backend.close()


def batch_case(args) -> None:
    import torch

    from . import sweep
    from .backend import B200Backend
    from .types import ContactDynamicsParameters

    backend = B200Backend(0)
    batch = sweep.sweep_batch(count=args.colonies, seed=args.seed)
    dyn = ContactDynamicsParameters(overlap_tolerance=5e-4)
    for k in range(args.steps):
        batch.divide(0.02, seed=k)
        report, colonies = batch.step(backend, 0.02, dyn)
    torch.cuda.synchronize()
    print(json.dumps({"cells": int(batch.counts().sum()), "iterations": int(colonies["iterations"].sum()),
                      "tuning": backend.batch_tuning(), "solves": backend.last_step_solves()["iterations"].tolist()}))
    backend.close()


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--case", default="bb", choices=["bb", "mlp", "batch"])
    p.add_argument("--colonies", type=int, default=64)
    p.add_argument("--cells", type=int, default=500_000)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--iterations", type=int, default=3)
    p.add_argument("--seed", type=int, default=42)
    args = p.parse_args()
    if args.case == "mlp":
        mlp_case(args)
        return
    if args.case == "batch":
        batch_case(args)
        return

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
