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

--case train: training steps of the warm-start network (``forward_tc_kernel``
keeping activations, ``gemm_tc_kernel``, ``gemm_reduce_kernel``):

  python -m microsimulator_b200.profile_case --case train --cells 8192 --iterations 5

--case batch: one step of a batch of sweep colonies (``batch_solve_kernel``;
the first call's autotuner launches the kernel once per launch shape first):

  python -m microsimulator_b200.profile_case --case batch --colonies 64

--case guess: the upper bound of any motion-guess warm start.  Each step of a
jammed colony runs plain, then again from the same state with the plain
step's own displacement as the guess (warm-start flag 2) and with carried
forces (flag 1); prints the iterations of each solve of each:

  python -m microsimulator_b200.profile_case --case guess --cells 1000000 --warm 3 --steps 3

--case graph: the contact graph index (msb_build_contact_graph) of a jammed
colony's contacts after `--steps` steps, from device-resident contacts:

  python -m microsimulator_b200.profile_case --case graph --cells 1000000 --steps 1 --iterations 5

--case trap: steps of the trap colony with its wall boxes, drifting in a
slow swirl (flow drift on), so that every kernel of a step runs:

  python -m microsimulator_b200.profile_case --case trap --cells 300000 --steps 2
"""

from __future__ import annotations

import argparse
import json

import numpy as np


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


def train_case(args) -> None:
    """Training steps of the warm-start network on random bf16 features: the
    tcgen05 forward keeping its activations, the backward pass's tcgen05
    GEMMs (split-K at this batch size) and Adam, --iterations steps of a
    batch of --cells rows, timed with CUDA events."""
    import torch

    from . import learned
    from .backend import B200Backend

    backend = B200Backend(0)
    net = learned.WarmStartNetwork("cuda:0", seed=args.seed, library=backend._lib)
    gen = torch.Generator(device="cuda:0").manual_seed(args.seed)
    x = torch.randn((args.cells, 96), device="cuda:0", generator=gen).to(torch.bfloat16).view(torch.int16)
    x[:, 81:] = 0
    target = torch.randn((args.cells, 3), device="cuda:0", generator=gen)
    times = []
    for _ in range(args.iterations):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        out, act = net.forward(x, keep=True)
        diff, factor = net.loss_and_grad(out, target)
        net.backward(x, act, (diff * factor).contiguous())
        net.adam(1e-3)
        s1.record()
        torch.cuda.synchronize()
        times.append(s0.elapsed_time(s1))
    # forward 2*n*(96*128 + 2*128*128 + 8*128); backward about twice that
    flops = 3 * 2.0 * args.cells * (96 * 128 + 2 * 128 * 128 + 8 * 128)
    print(json.dumps({"step_ms": times, "rows": args.cells, "approx_flops": flops,
                      "approx_tflops": flops / (min(times) * 1e-3) / 1e12}))
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


def guess_case(args) -> None:
    import torch

    from . import workloads
    from .backend import B200Backend, DeviceCells
    from .types import ContactDynamicsParameters

    backend = B200Backend(0)
    dyn = ContactDynamicsParameters(overlap_tolerance=5e-4)
    world = workloads.jammed(n=args.cells, seed=args.seed)

    def run(w, mode, guess=None):
        backend.set_warm_start(mode)
        if guess is not None:
            backend.set_motion_guess(guess, 0.02)
        cells = DeviceCells(w)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        report = backend.advance_contact_dynamics_device(cells, None, 0.02, dyn)
        end.record()
        torch.cuda.synchronize()
        cells.download(w)
        w.next_id = int(w.ids.max()) + 1
        solves = backend.last_step_solves()
        return {"ms": round(start.elapsed_time(end), 2), "iterations": report.iterations,
                "solves": solves["iterations"].tolist(), "rows": solves["rows"].tolist(),
                "max_overlap": report.max_overlap}

    def divide(w, k):
        plan = workloads.plan_divisions(w, 0.02, seed=args.seed * 100003 + k)
        w.divide_many(plan.parents, 0.5, plan.rotations)

    previous = None  # the state before step k - 1's divisions
    for k in range(args.warm + args.steps):
        undivided = world.copy()
        divide(world, k)
        before = world.copy()
        plain = run(world, 0)
        if k < args.warm:
            previous = undivided
            continue
        exact = np.zeros((len(before), 3), np.float32)
        exact[:, 0] = world.position_x - before.position_x
        exact[:, 1] = world.position_y - before.position_y
        exact[:, 2] = np.arctan2(before.direction_x * world.direction_y - before.direction_y * world.direction_x,
                                 before.direction_x * world.direction_x + before.direction_y * world.direction_y)
        guessed = run(before.copy(), 2, exact)
        # The upper bound of any start of the multipliers: the step run once
        # with carry-over on (it remembers its own final forces), then the
        # same step again from the same state starting from them.
        run(before.copy(), 1)
        own = run(before.copy(), 1)
        carried_world = previous.copy()
        divide(carried_world, k - 1)
        run(carried_world, 1)  # the previous step, remembered
        divide(carried_world, k)
        carried = run(carried_world, 1) if len(carried_world) == len(before) else None
        backend.set_warm_start(0)
        previous = undivided
        print(json.dumps({"step": k, "cells": len(before), "plain": plain, "exact_guess": guessed,
                          "own_final_forces": own, "carried": carried}))
    backend.close()


def graph_case(args) -> None:
    """The contact graph index of a settled jammed colony's contacts, built
    `--iterations` times from device-resident contacts."""
    import time

    import torch

    from . import workloads
    from .backend import B200Backend
    from .graph import device_index
    from .types import ContactDynamicsParameters

    backend = B200Backend(0)
    world = workloads.jammed(n=args.cells, seed=args.seed)
    for _ in range(args.steps):
        backend.advance_contact_dynamics(world, None, 0.02, ContactDynamicsParameters(overlap_tolerance=5e-4))
    contacts = backend.find_cell_contacts(world)
    records = torch.from_numpy(contacts.view(np.uint8).copy()).to("cuda:0")
    index, _ = device_index(len(world), 2 * len(contacts), "cuda:0")
    torch.cuda.synchronize()
    times = []
    for _ in range(args.iterations):
        t0 = time.perf_counter()
        packed = backend.build_contact_graph_device(records.data_ptr(), len(contacts), len(world), index)
        times.append((time.perf_counter() - t0) * 1e3)
    print(json.dumps({"cells": len(world), "contacts": len(contacts), "neighbor_ids": packed, "call_ms": times}))
    backend.close()


def trap_case(args) -> None:
    """Steps of the trap colony (capsules in a trap with the trap-channel
    device's wall boxes) drifting in a swirling flow: every kernel of the
    step runs, wall contacts and flow drift included."""
    import time

    from . import workloads
    from .backend import B200Backend
    from .types import ContactDynamicsParameters, FlowField

    backend = B200Backend(0)
    world, walls = workloads.trap_colony(n=args.cells, seed=args.seed)
    x = np.concatenate([world.position_x, [0.0]])
    y = np.concatenate([world.position_y, [0.0]])
    spacing = 4.0
    origin = (float(x.min()) - 200.0, float(y.min()) - 200.0, -0.5)
    shape = (int((x.max() - x.min() + 400.0) / spacing) + 1, int((y.max() - y.min() + 400.0) / spacing) + 1, 1)
    sx, sy, sz = shape
    x_faces = np.zeros((sx + 1, sy, sz), np.float32)
    y_faces = np.zeros((sx, sy + 1, sz), np.float32)
    z_faces = np.zeros((sx, sy, sz + 1), np.float32)
    # A slow solid-body swirl, zero on the lattice boundary.
    xs = origin[0] + spacing * np.arange(sx + 1)
    ys = origin[1] + spacing * (np.arange(sy) + 0.5)
    x_faces[1:-1, :, 0] = (-0.002 * (ys[None, :] - ys.mean()) + 0.0 * xs[1:-1, None]).astype(np.float32)
    xs = origin[0] + spacing * (np.arange(sx) + 0.5)
    y_faces[:, 1:-1, 0] = (0.002 * (xs[:, None] - xs.mean())).astype(np.float32)
    backend.set_flow_field(FlowField(shape, origin, (spacing, spacing, 1.0), x_faces, y_faces, z_faces, None))
    dyn = ContactDynamicsParameters(overlap_tolerance=5e-4, flow_drift=True)
    for step in range(args.steps):
        plan = workloads.plan_divisions(world, 1.0, seed=args.seed * 7919 + step, minimum_length=4.0)
        world.divide_many(plan.parents, 0.5, plan.rotations)
        t0 = time.perf_counter()
        result = backend.advance_contact_dynamics(world, walls, 0.02, dyn)
        world.next_id = int(world.ids.max()) + 1
        print(json.dumps({"step": step, "cells": len(world), "ms": round(1e3 * (time.perf_counter() - t0), 2),
                          "iterations": result.report.iterations, "substeps": result.report.substeps,
                          "phases": backend.last_step_phases()}))
    backend.close()


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--case", default="bb", choices=["bb", "mlp", "train", "batch", "guess", "graph", "trap"])
    p.add_argument("--warm", type=int, default=3)
    p.add_argument("--colonies", type=int, default=64)
    p.add_argument("--cells", type=int, default=500_000)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--iterations", type=int, default=3)
    p.add_argument("--seed", type=int, default=42)
    args = p.parse_args()
    if args.case == "mlp":
        mlp_case(args)
        return
    if args.case == "train":
        train_case(args)
        return
    if args.case == "batch":
        batch_case(args)
        return
    if args.case == "guess":
        guess_case(args)
        return
    if args.case == "graph":
        graph_case(args)
        return
    if args.case == "trap":
        trap_case(args)
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
