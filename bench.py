"""Throughput of the capsule contact-mechanics step: cell-steps/s.

Workload (default): 1,000,000 capsules near jamming (area fraction 0.85,
lengths log-normal mu = ln 3 um, sigma 0.2, radius 0.5 um, orientations
uniform), open domain derived from N and the fraction, growth rate 0.5
(+1 % length per step), 2 % of the cells divided per step with +-0.02 rad
daughter turns, dt 0.02, overlap tolerance 5e-4 um (1e-3 radius).  A step is
Simulation::step(dt, dynamics): the whole contact-dynamics step, relaxed to
the tolerance.  Divisions are input preparation and run between steps.

  value  steps on cells resident in HBM (device-pointer C-ABI call), timed
         with CUDA events, max over ranks
  e2e    the same steps through the host-buffer C-ABI call with the world in
         page-locked host arrays, host<->device copies inside the timed
         region (and, beside it, with ordinary pageable arrays)
  roofline  the BB iteration (body pass + row pass) of the last solved
         system, CUDA events on the backend's stream, against algorithmic
         bytes R*96 + N*128 per iteration
  cpu_baseline  the reference CPU backend (compiled from its sources) on the
         first timed steps of the same colony from the same state, about
         15 s of stepping, all host threads

--impl reference prints the reference CPU backend's line for the same K
timed steps from the same state.
Multi-GPU: each rank steps its own independent colony (replicas; there is no
data-path collective).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

DT = 0.02
TOLERANCE = 5.0e-4
DIVISION_FRACTION = 0.02


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cells", type=int, default=1_000_000)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-learned", action="store_true")
    p.add_argument("--no-sweep", action="store_true")
    p.add_argument("--no-graph", action="store_true")
    p.add_argument("--no-walls", action="store_true")
    p.add_argument("--wall-cells", type=int, default=100_000)
    p.add_argument("--wall-steps", type=int, default=10)
    p.add_argument("--sweep-colonies", type=int, default=256)
    p.add_argument("--train-cells", type=int, default=200_000)
    p.add_argument("--train-steps", type=int, default=1500)
    return p.parse_args()


def dynamics():
    from microsimulator_b200.types import ContactDynamicsParameters

    return ContactDynamicsParameters(overlap_tolerance=TOLERANCE)


def divide(world, step, seed):
    from microsimulator_b200 import workloads

    plan = workloads.plan_divisions(world, DIVISION_FRACTION, seed=seed * 100003 + step)
    world.divide_many(plan.parents, 0.5, plan.rotations)
    return plan


class Clocks:
    """SM clock and throttle reasons sampled through NVML from a background
    thread during a region (every 50 ms, one device).  An external
    `nvidia-smi -lms` poller takes driver locks often enough to stall the
    step's host synchronizations, so the sampling stays in-process and light."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, device, period=0.05):
        self.device = device
        self.period = period
        self.samples = []
        self._stop = None
        self._thread = None
        self._handle = None
        self._max = None

    def __enter__(self):
        import threading

        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            props = torch.cuda.get_device_properties(self.device)
            want = (int(props.pci_domain_id), int(props.pci_bus_id), int(props.pci_device_id))
            # Match on NVML's PCI info (integers): the bus-id lookup takes a
            # string, and CUDA_VISIBLE_DEVICES may renumber the devices.
            for index in range(pynvml.nvmlDeviceGetCount()):
                handle = pynvml.nvmlDeviceGetHandleByIndex(index)
                pci = pynvml.nvmlDeviceGetPciInfo(handle)
                if (int(pci.domain), int(pci.bus), int(pci.device)) == want:
                    self._handle = handle
                    break
            if self._handle is None:
                return self
            self._max = pynvml.nvmlDeviceGetMaxClockInfo(self._handle, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._handle = None
            return self
        self._stop = threading.Event()

        def run():
            import pynvml

            while True:
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(self._handle, pynvml.NVML_CLOCK_SM)
                    reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self._handle)
                    self.samples.append((sm, reasons))
                except Exception:
                    pass
                if self._stop.wait(self.period):
                    break

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self._max, "reasons": ["unsampled"], "samples": 0}
        reasons = sorted({name for _, bits in self.samples for mask, name in self.REASONS.items() if bits & mask})
        return {"sm_mhz": float(np.median([s for s, _ in self.samples])), "sm_max_mhz": self._max,
                "reasons": reasons, "samples": len(self.samples), "source": "nvml"}


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes of one BB iteration as a multiple of its algorithmic bytes,
    from the committed ncu capture (profiles/bb_iteration_traffic.json, the
    1M-capsule colony's system after 2 steps: 2.2M rows, 1.04M bodies); None
    without one.  The bench scales it to its own launches by the algorithmic
    bytes, which grow with rows and bodies as the traffic does."""
    path = ROOT / "profiles" / "bb_iteration_traffic.json"
    if not path.exists():
        return None
    return json.loads(path.read_text())


def reference_steps(args, world, first_step, seconds, steps_cap, seed):
    """The reference CPU backend (oracle/_ref, compiled from its sources)
    stepping `world` through its own Simulation::step: the benchmark's
    divisions before each step (steps first_step, first_step + 1, ...), timed
    steps until `seconds` of stepping or `steps_cap` steps.  None without the
    library."""
    from oracle.native import REFERENCE_PATH, Reference

    if not REFERENCE_PATH.exists():
        return None
    ref = Reference()
    plan_world = world.copy()
    handle = ref.world_create(plan_world)
    try:
        cells_steps, elapsed, steps, first_cells = 0, 0.0, 0, len(plan_world)
        while steps < steps_cap and (elapsed < seconds or steps == 0):
            plan = divide(plan_world, first_step + steps, seed)
            ref.world_divide(handle, plan.parents, plan.rotations)
            n = len(plan_world)
            t0 = time.perf_counter()
            ref.world_step(handle, DT, dynamics())
            elapsed += time.perf_counter() - t0
            cells_steps += n
            ref.world_read(handle, plan_world)
            plan_world.next_id = int(plan_world.ids.max()) + 1
            steps += 1
        return {"value": cells_steps / elapsed, "unit": "cell-steps/s", "cores": ref.thread_count(),
                "kind": "reference", "steps": steps, "seconds": elapsed, "first_cells": first_cells,
                "last_cells": len(plan_world)}
    finally:
        ref.world_destroy(handle)


def warmed_colony(args, rank=0):
    """The benchmark's colony after its --warmup steps: the jammed random
    start with its divisions, stepped by the GPU stepper (by the reference
    where no GPU is present).  The warm-up steps resolve the random start's
    deep overlaps; on the reference CPU backend the first of them alone takes
    many minutes at 1M capsules, so both arms take the state after them from
    the GPU stepper (the same bits), and the reference's timed steps start
    from it.  Returns the colony and what stepped the warm-up."""
    import torch

    from microsimulator_b200 import workloads

    world = workloads.jammed(n=args.cells, seed=args.seed + rank)
    if not torch.cuda.is_available():
        from oracle.native import Reference

        ref = Reference()
        handle = ref.world_create(world)
        try:
            for step in range(args.warmup):
                plan = divide(world, step, args.seed + rank)
                ref.world_divide(handle, plan.parents, plan.rotations)
                ref.world_step(handle, DT, dynamics())
                ref.world_read(handle, world)
                world.next_id = int(world.ids.max()) + 1
        finally:
            ref.world_destroy(handle)
        return world, "the reference CPU backend (no GPU present)"
    from microsimulator_b200.backend import B200Backend, DeviceCells

    local = int(os.environ.get("LOCAL_RANK", "0"))
    backend = B200Backend(local)
    try:
        for step in range(args.warmup):
            divide(world, step, args.seed + rank)
            cells = DeviceCells(world, device=f"cuda:{local}")
            backend.advance_contact_dynamics_device(cells, None, DT, dynamics())
            torch.cuda.synchronize()
            cells.download(world)
            world.next_id = int(world.ids.max()) + 1
    finally:
        backend.close()
    return world, "the GPU stepper, as for the GPU arm"


def config(args, world_size):
    return {
        "workload": f"jammed colony, {args.cells} capsules, area fraction 0.85, log-normal lengths, "
                    "growth 0.5, 2% divisions/step, dt 0.02, tol 5e-4 um (1e-3 r)",
        "cells_per_gpu": args.cells,
        "parallelism": f"replicas{world_size}",
        "l2": "inputs larger than L2 (working set > 126 MB at 1M capsules)",
    }


def reference_arm(args):
    """The reference CPU backend on this arm's workload: the 1M-capsule
    colony's K timed steps (with the same divisions) from the state after the
    warm-up steps, all host threads.  Stops early after 600 s of stepping and
    says so in cpu_baseline.sample."""
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle.native import REFERENCE_PATH

    if not REFERENCE_PATH.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmsref.so was not built"}))
        return
    world, warm_by = warmed_colony(args)
    sample = reference_steps(args, world, args.warmup, seconds=600.0, steps_cap=max(1, args.steps), seed=args.seed)
    sample["sample"] = (f"the {args.cells}-capsule colony's timed steps {args.warmup}..{args.warmup + sample['steps'] - 1}"
                        f" ({sample['first_cells']} -> {sample['last_cells']} capsules) from the state after "
                        f"{args.warmup} warm-up steps (stepped by {warm_by}), {sample['seconds']:.1f} s of stepping")
    for key in ("steps", "seconds", "first_cells", "last_cells"):
        sample.pop(key)
    print(json.dumps({
        "impl": "reference",
        "metric": "cell-steps/s at 1M capsules, 1e-3 overlap tol",
        "value": sample["value"], "unit": "cell-steps/s", "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": config(args, world_size),
        "cpu_baseline": sample,
        "e2e": {"value": sample["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def walls_arm(args, backend, local, with_cpu):
    """Capsules at area fraction 0.7 in a trap opening onto a channel with
    the trap-channel device's wall boxes (100,000 by default), growth 0.5
    (+1 %/step), every cell of length >= 4 um divided before a step (daughter
    turns +-0.02 rad).  Device-resident steps timed with CUDA events; beside
    them the reference CPU backend on the same workload."""
    import torch

    from microsimulator_b200 import workloads
    from microsimulator_b200.backend import DeviceCells

    world, walls = workloads.trap_colony(n=args.wall_cells, seed=args.seed)
    dyn = dynamics()

    def divide_long(w, k):
        plan = workloads.plan_divisions(w, 1.0, seed=args.seed * 7919 + k, minimum_length=4.0)
        w.divide_many(plan.parents, 0.5, plan.rotations)
        return plan

    def step(w, k):
        divide_long(w, k)
        cells = DeviceCells(w, device=f"cuda:{local}")
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        report = backend.advance_contact_dynamics_device(cells, walls, DT, dyn)
        end.record()
        torch.cuda.synchronize()
        cells.download(w)
        w.next_id = int(w.ids.max()) + 1
        return start.elapsed_time(end), report

    for k in range(3):
        step(world, k)
    snapshot = world.copy()
    total_ms, cell_steps, iterations, rows = 0.0, 0, 0, 0
    for k in range(args.wall_steps):
        ms, report = step(world, 3 + k)
        total_ms += ms
        cell_steps += len(world)
        iterations += report.iterations
        rows = max(rows, report.max_rows)
    out = {"workload": f"{args.wall_cells} capsules, lengths U[2, 4] um, area fraction 0.7 in a trap opening onto a "
                       "channel (trap-channel device wall boxes, 100 x 40 um trap aspect scaled to hold them), "
                       "growth 0.5, division at 4 um, dt 0.02, tol 5e-4 um",
           "walls": len(walls), "cells_after": len(world), "steps": args.wall_steps,
           "value": cell_steps / (total_ms * 1e-3), "unit": "cell-steps/s", "ms_per_step": total_ms / args.wall_steps,
           "bb_iterations_per_step": iterations / args.wall_steps, "max_rows": rows}
    if with_cpu:
        from oracle.native import REFERENCE_PATH, Reference

        if REFERENCE_PATH.exists():
            ref = Reference()
            plan_world = snapshot.copy()
            handle = ref.world_create(plan_world, walls)
            try:
                elapsed, ref_cells, ref_steps = 0.0, 0, 0
                while ref_steps < min(3, args.wall_steps) and (elapsed < 20.0 or ref_steps == 0):
                    plan = divide_long(plan_world, 3 + ref_steps)
                    ref.world_divide(handle, plan.parents, plan.rotations)
                    t0 = time.perf_counter()
                    ref.world_step(handle, DT, dyn)
                    elapsed += time.perf_counter() - t0
                    ref.world_read(handle, plan_world)
                    plan_world.next_id = int(plan_world.ids.max()) + 1
                    ref_cells += len(plan_world)
                    ref_steps += 1
                out["cpu_baseline"] = {"value": ref_cells / elapsed, "unit": "cell-steps/s",
                                       "cores": ref.thread_count(), "kind": "reference",
                                       "sample": f"the first {ref_steps} timed steps of the same workload, "
                                                 f"{elapsed:.1f} s"}
            finally:
                ref.world_destroy(handle)
    return out


def contact_graph_arm(backend, world, local, with_cpu):
    """The contact graph index (ContactGraph's constructor) of the colony's
    contacts: the C-ABI call on device-resident contacts (wall clock around
    the synchronous call, which reads the validation result once), the
    host-buffer call, and the reference constructor on the same list."""
    import torch

    from microsimulator_b200.graph import device_index

    contacts = backend.find_cell_contacts(world)
    n, count = len(world), len(contacts)
    device = torch.device("cuda", local)
    records = torch.from_numpy(contacts.view(np.uint8).copy()).to(device)
    index, _arrays = device_index(n, 2 * count, device)
    torch.cuda.synchronize()

    def call():
        backend.build_contact_graph_device(records.data_ptr(), count, n, index)

    for _ in range(3):
        call()
    times = []
    for _ in range(10):
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
    device_ms = float(np.median(times)) * 1e3
    host_times = []
    for _ in range(4):
        t0 = time.perf_counter()
        graph = backend.build_contact_graph(contacts, n)
        host_times.append(time.perf_counter() - t0)
    host_ms = float(np.median(host_times[1:])) * 1e3
    packed = int(index.neighbor_count)
    # Every field of every contact is read (validation), the incidence and
    # neighbour ids and both offset arrays written once.
    algorithmic = count * 64 + 2 * count * 8 + packed * 8 + 2 * (n + 1) * 8
    peak, peak_kind = measured_peak()
    achieved = algorithmic / (device_ms * 1e-3) / 1e9
    out = {"workload": f"the contacts of the jammed colony after the timed steps (margin 0), {count} contacts, "
                       f"{n} cells", "contacts": count, "cells": n, "neighbor_ids": packed,
           "device_call_ms": device_ms, "host_buffer_call_ms": host_ms, "algorithmic_bytes": algorithmic,
           "achieved_gbs": achieved, "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
           "check": bool(graph.incidence_offsets[-1] == 2 * count and len(graph.packed_neighbor_ids) == packed)}
    if with_cpu:
        from oracle.native import REFERENCE_PATH, Reference

        if REFERENCE_PATH.exists():
            ref = Reference()
            ref_times = []
            for _ in range(2):
                t0 = time.perf_counter()
                ref.contact_graph(contacts, n)
                ref_times.append(time.perf_counter() - t0)
            out["cpu_baseline"] = {"ms": min(ref_times) * 1e3, "cores": ref.thread_count(), "kind": "reference",
                                   "sample": "ContactGraph(cell_count, contacts) on the same list, "
                                             "including the driver's copies in and out"}
    return out


def learned_arm(args, backend, snapshot, timed, device_step, local, rank, barrier, dist):
    """The learned warm start: a network trained on the GPU on trajectories
    of the plain stepper on a separate colony of the same distribution
    (args.train_cells capsules), then the same K steps as the plain
    measurement from the same state with the network's guess (flag 4) and
    with the guess plus the previous step's forces (flags 4 | 1)."""
    import torch

    from microsimulator_b200 import learned, replicas, workloads

    device = f"cuda:{local}"
    t0 = time.perf_counter()
    train_world = workloads.jammed(n=args.train_cells, seed=args.seed + 1000 + rank)
    for k in range(25):  # the random start's overlaps relax
        device_step(train_world, 5000 + k)
    net, report = learned.train_warm_start(
        backend, train_world, dynamics(), DT, lambda w, k: divide(w, 6000 + k, args.seed + rank),
        collect_steps=4, train_steps=args.train_steps, seed=args.seed, device=device)
    training_s = time.perf_counter() - t0
    net.install(backend)
    out = {"training": {"cells": args.train_cells, "samples": report.samples,
                        "validation_samples": report.validation_samples, "adam_steps": report.steps,
                        "validation_mse": report.validation_loss,
                        "zero_guess_mse": report.validation_variance,
                        "seconds_with_data": training_s}}
    for name, mode in (("learned", 4), ("learned_carry", 5), ("carry", 1)):
        world = snapshot.copy()
        device_step(world.copy(), args.warmup - 1, mode)  # one untimed step in this mode
        backend.set_warm_start(0)  # forget its forces: the timed steps start as the plain ones do
        barrier()
        total_ms, cell_steps, iterations, phases = timed(world, mode)
        barrier()
        total_ms = replicas.max_over_ranks(total_ms, dist, device)
        cells_all = replicas.sum_over_ranks(cell_steps, dist, device)
        out[name] = {"value": cells_all / (total_ms * 1e-3), "ms_per_step": total_ms / args.steps,
                     "bb_iterations_per_step": iterations / args.steps, "phase_ms_per_step": phases}
    backend.set_warm_start(0)
    return out


def sweep_arm(args, backend, local, rank, dist):
    """The parameter sweep: args.sweep_colonies independent colonies
    (log-uniform sizes in [500, 50,000], per-colony stiffness and drag
    factors in [0.5, 2], trap-workload capsule shapes at area fraction 0.7),
    stepped together through the batch C-ABI with cells resident in HBM;
    beside it the same colonies stepped one call each from the same state."""
    import torch

    from microsimulator_b200 import sweep
    from microsimulator_b200.backend import DeviceCells

    from microsimulator_b200 import replicas

    device = f"cuda:{local}"
    full = sweep.sweep_batch(count=args.sweep_colonies, seed=args.seed)
    world_size = dist.get_world_size() if dist is not None else 1
    mine = replicas.shard(full.counts(), rank, world_size)  # every colony on one rank
    batch = sweep.ColonyBatch([full.worlds[i] for i in mine], full.drag[mine], full.stiffness[mine])
    dyn = dynamics()

    def step(k):
        batch.divide(DIVISION_FRACTION, seed=args.seed * 1000 + k)
        cat = batch.concatenated()
        cells = DeviceCells(cat, device=device)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        report, colonies = backend.advance_contact_dynamics_batch(cells, batch.counts(), batch.drag, batch.stiffness,
                                                                  DT, dyn)
        end.record()
        torch.cuda.synchronize()
        cells.download(cat)
        sweep.split_into(cat, batch.worlds)
        for w in batch.worlds:
            if len(w):
                w.next_id = int(w.ids.max()) + 1
        return start.elapsed_time(end), report, colonies, len(cat)

    for k in range(max(args.warmup, 3)):
        step(k)
    before = [w.copy() for w in batch.worlds]
    total_ms, cell_steps, iterations = 0.0, 0, 0
    phases = {name: 0.0 for name in backend.PHASES}
    steps_ms = []
    if dist is not None:
        dist.barrier()
    for k in range(args.steps):
        ms, report, colonies, n = step(100 + k)
        total_ms += ms
        steps_ms.append(round(ms, 2))
        cell_steps += n
        iterations += int(colonies["iterations"].sum())
        converged = int((colonies["status"] == 0).sum())
        deepest = float(colonies["max_overlap"].max()) if len(colonies) else 0.0
        for name, value in backend.last_step_phases().items():
            phases[name] += value / args.steps
    total_ms = replicas.max_over_ranks(total_ms, dist, device)
    cell_steps = replicas.sum_over_ranks(cell_steps, dist, device)
    tuning = backend.batch_tuning()
    # The same colonies one call each, one step, from the state before the timed steps.
    one = sweep.ColonyBatch([w.copy() for w in before], batch.drag, batch.stiffness)
    one.divide(DIVISION_FRACTION, seed=args.seed * 1000 + 100)
    sequential_ms, sequential_cells = 0.0, 0
    from microsimulator_b200.types import ContactDynamicsParameters

    for w, d, st in zip(one.worlds, one.drag, one.stiffness):
        p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE, drag=float(d), contact_stiffness=float(st))
        cells = DeviceCells(w, device=device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        backend.advance_contact_dynamics_device(cells, None, DT, p)
        torch.cuda.synchronize()
        sequential_ms += (time.perf_counter() - t0) * 1e3
        sequential_cells += len(w)
    sizes = full.counts()
    return {
        "sharding": f"{len(full)} colonies shared out over {world_size} rank(s), largest first to the least-loaded "
                    "rank; no collective in the step",
        "workload": f"{len(full)} colonies, {int(sizes.min())}..{int(sizes.max())} capsules (log-uniform 500..50000), "
                    "drag and stiffness factors U[0.5, 2], lengths U[2, 4] um, area fraction 0.7, growth 0.5, "
                    "2% divisions/step, tol 5e-4 um",
        "cells": int(sizes.sum()),
        "cells_this_rank": int(batch.counts().sum()),
        "value": cell_steps / (total_ms * 1e-3),
        "unit": "cell-steps/s",
        "ms_per_step": total_ms / args.steps,
        "bb_iterations_per_step_summed_over_colonies": iterations / args.steps,
        "phase_ms_per_step": phases,
        "steps_ms": steps_ms,
        "colonies_converged_last_step": f"{converged} of {len(batch)} on this rank",
        "deepest_overlap_last_step_um": deepest,
        "tuning": tuning,
        "one_call_per_colony": {"value": sequential_cells / (sequential_ms * 1e-3), "unit": "cell-steps/s",
                                "ms_per_step": sequential_ms, "timing": "host wall clock around each device call"},
    }


def compact(arm):
    """An arm's record without its workload text and per-phase breakdowns
    (those go to stderr in full)."""
    if arm is None:
        return None
    out = {}
    for key, value in arm.items():
        if key in ("workload", "phase_ms_per_step", "sharding", "sample", "how", "timing", "steps_ms"):
            continue
        out[key] = compact(value) if isinstance(value, dict) else value
    return out


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch

    from microsimulator_b200 import replicas, workloads
    from microsimulator_b200.backend import B200Backend, DeviceCells

    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    backend = B200Backend(local)
    world = workloads.jammed(n=args.cells, seed=args.seed + rank)
    dyn = dynamics()

    def device_step(world, step, mode=0):
        backend.set_warm_start(mode)
        divide(world, step, args.seed + rank)
        cells = DeviceCells(world, device=f"cuda:{local}")
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        report = backend.advance_contact_dynamics_device(cells, None, DT, dyn)
        end.record()
        torch.cuda.synchronize()
        cells.download(world)
        world.next_id = int(world.ids.max()) + 1
        return start.elapsed_time(end), report

    # The BB iterations of the timed steps, live: algorithmic bytes of each
    # solve (rows * 96 + cells * 128 per iteration) and the solve phase's
    # CUDA-event time on the backend's stream.
    live = {"bytes": 0, "iterations": 0, "solve_ms": 0.0}
    rechecks = {"full": 0, "kept": 0, "partial": 0}

    def timed(world, mode, record=False):
        """K steps from `world`; device time, cell-steps, iterations and
        phases."""
        total_ms, cell_steps, iterations = 0.0, 0, 0
        phases = {name: 0.0 for name in backend.PHASES}
        per_step = []
        for k in range(args.steps):
            ms, report = device_step(world, args.warmup + k, mode)
            total_ms += ms
            cell_steps += len(world)  # the cells of the step (divisions run before it)
            iterations += report.iterations
            step_phases = backend.last_step_phases()
            for name, value in step_phases.items():
                phases[name] += value / args.steps
            per_step.append({"cells": len(world), "ms": round(ms, 3), "iterations": int(report.iterations),
                             "load_ms": round(step_phases["load"], 3), "solve_ms": round(step_phases["solve"], 3)})
            if record:
                # Every timed step's solves: bytes and iterations, and the
                # solve phase's device time.
                for solve in backend.last_step_solves():
                    live["bytes"] += (int(solve["rows"]) * 96 + len(world) * 128) * int(solve["iterations"])
                    live["iterations"] += int(solve["iterations"])
                live["solve_ms"] += step_phases["solve"]
                for name, count in backend.last_step_searches().items():
                    rechecks[name] += count
        if record and rank == 0:
            print(json.dumps({"arm": "timed_steps", "mode": mode, "steps": per_step}), file=sys.stderr)
        return total_ms, cell_steps, iterations, phases

    for step in range(args.warmup):
        device_step(world, step)
    snapshot = world.copy()
    barrier()
    launches0 = backend.launch_count()
    with Clocks(local) as clocks:
        total_ms, cell_steps, iterations, phases = timed(world, 0, record=True)
    barrier()
    launches = backend.launch_count() - launches0
    prof = backend.profile_iterations(20)

    # e2e: the same steps from the same state through the host-buffer call,
    # host<->device copies inside the timed region.  The world's arrays are
    # kept in page-locked host memory (PinnedCells), which the call copies
    # directly; each step's divisions and the copy of the divided world into
    # those arrays are input preparation, outside the timed region.  Beside
    # it, the same steps with the world in ordinary pageable numpy arrays,
    # which the call stages through its own pinned buffers.
    e2e = None
    if not args.no_e2e:
        from microsimulator_b200.backend import PinnedCells

        def host_steps(pinned):
            world = snapshot.copy()
            # One untimed call first (from a copy): it sizes the context's
            # staging buffers and starts its copy threads.
            warm = snapshot.copy()
            divide(warm, args.warmup - 1, args.seed + rank)
            backend.advance_contact_dynamics(warm, None, DT, dyn)
            cells = PinnedCells(int(len(snapshot) * 1.5) + 1024) if pinned else None
            seconds, cells_total, h2d, d2h = 0.0, 0, 0, 0
            for k in range(args.steps):
                divide(world, args.warmup + k, args.seed + rank)
                n = len(world)
                if pinned:
                    cells.load(world)
                barrier()
                t0 = time.perf_counter()
                if pinned:
                    backend.advance_contact_dynamics(cells, None, DT, dyn, outputs=cells.outputs())
                else:
                    backend.advance_contact_dynamics(world, None, DT, dyn)
                torch.cuda.synchronize()
                seconds += time.perf_counter() - t0
                if pinned:
                    cells.store(world)
                world.next_id = int(world.ids.max()) + 1
                cells_total += n
                h2d += n * (8 + 8 * 4 + 4 + 1)
                d2h += n * (7 * 4 + 5 * 4)
            seconds = replicas.max_over_ranks(seconds, dist, f"cuda:{local}")
            cells_total = replicas.sum_over_ranks(cells_total, dist, f"cuda:{local}")
            return cells_total / seconds, h2d // args.steps, d2h // args.steps

        value_pinned, h2d, d2h = host_steps(True)
        value_pageable, _, _ = host_steps(False)
        e2e = {"value": value_pinned, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "host_memory": "the world's arrays page-locked (PinnedCells), copied by DMA without staging",
               "pageable": {"value": value_pageable,
                            "host_memory": "ordinary numpy arrays, staged through the library's pinned buffers"}}

    walls_line = None
    if not args.no_walls and world_size == 1:
        walls_line = walls_arm(args, backend, local, with_cpu=not args.no_cpu)

    graph_line = None
    if not args.no_graph and world_size == 1:
        graph_line = contact_graph_arm(backend, world, local, with_cpu=not args.no_cpu)

    sweep_line = None
    if not args.no_sweep:
        sweep_line = sweep_arm(args, backend, local, rank, dist)
    learned = None
    if not args.no_learned:
        learned = learned_arm(args, backend, snapshot, timed, device_step, local, rank, barrier, dist)

    total = replicas.max_over_ranks(total_ms, dist, f"cuda:{local}")
    value = replicas.sum_over_ranks(cell_steps, dist, f"cuda:{local}") / (total * 1e-3)

    # The dominant kernel is the BB iteration (body pass + row pass), run by
    # the solve graph.  achieved = the live algorithmic bytes of every
    # iteration of the timed steps over the solve phase's time: the phase
    # also holds each solve's bound and initial passes and its graph launch,
    # so the figure is a lower bound.  The timing hook's separate launches
    # give the two passes apart (their split, for the ncu shares).
    peak, peak_kind = measured_peak()
    algorithmic = live["bytes"] / max(1, live["iterations"])
    iteration_ms = live["solve_ms"] / max(1, live["iterations"])
    achieved = live["bytes"] / (live["solve_ms"] * 1e-3) / 1e9 if live["solve_ms"] > 0 else 0.0
    traffic = ncu_traffic()
    traffic_bytes = None
    if traffic is not None:
        traffic_bytes = algorithmic * traffic["ratio_to_algorithmic"]

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu:
        # The reference CPU backend on the first timed steps of the same
        # colony from the same state (the snapshot after the warm-up).
        cpu = reference_steps(args, snapshot, args.warmup, seconds=args.cpu_seconds, steps_cap=args.steps,
                              seed=args.seed + rank)
        if cpu is not None:
            cpu["sample"] = (f"the first {cpu['steps']} timed steps of the same colony from the same state "
                             f"({cpu['first_cells']} capsules), {cpu['seconds']:.1f} s of stepping")
            for key in ("steps", "seconds", "first_cells", "last_cells"):
                cpu.pop(key)

    if rank == 0:
        # The arms' full records go to stderr, one JSON line each; the
        # benchmark line keeps their headline figures.
        for name, arm in (("learned", learned), ("sweep", sweep_line), ("walls", walls_line),
                          ("contact_graph", graph_line)):
            if arm is not None:
                print(json.dumps({"arm": name, **arm}), file=sys.stderr)
        learned, sweep_line, walls_line, graph_line = (compact(learned), compact(sweep_line), compact(walls_line),
                                                       compact(graph_line))
        line = {
            "metric": "cell-steps/s at 1M capsules, 1e-3 overlap tol",
            "value": value,
            "unit": "cell-steps/s",
            "n_gpus": world_size,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": config(args, world_size),
            "path": "plain (zero-start multipliers: the reference's semantics)",
            "bb_iterations_per_step": iterations / args.steps,
            "learned": learned,
            "sweep": sweep_line,
            "contact_graph": graph_line,
            "walls": walls_line,
            "phase_ms_per_step": phases,
            # The timed steps' overlap re-checks by how their candidates were found.
            "rechecks": rechecks,
            "roofline": {
                "kernel": "bb_iteration (body pass + row pass)",
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "peak_kind": f"{peak_kind} hbm_gbs",
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic_bytes,
                "algorithmic_bytes": algorithmic,
                "iteration_ms": iteration_ms,
                "iterations": live["iterations"],
                "measured": "CUDA events on the backend stream around the solve phase of the timed steps; bytes = "
                            "sum over solves of (rows * 96 + cells * 128) * iterations",
                "passes": {"body_ms": prof["body_ms"], "row_ms": prof["row_ms"], "rows": prof["rows"],
                           "bodies": prof["bodies"],
                           "how": "timing hook after the timed region: 20 iterations as separate launches"},
            },
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    backend.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
