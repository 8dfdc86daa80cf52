"""The learned warm start: a per-cell network that guesses each cell's
displacement over a step from its 16 nearest neighbours, trained on the GPU
with the library's own kernels (msb_cell_features, msb_mlp_forward,
msb_mlp_backward, msb_mlp_adam) on trajectories of the plain stepper.

A guess changes only the multipliers a step's first solve starts from
(warm-start flag 4): every solve still converges to the same tolerance and
the stepper's own overlap test decides acceptance.

torch tensors serve as device allocations; all arithmetic on them that
belongs to the network runs in the library's kernels.
"""

from __future__ import annotations

import ctypes
import math
from ctypes import c_float, c_void_p
from dataclasses import dataclass

import numpy as np

from . import abi

INPUT = 96
HIDDEN = 128
OUTPUTS = 3
OUTPUT_PAD = 8
FEATURES = 81
W_SHAPES = [(HIDDEN, INPUT), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUTPUT_PAD, HIDDEN)]
WEIGHTS = sum(a * b for a, b in W_SHAPES)
BIASES = 3 * HIDDEN + OUTPUT_PAD
PARAMETERS = WEIGHTS + BIASES


def initial_parameters(seed: int = 0) -> np.ndarray:
    """He-uniform hidden weights, a small output layer, zero biases; padded
    input columns and output rows zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMETERS, dtype=np.float32)
    at = 0
    for i, (o, k) in enumerate(W_SHAPES):
        limit = math.sqrt(6.0 / k) if i < 3 else math.sqrt(1.0 / k)
        w = rng.uniform(-limit, limit, size=(o, k)).astype(np.float32)
        if i == 0:
            w[:, FEATURES:] = 0.0
        if i == 3:
            w[OUTPUTS:] = 0.0
        p[at:at + o * k] = w.ravel()
        at += o * k
    return p


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round float32 to bf16 (nearest, ties to even) and return the bits."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def body_frame_displacement(before, after) -> np.ndarray:
    """(along the axis, across it, turn) of each cell from `before` to
    `after` (same slots), in the cell's frame before the step."""
    ax, ay = before.direction_x.astype(np.float64), before.direction_y.astype(np.float64)
    norm = np.hypot(ax, ay)
    norm[norm == 0] = 1.0
    ax, ay = ax / norm, ay / norm
    dx = after.position_x.astype(np.float64) - before.position_x
    dy = after.position_y.astype(np.float64) - before.position_y
    cross = before.direction_x * after.direction_y - before.direction_y * after.direction_x
    dot = before.direction_x * after.direction_x + before.direction_y * after.direction_y
    out = np.empty((len(before), 3), dtype=np.float32)
    out[:, 0] = dx * ax + dy * ay
    out[:, 1] = dy * ax - dx * ay
    out[:, 2] = np.arctan2(cross, dot)
    return out


@dataclass
class TrainingReport:
    samples: int
    validation_samples: int
    steps: int
    train_loss: float
    validation_loss: float
    validation_variance: float  # the loss of always guessing zero displacement
    seconds: float


class WarmStartNetwork:
    """Parameters, Adam state and the bf16 copies the kernels read, in GPU
    memory."""

    def __init__(self, device: str = "cuda:0", seed: int = 0, library=None):
        import torch

        self.torch = torch
        self.device = device
        self._lib = library or abi.load_library()
        p = initial_parameters(seed)
        self.params = torch.from_numpy(p).to(device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grads = torch.zeros_like(self.params)
        self.weights = torch.from_numpy(to_bf16_bits(p[:WEIGHTS]).view(np.int16)).to(device)
        self.biases = self.params[WEIGHTS:].clone()
        self.scale = np.ones(3, dtype=np.float32)
        self.step = 0

    def set_parameters(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        self.params.copy_(self.torch.from_numpy(p))
        self.weights.copy_(self.torch.from_numpy(to_bf16_bits(p[:WEIGHTS]).view(np.int16)))
        self.biases.copy_(self.params[WEIGHTS:])

    def _check(self, status: int) -> None:
        abi.raise_for_status(status, "warm-start network call failed")

    def forward(self, features, keep: bool = False):
        """Normalized outputs (n x 3) for bf16 features (n x 96, int16 bits);
        with keep, also the activations for ``backward``."""
        torch = self.torch
        n = int(features.shape[0])
        outputs = torch.empty((n, OUTPUTS), dtype=torch.float32, device=self.device)
        activations = None
        if keep:
            activations = torch.empty(int(self._lib.msb_mlp_activation_bytes(n)), dtype=torch.uint8,
                                      device=self.device)
        stream = c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        self._check(self._lib.msb_mlp_forward(
            c_void_p(self.weights.data_ptr()), c_void_p(self.biases.data_ptr()), c_void_p(features.data_ptr()), n,
            c_void_p(outputs.data_ptr()), c_void_p(activations.data_ptr()) if keep else None, stream))
        return (outputs, activations) if keep else outputs

    def backward(self, features, activations, output_grad):
        torch = self.torch
        n = int(features.shape[0])
        scratch = torch.empty(int(self._lib.msb_mlp_backward_scratch_bytes(n)), dtype=torch.uint8,
                              device=self.device)
        stream = c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        self._check(self._lib.msb_mlp_backward(
            c_void_p(self.weights.data_ptr()), c_void_p(features.data_ptr()), n, c_void_p(activations.data_ptr()),
            c_void_p(output_grad.data_ptr()), c_void_p(self.grads.data_ptr()), c_void_p(scratch.data_ptr()), stream))
        return self.grads

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, epsilon: float = 1e-8) -> None:
        self.step += 1
        stream = c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)
        self._check(self._lib.msb_mlp_adam(
            c_void_p(self.params.data_ptr()), c_void_p(self.grads.data_ptr()), c_void_p(self.m.data_ptr()),
            c_void_p(self.v.data_ptr()), self.step, c_float(lr), c_float(beta1), c_float(beta2), c_float(epsilon),
            c_void_p(self.weights.data_ptr()), c_void_p(self.biases.data_ptr()), stream))

    def loss_and_grad(self, outputs, targets):
        """Mean squared error over the batch and the outputs, and its gradient."""
        diff = outputs - targets
        return diff, 2.0 / diff.numel()

    def train(self, features, targets, validation_features=None, validation_targets=None, steps: int = 1500,
              batch: int = 8192, lr: float = 2e-3, seed: int = 0) -> TrainingReport:
        """Adam on normalized targets (targets / self.scale) with a cosine
        learning-rate decay."""
        import time

        torch = self.torch
        n = int(features.shape[0])
        scale = torch.from_numpy(self.scale).to(self.device)
        y = targets / scale
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        t0 = time.perf_counter()
        last = 0.0
        for k in range(steps):
            index = torch.randint(0, n, (min(batch, n),), device=self.device, generator=gen)
            xb = features[index].contiguous()
            yb = y[index].contiguous()
            out, act = self.forward(xb, keep=True)
            diff, factor = self.loss_and_grad(out, yb)
            grad = (diff * factor).contiguous()
            self.backward(xb, act, grad)
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * k / steps))
            self.adam(max(rate, lr * 1e-3))
            if k == steps - 1:
                last = float((diff * diff).mean())
        torch.cuda.synchronize(self.device)
        seconds = time.perf_counter() - t0
        val_loss = val_var = float("nan")
        vn = 0
        if validation_features is not None:
            vn = int(validation_features.shape[0])
            vy = validation_targets / scale
            out = self.forward(validation_features)
            val_loss = float(((out - vy) ** 2).mean())
            val_var = float((vy ** 2).mean())
        return TrainingReport(n, vn, steps, last, val_loss, val_var, seconds)

    def install(self, backend) -> None:
        """Gives a backend this network for warm-start flag 4."""
        scale = np.ascontiguousarray(self.scale, dtype=np.float32)
        self.torch.cuda.synchronize(self.device)
        backend._check(backend._lib.msb_set_warm_start_network(
            backend._handle, c_void_p(self.weights.data_ptr()), c_void_p(self.biases.data_ptr()),
            c_void_p(abi.ptr(scale))))


def cell_features(backend, cells, device: str = "cuda:0"):
    """Features (n x 96 bf16 bits as int16) of DeviceCells through the C-ABI."""
    import torch

    out = torch.empty((cells.count, INPUT), dtype=torch.int16, device=device)
    arrays = cells.arrays()
    torch.cuda.synchronize(device)
    backend._check(backend._lib.msb_cell_features(backend._handle, ctypes.byref(arrays), c_void_p(out.data_ptr())))
    return out


def collect_trajectories(backend, world, steps: int, dynamics, dt: float, divide, device: str = "cuda:0"):
    """Features before and body-frame displacements over `steps` plain steps
    of `world` (updated in place); divide(world, k) runs before step k."""
    import torch

    from .backend import DeviceCells

    feats, targets = [], []
    backend.set_warm_start(0)
    for k in range(steps):
        divide(world, k)
        cells = DeviceCells(world, device=device)
        feats.append(cell_features(backend, cells, device))
        before = world.copy()
        backend.advance_contact_dynamics_device(cells, None, dt, dynamics)
        cells.download(world)
        world.next_id = int(world.ids.max()) + 1
        targets.append(torch.from_numpy(body_frame_displacement(before, world)).to(device))
    return torch.cat(feats), torch.cat(targets)


def train_warm_start(backend, world, dynamics, dt: float, divide, collect_steps: int = 4, train_steps: int = 1500,
                     validation_fraction: float = 0.1, seed: int = 0, device: str = "cuda:0"):
    """Trajectories of the plain stepper on `world`, a network trained on
    them, and its report."""
    import torch

    x, y = collect_trajectories(backend, world, collect_steps, dynamics, dt, divide, device)
    n = int(x.shape[0])
    gen = torch.Generator(device=device)
    gen.manual_seed(seed + 1)
    order = torch.randperm(n, device=device, generator=gen)
    cut = int(n * (1.0 - validation_fraction))
    train_x, train_y = x[order[:cut]].contiguous(), y[order[:cut]].contiguous()
    val_x, val_y = x[order[cut:]].contiguous(), y[order[cut:]].contiguous()
    net = WarmStartNetwork(device=device, seed=seed, library=backend._lib)
    std = train_y.std(dim=0).cpu().numpy().astype(np.float32)
    net.scale = np.maximum(std, 1e-9).astype(np.float32)
    report = net.train(train_x, train_y, val_x, val_y, steps=train_steps, seed=seed)
    return net, report
