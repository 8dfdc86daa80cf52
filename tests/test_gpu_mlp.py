"""The warm-start network's kernels through the C-ABI against the numpy
oracle (oracle/mlp_oracle.py): features bit for bit, the tcgen05 forward
(inference and training) and backward within bf16 tolerances, Adam,
training, and the learned warm start in the stepper."""

import numpy as np
import pytest

from microsimulator_b200 import learned, workloads
from microsimulator_b200.backend import B200Backend, DeviceCells
from microsimulator_b200.types import ContactDynamicsParameters
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEVICE = "cuda:0"


def bf16_tensor(values):
    return torch.from_numpy(mo.bf16_bits(values).view(np.int16)).to(DEVICE)


def random_batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, mo.INPUT)).astype(np.float32)
    x[:, mo.FEATURES:] = 0
    return mo.bf16_round(x)


def network(seed, lib):
    net = learned.WarmStartNetwork(DEVICE, seed=seed, library=lib)
    p = mo.init(seed)
    rng = np.random.default_rng(seed + 100)
    p[mo.WEIGHTS:] = rng.normal(0, 0.2, mo.PARAMETERS - mo.WEIGHTS).astype(np.float32)
    p[mo.B_OFFSETS[3] + 3:] = 0
    net.set_parameters(p)
    return net, p


def test_features_match_oracle_bit_for_bit(backend):
    world = workloads.jammed(n=700, seed=11)
    cells = DeviceCells(world, device=DEVICE)
    got = learned.cell_features(backend, cells, DEVICE).cpu().numpy().view(np.uint16)
    ref = mo.features(world.position_x, world.position_y, world.direction_x, world.direction_y, world.lengths)
    # The kernel searches the 3 x 3 bins of 6 um around a cell: it must agree
    # wherever the 16th nearest centre lies within 6 um.
    d = np.hypot(world.position_x[:, None] - world.position_x[None, :],
                 world.position_y[:, None] - world.position_y[None, :])
    np.fill_diagonal(d, np.inf)
    d16 = np.sort(d, axis=1)[:, 15]
    inside = d16 < 5.99
    assert inside.mean() > 0.5
    assert np.array_equal(got[inside], mo.bf16_bits(ref)[inside])
    assert np.all(got[:, mo.FEATURES:] == 0)


def test_forward_matches_oracle(backend):
    net, p = network(1, backend._lib)
    x = random_batch(1000, 2)
    y = net.forward(bf16_tensor(x)).cpu().numpy()
    ref, _ = mo.forward(p, x, round_like_kernels=True)
    scale = np.abs(ref).max()
    assert np.max(np.abs(y - ref)) <= 1e-2 * scale, np.max(np.abs(y - ref)) / scale
    # Rows beyond a tile's end and odd row counts.
    y7 = net.forward(bf16_tensor(x[:7])).cpu().numpy()
    assert np.array_equal(y7, y[:7])


def activations_of(act, n):
    """H1..H3 (bf16) and Z1..Z3 (fp32) from the buffer the training forward keeps."""
    raw = act.cpu().numpy()
    h_bytes, z_bytes = n * mo.HIDDEN * 2, n * mo.HIDDEN * 4
    h = [mo.from_bf16_bits(raw[l * h_bytes:(l + 1) * h_bytes].view(np.uint16).reshape(n, mo.HIDDEN)) for l in range(3)]
    base = 3 * h_bytes
    z = [raw[base + l * z_bytes:base + (l + 1) * z_bytes].view(np.float32).reshape(n, mo.HIDDEN) for l in range(3)]
    return h, z


def test_training_forward_on_tcgen05_matches_inference_and_the_oracle(backend):
    """Training and inference run the same tcgen05 kernel (TMEM
    accumulators): the outputs are the same bits with and without kept
    activations, and the kept pre-activations Z and activations H match the
    numpy oracle's, across tile edges (1, 127, 128, 129 rows) and a larger
    batch."""
    net, p = network(4, backend._lib)
    for n in (1, 127, 128, 129, 5000):
        xn = random_batch(n, 40 + n)
        x = bf16_tensor(xn)
        infer = net.forward(x).cpu().numpy()
        train, act = net.forward(x, keep=True)
        assert np.array_equal(train.cpu().numpy(), infer), n
        ref, cache = mo.forward(p, xn, round_like_kernels=True)
        scale = max(np.abs(ref).max(), 1e-6)
        assert np.max(np.abs(infer - ref)) <= 1e-2 * scale, (n, np.max(np.abs(infer - ref)) / scale)
        h, z = activations_of(act, n)
        for layer in range(3):
            zs = max(np.abs(cache["z"][layer]).max(), 1e-6)
            assert np.max(np.abs(z[layer] - cache["z"][layer])) <= 1e-2 * zs, (n, layer)
            hs = max(np.abs(cache["h"][layer + 1]).max(), 1e-6)
            assert np.max(np.abs(h[layer] - cache["h"][layer + 1])) <= 2e-2 * hs, (n, layer)


@pytest.mark.parametrize("n", [777, 20000])
def test_backward_matches_oracle_gradient(backend, n):
    """The backward GEMMs on tcgen05 (a long k split over several CTAs whose
    partial sums are added in a fixed order at 20,000 rows) against the
    oracle's FP64 gradient."""
    net, p = network(3, backend._lib)
    x = random_batch(n, 4)
    rng = np.random.default_rng(5)
    dy = rng.normal(0, 1, (n, mo.OUTPUTS)).astype(np.float32) / n
    xt = bf16_tensor(x)
    _, act = net.forward(xt, keep=True)
    g = net.backward(xt, act, torch.from_numpy(dy).to(DEVICE)).cpu().numpy().astype(np.float64)
    _, cache = mo.forward(p, x, round_like_kernels=True)
    ref = mo.backward(cache, dy.astype(np.float64))
    blocks = [(mo.W_OFFSETS[i], mo.W_OFFSETS[i + 1]) for i in range(4)]
    blocks += [(mo.B_OFFSETS[i], mo.B_OFFSETS[i + 1]) for i in range(4)]
    for lo, hi in blocks:
        err = np.linalg.norm(g[lo:hi] - ref[lo:hi]) / max(np.linalg.norm(ref[lo:hi]), 1e-30)
        # bf16 output and hidden gradients feed the tensor-core GEMMs.
        assert err < 2e-2, (lo, hi, err)
    assert np.all(g[mo.W_OFFSETS[3] + 3 * mo.HIDDEN:mo.W_OFFSETS[4]] == 0)


def test_adam_matches_oracle(backend):
    net, p = network(6, backend._lib)
    rng = np.random.default_rng(7)
    g = rng.normal(0, 1e-2, mo.PARAMETERS).astype(np.float32)
    net.grads.copy_(torch.from_numpy(g))
    net.adam(1e-3)
    net.grads.copy_(torch.from_numpy(0.5 * g))
    net.adam(1e-3)
    ref, m, v = mo.adam(p.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1, lr=1e-3)
    ref, m, v = mo.adam(ref, 0.5 * g.astype(np.float64), m, v, 2, lr=1e-3)
    got = net.params.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-7)
    assert np.array_equal(net.weights.cpu().numpy().view(np.uint16), mo.bf16_bits(got[:mo.WEIGHTS]))
    assert np.array_equal(net.biases.cpu().numpy(), got[mo.WEIGHTS:])


def test_training_fits_a_teacher_network(backend):
    teacher, _ = network(8, backend._lib)
    x = bf16_tensor(random_batch(20000, 9))
    with torch.no_grad():
        y = teacher.forward(x)
    y = y / y.std(dim=0)
    student = learned.WarmStartNetwork(DEVICE, seed=10, library=backend._lib)
    before = float(((student.forward(x) - y) ** 2).mean())
    report = student.train(x, y, x[:4000], y[:4000], steps=300, batch=4096, lr=2e-3)
    assert report.validation_loss < 0.3 * before, (before, report)


def test_learned_warm_start_predicts_motion_and_keeps_the_tolerance(backend):
    """What the trained network gains: its validation error against the
    zero guess, and the stepper's iterations with its guess against the
    same start without it (printed); the step it warm-starts lands within
    tolerance of the zero-start step."""
    from tests.test_gpu_warm_start import colony, divide, TOLERANCE, DT

    p = ContactDynamicsParameters(overlap_tolerance=TOLERANCE)
    trainer = B200Backend(0)
    try:
        world = colony(seed=21, n=4000)
        net, report = learned.train_warm_start(trainer, world, p, DT, lambda w, k: divide(w, 500 + k, 21),
                                               collect_steps=3, train_steps=400)
    finally:
        trainer.close()
    print("training", report)
    assert report.validation_loss < 0.9 * report.validation_variance
    divide(world, 900, 21)
    b = B200Backend(0)
    try:
        net.install(b)
        plain = world.copy()
        rp = b.advance_contact_dynamics(plain, None, DT, p)
        b.set_warm_start(b.WARM_START_LEARNED)
        warm = world.copy()
        rw = b.advance_contact_dynamics(warm, None, DT, p)
        log = b.last_step_solves()
    finally:
        b.close()
    print("iterations plain", rp.report.iterations, "learned", rw.report.iterations)
    assert log["status"][-1] == 0
    spread = np.max(np.abs(warm.geometry()[:, :3] - plain.geometry()[:, :3]))
    assert spread < 4 * TOLERANCE, spread


def test_learned_mode_needs_a_network():
    b = B200Backend(0)
    try:
        b.set_warm_start(b.WARM_START_LEARNED)
        world = workloads.jammed(n=200, seed=1)
        with pytest.raises(ValueError):
            b.advance_contact_dynamics(world, None, 0.02, ContactDynamicsParameters())
    finally:
        b.close()
