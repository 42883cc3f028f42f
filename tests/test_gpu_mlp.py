"""The MLP radiance cache's tensor-core kernels against a plain PyTorch fp32
reference of the same network: BF16-rounded inputs, weights and hidden
activations, FP32 accumulation, ReLU, exp on the first three outputs."""
import numpy as np
import pytest
import torch

import vgi

pytestmark = pytest.mark.gpu

LAYERS = vgi.GpuTracer.MLP_LAYERS


def random_weights(seed):
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, 1.0 / np.sqrt(i), size=(i, o)).astype(np.float32) for i, o in LAYERS]
    return np.concatenate([p.reshape(-1) for p in parts])


def split(master):
    out, k = [], 0
    for i, o in LAYERS:
        out.append(master[k:k + i * o].reshape(i, o))
        k += i * o
    return out


def torch_forward(master, features):
    x = torch.tensor(features).bfloat16().float()
    ws = [torch.tensor(w).bfloat16().float() for w in split(master)]
    for l, w in enumerate(ws):
        x = x @ w
        if l + 1 < len(ws):
            x = torch.relu(x).bfloat16().float()
    return torch.exp(x[:, :3]).numpy()


@pytest.mark.parametrize("n", [1, 127, 128, 4099])
def test_mlp_forward_matches_torch(gpu, n):
    master = random_weights(3)
    rng = np.random.default_rng(n)
    features = np.zeros((n, 96), np.float32)
    features[:, :81] = rng.uniform(-1.0, 1.0, size=(n, 81))
    gpu.mlp_set_weights(master)
    got = gpu.mlp_forward(features)
    want = torch_forward(master, features)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-3)
    # The tensor cores sum in another order than torch; a hidden value that
    # lands next to a BF16 rounding boundary then rounds the other way.
    assert np.median(rel) < 1e-3 and rel.max() < 3e-2, (np.median(rel), rel.max())
    assert np.allclose(gpu.mlp_get_weights(), master)


LUMA = np.array([0.2126, 0.7152, 0.0722], np.float32)


def torch_gradients(master, features, targets):
    """Autograd of the relative-luminance loss through the same roundings:
    BF16 inputs, weights and hidden activations (the casts also round the
    gradients flowing back through them), FP32 products."""
    x = torch.tensor(features).bfloat16().float()
    ws = [torch.tensor(w).bfloat16().float().requires_grad_() for w in split(master)]
    h = x
    for l, w in enumerate(ws):
        z = h @ w
        if l + 1 < len(ws):
            h = torch.relu(z).bfloat16().float()
    p = torch.exp(z[:, :3])
    y = torch.tensor(targets)
    lum = (p @ torch.tensor(LUMA)).detach()
    loss = (((p - y) ** 2).sum(1) / (lum ** 2 + 0.01)).sum() / len(features)
    loss.backward()
    return np.concatenate([w.grad.numpy().reshape(-1) for w in ws]), float(loss.detach())


def batch(n, seed):
    rng = np.random.default_rng(seed)
    features = np.zeros((n, 96), np.float32)
    features[:, :81] = rng.uniform(-1.0, 1.0, size=(n, 81))
    targets = rng.uniform(0.05, 2.0, size=(n, 3)).astype(np.float32)
    return features, targets


@pytest.mark.parametrize("n", [1, 200, 4099, 65536])
def test_mlp_gradients_match_torch_autograd(gpu, n):
    master = random_weights(5)
    features, targets = batch(n, n + 1)
    gpu.mlp_set_weights(master)
    got, loss = gpu.mlp_gradients(features, targets)
    want, want_loss = torch_gradients(master, features, targets)
    assert abs(loss - want_loss) <= 1e-3 * abs(want_loss), (loss, want_loss)
    k = 0
    for i, o in LAYERS:
        g, w = got[k:k + i * o], want[k:k + i * o]
        k += i * o
        # The output gradient is rounded to BF16 before the products (torch
        # keeps it in FP32) and the tensor cores sum in another order.
        err = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-30)
        assert err < 2e-2, ((i, o), err)
    assert np.allclose(gpu.mlp_get_weights(), master)


def test_mlp_adam_steps_match_numpy(gpu):
    master = random_weights(7)
    features, targets = batch(3000, 11)
    gpu.mlp_set_weights(master)
    m = np.zeros_like(master)
    v = np.zeros_like(master)
    w = master.copy()
    lr, b1, b2 = 1e-2, 0.9, 0.99
    for step in (1, 2, 3):
        g, loss = gpu.mlp_gradients(features, targets)
        train_loss = gpu.mlp_train(features, targets, lr)
        assert train_loss == pytest.approx(loss, rel=1e-6)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + 1e-8)
        got = gpu.mlp_get_weights()
        # The kernel's Adam rounds in FP32 and numpy's here in FP64; the
        # bound leaves room for a gradient near 0, where Adam's
        # normalisation makes the step most sensitive to rounding.
        diff = np.abs(got - w)
        assert diff[np.abs(g) > 1e-6].max() < 1e-4, diff.max()
        assert np.mean(diff < 1e-4) > 0.999
        w = got


def test_mlp_apply_gradients_takes_the_train_step(gpu):
    """The data-parallel step: the gradient of a batch (mlp_gradients)
    applied with mlp_apply_gradients is the step mlp_train takes on that
    batch; a CUDA tensor and a host array of the same gradient give the
    same step exactly."""
    master = random_weights(9)
    features, targets = batch(2000, 4)
    gpu.mlp_set_weights(master)
    g, loss = gpu.mlp_gradients(features, targets)
    gpu.mlp_apply_gradients(g, loss, 1e-2)
    via_apply = gpu.mlp_get_weights()
    gpu.mlp_set_weights(master)
    gpu.mlp_train(features, targets, 1e-2)
    via_train = gpu.mlp_get_weights()
    diff = np.abs(via_apply - via_train)
    assert diff[np.abs(g) > 1e-6].max() < 1e-4, diff.max()
    assert np.mean(diff < 1e-4) > 0.999
    gpu.mlp_set_weights(master)
    gpu.mlp_apply_gradients(torch.tensor(g).cuda(), loss, 1e-2)
    assert np.array_equal(gpu.mlp_get_weights(), via_apply)


def test_mlp_training_fits_a_smooth_field(gpu):
    """65,536 rows (one frame's training batch) of a smooth radiance field:
    200 Adam steps at lr 1e-2 bring the loss down by more than 10x."""
    rng = np.random.default_rng(2)
    n = 65536
    features = np.zeros((n, 96), np.float32)
    features[:, :81] = rng.uniform(-1.0, 1.0, size=(n, 81))
    base = features[:, :3]
    targets = (0.6 + 0.5 * np.sin(2.0 * base + np.array([0.0, 1.0, 2.0], np.float32))).astype(np.float32)
    gpu.mlp_set_weights(random_weights(9) * 0.5)
    first = gpu.mlp_train(features, targets, 1e-2)
    for _ in range(199):
        last = gpu.mlp_train(features, targets, 1e-2)
    assert np.isfinite(last) and last < first / 10.0, (first, last)
    pred = gpu.mlp_forward(features[:1024])
    assert np.all(np.isfinite(pred))
