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
