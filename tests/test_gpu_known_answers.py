"""Analytic known answers of the reference's GPU tests, on the B200 path.

In a closed furnace whose walls share emission E and reflectance r, every
face receives E / (1 - r) once bounces are unlimited, and E * sum(r^k),
k = 0..H, with H explicit diffuse hits (research.rs:19-21, 71-115). The
cache-terminated world cache must converge to the first
(gpu/cache_tests.rs:41-101); a cacheless trace must match the second
(gpu/view_tests.rs:388-460). Tolerances are the reference's.
"""
import numpy as np
import pytest

import vgi
from test_gpu_parity import furnace_case

E = np.array([0.7, 1.3, 0.2])
R = np.array([0.3, 0.55, 0.7])


@pytest.mark.gpu
def test_cached_furnace_converges_to_infinite_bounce_series(gpu):
    case = furnace_case(history_limit=256)
    assert case.faces.shape[0] == 6 * 14 * 14
    case.load(gpu)
    expected = E / (1.0 - R)
    averages = np.zeros(3)
    for batch in range(400):
        gpu.frame(16, clock_ms=16 * batch)
        if batch % 50 == 49 and batch >= 300:
            mean = gpu.read_state()[:, 0:3].view(np.float32).astype(np.float64).mean(axis=0)
            averages += mean / 2.0
    ratio = averages / expected
    assert np.all(np.abs(ratio - 1.0) < 0.02), (averages, expected)


@pytest.mark.gpu
@pytest.mark.parametrize("bounces", [1, 2, 3])
def test_cacheless_furnace_matches_finite_bounce_sums(gpu, bounces):
    case = furnace_case(bounces=bounces)
    case.load(gpu)
    receivers = np.array([[16, 8, 16, 2, 4], [9, 8, 9, 2, 4], [23, 16, 16, 1, 4]], np.int32)
    total = np.zeros((3, 3))
    count = 0
    for batch in range(32):
        tasks = vgi.tasks_for(receivers, batch * 1024)
        results = gpu.trace_tasks(tasks, 1024)
        total += results[:, 0:3].view(np.float32).astype(np.float64)
        count += 1
        # Closed world: every sample resolves.
        assert np.all(results[:, 5].view(np.float32) == 1024.0)
    mean = total.mean(axis=0) / count
    expected = E * (1.0 - R ** (bounces + 1)) / (1.0 - R)
    assert np.all(np.abs(mean - expected) / expected < 0.015), (bounces, mean, expected)


@pytest.mark.gpu
def test_fp64_reference_converges_in_the_furnace(gpu):
    # The unbiased FP64 estimate (roulette, no cache, no depth cut) of the
    # closed furnace's incident radiance is E / (1 - r).
    case = furnace_case()
    case.load(gpu)
    receivers = np.array([[16, 8, 16, 2, 4], [9, 8, 9, 2, 4], [23, 16, 16, 1, 4]], np.int32)
    mean, second, known = gpu.reference_fp64(vgi.tasks_for(receivers), 65536, seed=7)
    assert np.all(known == 65536)
    expected = E / (1.0 - R)
    assert np.all(np.abs(mean / expected - 1.0) < 0.01), mean


@pytest.mark.gpu
def test_fp64_reference_agrees_with_the_unbiased_fp32_view_estimate(gpu):
    # Both estimate the same expectation on the terrain with emitters and a
    # sun: the FP64 reference with independent samples and power-proportional
    # emitter choice, the FP32 view tier with the production sampler, the
    # light tree, depth 0 (roulette only) and no world cache. Their per-face
    # difference is within the combined standard error.
    from test_gpu_parity import terrain_case
    case = terrain_case(bounces=2)
    case.load(gpu, with_faces=False)
    rng = np.random.default_rng(3)
    faces = case.faces[rng.choice(len(case.faces), 64, replace=False)]
    m64, s64, k64 = gpu.reference_fp64(vgi.tasks_for(faces), 8192, seed=11)
    gpu.view_set_receivers(faces)
    for _ in range(64):
        gpu.view_frame(max_hits=8, depth=0, view_first=True, shared=False, invocations=32 * 64)
    est = gpu.view_read()["estimates"]
    m32 = est[:, 0:3].view(np.float32).astype(np.float64)
    n32 = est[:, 3].view(np.float32).astype(np.float64)
    q32 = est[:, 4:7].view(np.float32).astype(np.float64)
    assert n32.min() >= 2000 and k64.min() == 8192
    var = np.maximum(s64 - m64 ** 2, 0.0) / k64[:, None] + np.maximum(q32 - m32 ** 2, 0.0) / n32[:, None]
    z = (m32 - m64) / np.sqrt(var + 1e-30)
    assert np.abs(z).max() < 5.0, np.abs(z).max()
    assert abs(z.mean()) < 0.5, z.mean()
