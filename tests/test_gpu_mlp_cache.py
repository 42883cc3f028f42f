"""The MLP cache mode of the frame: the network's inputs, MLP-terminated
frames against the oracle given the same predictions, the plain warm-up
frames, graph replay, and what the trained network gains over the method
without it."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_mlp import random_weights, torch_forward
from test_gpu_parity import assert_words_equal, lanes_for, terrain_case

pytestmark = pytest.mark.gpu


def encode_reference(faces, bounds, material_words):
    """The 96 inputs in float64 trigonometry of the same float32 position."""
    faces = np.asarray(faces, np.int64).reshape(-1, 5)
    lo = (np.asarray(bounds[:3], np.float32) * np.float32(16.0)).astype(np.float32)
    hi = ((np.asarray(bounds[3:6], np.float32) + np.float32(1.0)) * np.float32(16.0)).astype(np.float32)
    inv = (np.float32(1.0) / np.maximum(hi - lo, np.float32(1.0))).astype(np.float32)
    axis, side = faces[:, 3] >> 1, np.where(faces[:, 3] & 1, -0.5, 0.5)
    out = np.zeros((faces.shape[0], 96), np.float64)
    for a in range(3):
        centre = faces[:, a].astype(np.float32) + np.float32(0.5) + np.where(axis == a, side, 0.0).astype(np.float32)
        x = ((centre - lo[a]).astype(np.float32) * inv[a]).astype(np.float32).astype(np.float64)
        for k in range(12):
            out[:, 24 * a + 2 * k] = np.sin(np.pi * 2.0 ** k * x)
            out[:, 24 * a + 2 * k + 1] = np.cos(np.pi * 2.0 ** k * x)
    out[np.arange(faces.shape[0]), 72 + faces[:, 3]] = 1.0
    out[:, 78:81] = np.asarray(material_words, np.float32).reshape(-1, 16)[faces[:, 4], 0:3]
    return out


def test_mlp_inputs_match_the_encoding(gpu):
    case = terrain_case()
    case.load(gpu, with_faces=False)
    faces = vgi.exposed_faces(case.coords, case.vox)
    got = gpu.mlp_encode(faces)
    want = encode_reference(faces, gpu.geometry()[3], case.materials)
    # sincospif at two frequencies, the rest by at most five doublings.
    assert np.abs(got - want).max() < 2e-5, np.abs(got - want).max()


def surface_faces(case):
    """All six faces of every solid voxel with an air cell among its 26
    neighbours: a ray that passes a voxel's edge or corner can report a face
    whose neighbour is solid (the traversal's normal is the axis of its last
    step), and the network is asked about that face like any other."""
    coords = np.asarray(case.coords, np.int64).reshape(-1, 3)
    vox = np.asarray(case.vox).reshape(-1, 16, 16, 16)  # [region][z][y][x]
    lo = coords.min(axis=0) * 16
    size = (coords.max(axis=0) + 1) * 16 - lo
    material = np.full((size[2] + 2, size[1] + 2, size[0] + 2), 256, np.int64)  # [z][y][x], air border
    for r, (cx, cy, cz) in enumerate(coords * 16 - lo):
        material[cz + 1:cz + 17, cy + 1:cy + 17, cx + 1:cx + 17] = vox[r]
    air = material == 256
    near_air = np.zeros_like(air)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                near_air |= np.roll(air, (dz, dy, dx), axis=(0, 1, 2))
    z, y, x = np.nonzero(~air & near_air)
    n = x.size
    out = np.zeros((n * 6, 5), np.int32)
    out[:, 0] = np.repeat(x - 1 + lo[0], 6)
    out[:, 1] = np.repeat(y - 1 + lo[1], 6)
    out[:, 2] = np.repeat(z - 1 + lo[2], 6)
    out[:, 3] = np.tile(np.arange(6), n)
    out[:, 4] = np.repeat(material[z, y, x], 6)
    return out


def oracle_frames(gpu, case, samples):
    geometry = gpu.geometry()
    lanes = lanes_for(case.transport, samples)
    t = case.transport
    one_hit = O.Pipeline(1, 1 if min(max(t.reach, 1.0), 768.0) < 768.0 else 0, t.path_steps, int(t.budgeted), lanes)
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                   case.pipe(lanes))
    return ref, one_hit


def assert_close_results(got, want, outliers=0.0):
    """Frame results of MLP-terminated frames (as accumulate leaves them):
    the sample counts and the receivers' direct light are exact; the
    accumulated means and second moments carry the tensor cores' summation
    order through the network (up to a few percent where a hidden value
    rounds the other way to BF16). The display words are not compared: they
    are thresholded functions of the means. Once faces reach 16 samples the
    cache answers paths, and whether it may (the binding flag) is also a
    threshold on the means, so a face can take the cache on one side and the
    network on the other: `outliers` is the share of faces allowed outside
    the tolerance."""
    got, want = np.asarray(got), np.asarray(want)
    assert_words_equal(got[:, 4:7], want[:, 4:7], "sample counts")
    assert_words_equal(got[:, 16:24], want[:, 16:24], "receiver direct light")
    cols = [0, 1, 2, 8, 9, 10]  # means, second moments
    g = np.ascontiguousarray(got[:, cols]).view(np.float32).astype(np.float64)
    w = np.ascontiguousarray(want[:, cols]).view(np.float32).astype(np.float64)
    err = np.abs(g - w)
    rel = err / np.maximum(np.abs(w), 1e-3)
    worst = np.unravel_index(np.argmax(err / (5e-2 * np.abs(w) + 1e-4)), err.shape)
    detail = (np.median(rel), rel.max(axis=0), worst, g[worst[0]], w[worst[0]])
    assert np.median(rel) < 2e-3, detail
    bad = np.any(err > 5e-2 * np.abs(w) + 1e-4, axis=1)
    assert bad.mean() <= outliers, (bad.sum(), detail)


def test_mlp_terminated_frames_match_oracle(gpu):
    case = terrain_case(bounces=2)
    case.load(gpu)
    every_face = surface_faces(case)
    inputs = gpu.mlp_encode(every_face)
    gpu.mlp_set_weights(random_weights(3))
    gpu.set_mlp_cache(True, warm_frames=0, samples=4096, steps_per_frame=1, lr=1e-3)
    try:
        ref, one_hit = oracle_frames(gpu, case, 8)
        for f in range(3):
            weights = gpu.mlp_get_weights()  # this frame's network: trained by the frames before
            prediction = torch_forward(weights, inputs)
            gpu.frame(8, clock_ms=16 * f)
            counts = ref.frame(8, clock_ms=16 * f, predicted=(every_face[:, :4], prediction), pipe=one_hit)
            assert counts["predicted_misses"] == 0, counts["last_miss"]
            # Frame 0 has no cache answers: every face within the tolerance.
            assert_close_results(gpu.read_results(), ref.results, outliers=0.0 if f == 0 else 0.005)
            stats = gpu.mlp_stats()
            assert stats["error"] == 0 and stats["terminating"] == 1 and stats["queries"] > 0
            assert stats["steps"] == f + 1 and stats["frames"] == f + 1
        assert not np.array_equal(gpu.mlp_get_weights(), random_weights(3))  # online training moved the weights
    finally:
        gpu.set_mlp_cache(False)


def test_mlp_warm_up_frames_trace_plainly(gpu):
    case = terrain_case(bounces=2)
    case.load(gpu)
    gpu.mlp_set_weights(random_weights(4))
    gpu.set_mlp_cache(True, warm_frames=2, samples=4096, steps_per_frame=2, lr=1e-3)
    try:
        ref, one_hit = oracle_frames(gpu, case, 8)
        for f in range(2):
            assert gpu.mlp_stats()["terminating"] == 0
            gpu.frame(8, clock_ms=16 * f)
            ref.frame(8, clock_ms=16 * f)
            assert_words_equal(gpu.read_results(), ref.results, "warm-up frame results")
            assert_words_equal(gpu.read_state(), ref.state, "warm-up frame state")
        stats = gpu.mlp_stats()
        assert stats["steps"] == 4 and stats["terminating"] == 1 and stats["error"] == 0 and np.isfinite(stats["loss"])
        every_face = surface_faces(case)
        prediction = torch_forward(gpu.mlp_get_weights(), gpu.mlp_encode(every_face))
        gpu.frame(8, clock_ms=32)
        counts = ref.frame(8, clock_ms=32, predicted=(every_face[:, :4], prediction), pipe=one_hit)
        assert counts["predicted_misses"] == 0, counts["last_miss"]
        assert_close_results(gpu.read_results(), ref.results, outliers=0.005)
    finally:
        gpu.set_mlp_cache(False)


def test_mlp_graph_frames_match_direct_frames(gpu):
    """Frames replayed from a captured graph (training included) leave the
    same results and weights as frames run directly."""
    outs = []
    for graph in (False, True):
        case = terrain_case(bounces=2)
        case.load(gpu)
        gpu.mlp_set_weights(random_weights(5))
        gpu.set_graph(graph)
        gpu.set_mlp_cache(True, warm_frames=1, samples=4096, steps_per_frame=1, lr=1e-3)
        try:
            for f in range(5):
                gpu.frame(8, clock_ms=16 * f)
            outs.append((gpu.read_results(), gpu.mlp_get_weights(), gpu.mlp_stats()))
        finally:
            gpu.set_mlp_cache(False)
            gpu.set_graph(False)
    (r0, w0, s0), (r1, w1, s1) = outs
    assert s0["steps"] == s1["steps"] == 5 and s0["error"] == s1["error"] == 0
    # The frame's queries are queued by atomic appends, so the training
    # rows drawn from the queue differ between runs; Adam turns a gradient
    # near 0 into a step of up to lr either way, and the next frames train on
    # what the moved network predicted. The two runs stay close as a whole.
    rel = np.linalg.norm(w0 - w1) / np.linalg.norm(w0)
    assert rel < 2e-2, rel
    g, w = r0[:, :3].view(np.float32), r1[:, :3].view(np.float32)
    assert np.median(np.abs(g - w) / np.maximum(np.abs(w), 1e-3)) < 1e-2


def relmse(estimate, reference):
    w = np.array([0.2126, 0.7152, 0.0722])
    le, lr = estimate @ w, reference @ w
    return float(np.mean((le - lr) ** 2 / (lr ** 2 + 0.01)))


def test_trained_network_gains_over_the_method_without_it(gpu):
    """One diffuse hit per path, 40 frames of 8 samples: paths whose first
    hit the world cache cannot answer end with terminal emission in the
    plain method, and with the network's prediction in the MLP cache mode.
    Against the FP64 converged reference the network removes most of the
    plain method's missing-bounce bias."""
    case = terrain_case(bounces=1)
    case.load(gpu)
    mean, _, known = gpu.reference_fp64(vgi.tasks_for(case.faces), 1024, seed=3)
    sel = known > 0
    errors = {}
    for mode in ("plain", "mlp"):
        case.load(gpu)
        if mode == "mlp":
            gpu.mlp_set_weights(random_weights(6) * 0.5)
            gpu.set_mlp_cache(True, warm_frames=8, samples=65536, steps_per_frame=16, lr=1e-2)
        try:
            for f in range(40):
                gpu.frame(8, clock_ms=16 * f)
            est = gpu.read_state()[:, 0:3].view(np.float32).astype(np.float64)
            errors[mode] = relmse(est[sel], mean[sel])
            if mode == "mlp":
                assert gpu.mlp_stats()["error"] == 0
        finally:
            gpu.set_mlp_cache(False)
    print("relMSE vs FP64:", errors)
    assert errors["mlp"] < 0.7 * errors["plain"], errors


def test_mlp_schedule_refuses_bad_settings_caps_counts_and_cycles_batches(gpu):
    """vgi_set_mlp_schedule: a history share outside [0, 1] or more than
    2^22 rows a step is refused. With share 0.5 at 2 samples a frame, the
    k-th frame the network answers caps every face's count at max(32, k);
    faces traced every frame sit at the cap. Steps of 4,096 rows over a
    frame's 4,096 samples (every step a full pass) take the frame's steps
    without a tensor-core error."""
    case = terrain_case(bounces=2)
    case.load(gpu)
    gpu.mlp_set_weights(random_weights(7))
    for bad in ((0, -0.5), (0, 1.5), (1 << 23, 0.0)):
        with pytest.raises(vgi.VgiError) as err:
            gpu.set_mlp_schedule(*bad)
        assert err.value.status == vgi.ERR_INVALID
    spp, warm, frames = 2, 2, 40
    gpu.set_mlp_cache(True, warm_frames=warm, samples=4096, steps_per_frame=2, lr=1e-3)
    gpu.set_mlp_schedule(4096, 0.5)
    try:
        for f in range(warm + frames):
            gpu.frame(spp, clock_ms=16 * f)
            k = f - warm + 1
            if k in (1, 20, 33, frames):
                cap = max(32, int(np.ceil(0.5 * spp * k)))
                counts = gpu.read_state()[:, 5] & 0x7fffffff
                assert counts.max() <= cap, (k, counts.max(), cap)
        assert (counts == frames).mean() > 0.5, np.bincount(counts)[-8:]
        st = gpu.mlp_stats()
        assert st["error"] == 0 and st["steps"] == 2 * (warm + frames) and np.isfinite(st["loss"])
        assert np.isfinite(gpu.mlp_get_weights()).all()
    finally:
        gpu.set_mlp_cache(False)
        gpu.set_mlp_schedule(0, 0.0)
