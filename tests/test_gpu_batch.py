"""Batched scenes (vgi_batch_*): several contexts traced together, each
stage's traversal one launch over the rays of all scenes. Every scene's
results and state must be bit-identical to its own frames."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal, terrain_case

pytestmark = pytest.mark.gpu

SCENES = [dict(seed=5, n=(6, 4, 6), emitters=48), dict(seed=7, n=(3, 2, 4), emitters=8), dict(seed=9, n=(8, 4, 3), emitters=24),
          dict(seed=11, n=(2, 2, 2), emitters=4)]


def scenes(**transport):
    return [terrain_case(bounces=2, **s, **transport) for s in SCENES]


@pytest.fixture(scope="module")
def tracers():
    ts = [vgi.GpuTracer(0) for _ in SCENES]
    yield ts
    for t in ts:
        t.close()


def own_frames(tracers, cases, frames, samples):
    out = []
    for t, case in zip(tracers, cases):
        case.load(t)
        for f in range(frames):
            t.frame(samples, clock_ms=16 * f)
        out.append((t.read_results(), t.read_state()))
    return out


@pytest.mark.parametrize("graph", [False, True])
def test_batched_frames_equal_each_scenes_own_frames(tracers, graph):
    cases = scenes()
    want = own_frames(tracers, cases, 5, 8)
    for t, case in zip(tracers, cases):
        case.load(t)
    batch = vgi.GpuBatch(tracers)
    try:
        batch.set_graph(graph)
        for f in range(5):
            batch.frame(8, clock_ms=16 * f)
        batch.sync()
        for k, (t, (results, state)) in enumerate(zip(tracers, want)):
            assert_words_equal(t.read_results(), results, f"scene {k} results")
            assert_words_equal(t.read_state(), state, f"scene {k} state")
    finally:
        batch.close()


def test_batch_autotune_keeps_state_and_frames(tracers):
    cases = scenes()
    want = own_frames(tracers, cases, 3, 8)
    for t, case in zip(tracers, cases):
        case.load(t)
    batch = vgi.GpuBatch(tracers)
    try:
        before = [t.read_state() for t in tracers]
        choice = batch.autotune(8)
        assert choice["refill_min"] in (4, 8, 12, 16) and choice["blocks"] > 0 and choice["trace_ms"] > 0
        for t, state in zip(tracers, before):
            assert_words_equal(t.read_state(), state, "state after autotune")
        for f in range(3):
            batch.frame(8, clock_ms=16 * f)
        batch.sync()
        for k, (t, (results, state)) in enumerate(zip(tracers, want)):
            assert_words_equal(t.read_results(), results, f"scene {k} results after autotune")
    finally:
        batch.close()


def test_batch_rejects_mixed_transport(tracers):
    cases = scenes()
    for t, case in zip(tracers, cases):
        case.load(t)
    tracers[1].set_transport(vgi.TransportSettings(bounces=3))
    batch = vgi.GpuBatch(tracers)
    try:
        with pytest.raises(vgi.VgiError, match="share bounces"):
            batch.frame(8)
    finally:
        batch.close()
        tracers[1].set_transport(cases[1].transport)


def edit_stream(case, rng, mean=4.0):
    """One frame's edits for a scene, as the batched workload makes them:
    a Poisson(mean) number (1..512) of spheres of radius 1-5 at random
    surface voxels, carving air or placing an albedo material, inside the
    scene; one retention event per sphere over its box."""
    from test_gpu_parity import encode_events

    size = (case.coords.max(0) + 1) * 16
    k = int(np.clip(rng.poisson(mean), 1, 512))
    edits, events = [], []
    for row in case.faces[rng.integers(0, len(case.faces), k)]:
        c = row[:3].astype(np.int64)
        r = int(rng.integers(1, 6))
        value = 256 if rng.random() < 0.5 else int(rng.integers(0, 8))
        for dz in range(-r, r + 1):
            for dy in range(-r, r + 1):
                for dx in range(-r, r + 1):
                    p = c + (dx, dy, dz)
                    if dx * dx + dy * dy + dz * dz <= r * r and np.all(p >= 0) and np.all(p < size):
                        edits.append((*p, value))
        lo, hi = np.maximum(c - r, 0), np.minimum(c + r, size - 1)
        events.append((lo, hi, [(lo, hi, 40.0, 3)]))
    words, n = encode_events(events)
    return np.array(edits, np.int32), words, n


def test_batched_frames_with_edit_streams_equal_own_frames(tracers):
    cases = scenes(measured_retention=1.0)
    rng = np.random.default_rng(21)
    streams = [[edit_stream(case, rng) for _ in range(5)] for case in cases]
    want = []
    for t, case, stream in zip(tracers, cases, streams):
        case.load(t)
        for f, (edits, words, n) in enumerate(stream):
            t.edit_voxels(edits)
            t.apply_events(words, n)
            t.frame(8, clock_ms=16 * f)
        want.append((t.read_results(), t.read_state(), t.geometry()))
    for t, case in zip(tracers, cases):
        case.load(t)
    batch = vgi.GpuBatch(tracers)
    try:
        batch.set_graph(True)  # edits between frames must drop or keep the captured graph correctly
        for f in range(5):
            for t, stream in zip(tracers, streams):
                edits, words, n = stream[f]
                t.edit_voxels(edits)
                t.apply_events(words, n)
            batch.frame(8, clock_ms=16 * f)
        batch.sync()
        for k, (t, (results, state, geometry)) in enumerate(zip(tracers, want)):
            # The packing's cell offsets depend on the context's history; the
            # canonical form (per region, independent of layout) must agree.
            d, h, cl, _ = t.geometry()
            wd, wh, wcl, _ = geometry
            coords = cases[k].coords
            assert_words_equal(O.canonical(d, h, cl, coords), O.canonical(wd, wh, wcl, coords), f"scene {k} geometry")
            assert_words_equal(t.read_results(), results, f"scene {k} results")
            assert_words_equal(t.read_state(), state, f"scene {k} state")
    finally:
        batch.close()


def _mlp_frames(tracers, cases, weights, batched, graph, frames=4):
    for t, case, w in zip(tracers, cases, weights):
        case.load(t)
        t.mlp_set_weights(w)
        t.set_mlp_cache(True, warm_frames=1, samples=4096, steps_per_frame=2, lr=1e-2)
    batch = vgi.GpuBatch(tracers) if batched else None
    try:
        if batch:
            batch.set_graph(graph)
        for f in range(frames):
            # Training's gradient sums vary in their last bits between runs,
            # so every frame starts from the same weights in both runs.
            for t, w in zip(tracers, weights):
                t.mlp_set_weights(w)
            if batch:
                batch.frame(8, clock_ms=16 * f)
            else:
                for t in tracers:
                    t.frame(8, clock_ms=16 * f)
        if batch:
            batch.sync()
        out = [(t.read_results(), t.read_state(), t.mlp_stats()) for t in tracers]
    finally:
        if batch:
            batch.close()
        for t in tracers:
            t.set_mlp_cache(False)
    return out


@pytest.mark.parametrize("graph", [False, True])
def test_batched_mlp_frames_equal_each_scenes_own_frames(tracers, graph):
    """Scenes in the MLP cache mode, batched: after a plain warm-up frame,
    every scene's uncached first hits take its own network's prediction in
    one query launch over all scenes, then each scene trains on its own
    stream. Every frame's results and state equal the scene's own frames."""
    cases = scenes()
    rng = np.random.default_rng(12)
    weights = [np.concatenate([(rng.normal(0.0, 1.0 / np.sqrt(i), size=(i, o)) * 0.5).astype(np.float32).reshape(-1)
                               for i, o in vgi.GpuTracer.MLP_LAYERS]) for _ in cases]
    want = _mlp_frames(tracers, cases, weights, batched=False, graph=False)
    got = _mlp_frames(tracers, cases, weights, batched=True, graph=graph)
    for k, ((r, st, stats), (wr, wst, wstats)) in enumerate(zip(got, want)):
        assert wstats["queries"] > 0, "the network ended some paths"
        assert stats["queries"] == wstats["queries"], (k, stats, wstats)
        assert_words_equal(r, wr, f"scene {k} results")
        assert_words_equal(st, wst, f"scene {k} state")
