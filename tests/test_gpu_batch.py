"""Batched scenes (vgi_batch_*): several contexts traced together, each
stage's traversal one launch over the rays of all scenes. Every scene's
results and state must be bit-identical to its own frames."""
import numpy as np
import pytest

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
