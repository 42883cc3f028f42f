"""Parity at the benchmarked size: the 512x256x512 fBm terrain (16,384
regions) with its 1,371,468 faces turned towards the cube-map camera at
(256, 200, 256), 8 paths a face, 2 diffuse hits via the world cache, a sun
and 256 emissive voxels: the workload bench.py times.

The scene is made by the oracle library (the seeded generator and the
model records, no libvgi), uploaded through the C ABI, and then:
- the GPU's packed geometry equals the oracle's packing of the same voxels
  (canonical form: directory lookups, headers, brick tables and cells);
- three whole frames (two cold, one with every face cached) give the same
  results and resident state on every face, word for word;
- a seeded 256-face sample re-traced by vgi_trace_tasks against the warm
  state equals the oracle's trace of the same tasks.
The oracle runs on all host cores; the test takes some 30 s.
"""
import os

import numpy as np
import pytest

import oracle_lib as O
import vgi

pytestmark = pytest.mark.gpu

EYE = (256.0, 200.0, 256.0)
SPP = 8
BOUNCES = 2


def bench_scene():
    coords, vox = O.terrain(32, 16, 32, seed=2, octaves=4, period=64.0, base_height=128.0, falloff=400.0, emitters=256)
    rng = np.random.default_rng(2)
    entries = [((0.45, 0.45, 0.45), (0.0, 0.0, 0.0))] * 256
    for k in range(8):
        entries[k] = (tuple(rng.uniform(0.2, 0.8, 3)), (0.0, 0.0, 0.0))
    for k in range(248):
        r = float(rng.uniform(1.0, 10.0))
        entries[8 + k] = ((0.5, 0.5, 0.5), (r, r, r))
    words = O.material_words(entries)
    sun = O.directional_light_words((0.4, 0.8, 0.3), (3.0, 3.0, 3.0))
    faces = O.exposed_faces(coords, vox, facing=EYE)
    return coords, vox, words, sun, faces


def words_equal(got, want, what):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    bad = np.argwhere(got != want)
    if bad.size:
        r = bad[0][0]
        raise AssertionError(f"{what}: {len(bad)} words differ; first at {tuple(bad[0])}: got {got[r]} want {want[r]}")


def test_bench_terrain_matches_oracle():
    coords, vox, words, sun, faces = bench_scene()
    assert faces.shape[0] == 1371468
    ref_scene = O.Scene(coords, vox, top_mode=0)
    geometry = ref_scene.arrays()
    emitters, n_emit, total = O.emitters(coords, vox, words)
    d = geometry[0]

    def params(n, samples):
        return O.params_words(n, samples, d.size // 4, 1, geometry[3], 1, (0, 0, 0), total, n_emit)

    transport = vgi.TransportSettings(bounces=BOUNCES, path_steps=2048)
    g = vgi.GpuTracer(0)
    try:
        g.upload_regions(coords, vox)
        g.set_materials(words)
        g.set_lights(sun, 1)
        g.set_environment((0.0, 0.0, 0.0))
        g.build_emitters()
        g.set_transport(transport)
        g.set_faces(faces)
        gd, gh, gcl, gbounds = g.geometry()
        assert (gbounds == geometry[3]).all()
        words_equal(O.canonical(gd, gh, gcl, coords), O.canonical(*geometry[:3], coords), "canonical geometry")

        threads = os.cpu_count() or 0
        ref = O.Frames(geometry, params, words, sun, emitters, faces, O.transport_settings(bounces=BOUNCES, path_steps=2048),
                       O.Pipeline(BOUNCES, 0, 2048, 0, SPP), threads=threads)
        for f in range(3):
            g.frame(SPP, clock_ms=16 * f)
            cnt = ref.frame(SPP, clock_ms=16 * f)
        assert cnt["cache_hits"] > 0
        words_equal(g.read_results(), ref.results, "frame results")
        state = g.read_state()
        words_equal(state, ref.state, "resident state")

        rng = np.random.default_rng(7)
        sample = np.sort(rng.choice(faces.shape[0], size=256, replace=False))
        tasks = vgi.tasks_for(faces[sample])
        tasks[:, 4] = state[sample, 6]
        want, wcnt = O.trace_faces(geometry, params(sample.size, SPP), words, sun, emitters, tasks, O.Pipeline(BOUNCES, 0, 2048, 0, SPP),
                                   ref.state, ref.index, threads)
        got = g.trace_tasks(tasks, SPP)
        words_equal(got, want, "re-traced sample")
        assert wcnt["cache_hits"] > 0
    finally:
        g.close()
