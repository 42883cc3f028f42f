"""The cave workload at test scale (vgi_scene_cave: worm tunnels under a
roof with skylights, green and orange emitters), split into uneven chunks
traced as batched scenes. One chunk's frames against the oracle word for
word, and the batched chunks against each chunk's own frames."""
import numpy as np
import pytest

import vgi
from test_gpu_parity import Case, assert_words_equal, run_frames

pytestmark = pytest.mark.gpu

CHUNKS = [(0, 2), (2, 5), (5, 6), (6, 8)]  # region x ranges: uneven chunks


def cave_chunks(seed=3):
    coords, vox = vgi.cave(8, 4, 8, seed=seed, worms=12, steps=200, radius_min=3.0, radius_max=8.0, roof=6, skylights=4,
                           skylight_radius=4.0, emitters=40)
    m = vgi.VoxelGiMaterials()
    rng = np.random.default_rng(seed)
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    m.set(8, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(0.5, 4.0, 1.0)))
    m.set(9, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(6.0, 2.0, 0.3)))
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0))
    cases = []
    for lo, hi in CHUNKS:
        keep = np.nonzero((coords[:, 0] >= lo) & (coords[:, 0] < hi))[0]
        c = coords[keep]
        v = vox.reshape(-1, 4096)[keep].reshape(-1)
        faces = vgi.exposed_faces(c, v)[::5].copy()
        cases.append(Case(c, v, m, lights=[sun], n_directional=1, env=(0.3, 0.4, 0.5),
                          transport=vgi.TransportSettings(bounces=2), faces=faces))
    return cases


@pytest.fixture(scope="module")
def chunk_tracers():
    ts = [vgi.GpuTracer(0) for _ in CHUNKS]
    yield ts
    for t in ts:
        t.close()


def test_cave_chunk_frames_match_oracle(gpu):
    case = cave_chunks()[1]
    ref = run_frames(gpu, case, 3, 4)
    assert_words_equal(gpu.read_results(), ref.results, "cave chunk results")
    assert_words_equal(gpu.read_state(), ref.state, "cave chunk state")
    lit = ref.results.view(np.float32)[:, 0:3].sum(1) > 0
    assert lit.mean() > 0.5


def test_batched_cave_chunks_equal_their_own_frames(chunk_tracers):
    cases = cave_chunks()
    want = []
    for t, case in zip(chunk_tracers, cases):
        case.load(t)
        for f in range(4):
            t.frame(8, clock_ms=16 * f)
        want.append((t.read_results(), t.read_state()))
    for t, case in zip(chunk_tracers, cases):
        case.load(t)
    batch = vgi.GpuBatch(chunk_tracers)
    try:
        batch.set_graph(True)
        for f in range(4):
            batch.frame(8, clock_ms=16 * f)
        batch.sync()
        for k, (t, (results, state)) in enumerate(zip(chunk_tracers, want)):
            assert_words_equal(t.read_results(), results, f"chunk {k} results")
            assert_words_equal(t.read_state(), state, f"chunk {k} state")
    finally:
        batch.close()
