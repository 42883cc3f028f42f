"""The far tier (vgi_far_frame) against the oracle word for word: output
cells, cell histories and statistics over frames with a still and a moving
camera, every size measure, custom direct light, the world-cache gather and
the handoff from view receivers."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import Case, assert_words_equal, run_frames, terrain_case
from test_oracle_far import floor_scene

pytestmark = pytest.mark.gpu


def unit(v):
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def far_pair(gpu, case, cameras, settings, geometry=None, state=None, index=None, frames=None):
    """Runs the far frames on the GPU and in the oracle, comparing each."""
    gpu.far_reset()
    geometry = geometry or gpu.geometry()
    params = case.params_fn(geometry)(1, 1)
    t = case.transport
    limited = 1 if min(max(t.reach, 1.0), 768.0) < 768.0 else 0
    pipe = O.Pipeline(3, limited, min(max(settings.steps, 16), 2048), 1, 1)
    custom = bool(case.lights.size and np.any(case.lights.reshape(-1, 12)[:, 9:12] != 0))
    view = gpu.view_read() if getattr(gpu, "n_view", 0) else None
    ref = O.FarTier()
    frames = frames or list(range(len(cameras)))
    stats_seen = np.zeros(8, np.uint64)
    for frame, cam in zip(frames, cameras):
        eye, forward, up, tan_half, w, h = cam
        gpu.far_frame(eye, forward, up, tan_half, w, h, settings, frame)
        shape, output, cells, stats = gpu.far_read()
        want_cells, want_output, want_stats = ref.frame(geometry, params, case.materials, case.lights, case.emitters, pipe,
                                                        (eye, forward, up, tan_half, w, h), settings, frame, custom,
                                                        receivers=None if view is None else view["receivers"],
                                                        estimates=None if view is None else view["estimates"], state=state, index=index)
        assert tuple(shape[:2]) == ref.shape
        assert_words_equal(output, want_output, f"far output, frame {frame}")
        assert_words_equal(cells, want_cells, f"far cells, frame {frame}")
        np.testing.assert_array_equal(stats, want_stats)
        stats_seen += stats
    return stats_seen


def clear_view(gpu):
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))


def test_far_floor_with_slab_and_custom_light_matches_oracle(gpu):
    coords, vox = floor_scene(slab=True)
    m = vgi.VoxelGiMaterials()
    m.set(0, vgi.MaterialTransport(diffuse=(0.6, 0.6, 0.6)))
    m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(8.0, 8.0, 8.0)))
    point = vgi.PointTransportLight((16.0, 12.0, 16.0), (2.0, 2.0, 2.0), 64.0, custom_visible=(10.0, 10.0, 10.0))
    case = Case(coords, vox, m, lights=[point], env=(0.3, 0.4, 0.5), faces=np.zeros((0, 5), np.int32))
    case.load(gpu, with_faces=False)
    clear_view(gpu)
    cams = [((16.0 + 0.5 * k, 20.0, 16.0), np.float32([0, -1, 0]), (0.0, 0.0, -1.0), 0.5, 24, 20) for k in range(8)]
    stats = far_pair(gpu, case, cams, vgi.FarTierSettings(voxel_pixels=64.0, cell=3, rate=2))
    assert stats[1] > 0 and stats[3] > 0  # traced and reprojected cells


@pytest.mark.parametrize("measure,threshold", [(0, 8.0), (1, 16.0), (2, 40.0)])
def test_far_terrain_matches_oracle(gpu, measure, threshold):
    case = terrain_case(bounces=2)
    case.load(gpu, with_faces=False)
    clear_view(gpu)
    f = unit((0.2, -1.0, 0.3))
    cams = [((48.5 + 1.5 * k, 80.25, 47.75 - k), f, (0.0, 0.0, 1.0), 0.45, 80, 64) for k in range(6)]
    settings = vgi.FarTierSettings(voxel_pixels=threshold, measure=measure, cell=2, rate=3, steps=96)
    stats = far_pair(gpu, case, cams, settings)
    assert stats[0] > 1000 and stats[1] > 0 and stats[3] > 0


def test_far_terrain_gathers_the_world_cache(gpu):
    case = terrain_case(bounces=2)
    ref = run_frames(gpu, case, 2, 8)
    clear_view(gpu)
    f = unit((0.6, -0.45, 0.7))
    cams = [((6.5, 52.25, 8.75), f, (0.0, 1.0, 0.0), 0.6, 64, 48)] * 5
    settings = vgi.FarTierSettings(voxel_pixels=64.0, cell=1, rate=1, steps=256)
    far_pair(gpu, case, cams, settings, state=ref.state, index=ref.index)


def test_far_cells_take_over_view_receiver_history(gpu):
    case = terrain_case(bounces=2)
    case.load(gpu, with_faces=False)
    f = unit((0.2, -1.0, 0.3))
    cam = ((48.5, 80.25, 47.75), f, (0.0, 0.0, 1.0), 0.45, 80, 64)
    _, faces = gpu.discover_faces(*cam)
    gpu.view_set_receivers(faces)
    for k in range(3):
        gpu.view_frame(clock_ms=10 * k)
    settings = vgi.FarTierSettings(voxel_pixels=8.0, cell=2, rate=3, steps=96)
    stats = far_pair(gpu, case, [cam], settings, frames=[100])
    assert stats[4] > 100, stats  # seeded from the receivers' estimates
    clear_view(gpu)


def test_view_receivers_take_over_far_cells(gpu):
    """The far handoff in load_shared_faces: new view receivers start from
    the far cell at their centre; the view frame then matches the oracle's
    given the same far cells."""
    case = terrain_case(bounces=2)
    case.load(gpu, with_faces=False)
    clear_view(gpu)
    f = unit((0.2, -1.0, 0.3))
    cam = ((48.5, 80.25, 47.75), f, (0.0, 0.0, 1.0), 0.45, 80, 64)
    settings = vgi.FarTierSettings(voxel_pixels=64.0, cell=2, rate=1, steps=96)
    gpu.far_reset()
    for frame in range(3):
        gpu.far_frame(*cam, settings=settings, frame=frame)
    _, _, far_cells, _ = gpu.far_read()
    _, faces = gpu.discover_faces(*cam)
    gpu.view_set_receivers(faces)
    receivers = gpu.view_read()["receivers"]
    gpu.set_far_handoff(True)
    try:
        gpu.view_frame(clock_ms=5)
    finally:
        gpu.set_far_handoff(False)
    got = gpu.view_read()
    _, _, _, stats = gpu.far_read()
    geometry = gpu.geometry()
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, np.zeros((0, 5), np.int32),
                   case.transport, case.pipe(1))
    ref.view_start(receivers, faces[:, 4])
    words, _ = O.FarTier().view_words(cam, settings, 2, False)
    words[29] = 2  # the cells' stamp: the last far frame
    ref.view_frame(clock_ms=5, far=(words, far_cells))
    for key in ("estimates", "paths", "continuations"):
        assert_words_equal(got[key], ref.view[key], f"view {key} after the far handoff")
    assert stats[5] == ref.far_stats[5] and stats[5] > 100, (stats, ref.far_stats)
    clear_view(gpu)
