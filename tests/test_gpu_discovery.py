"""Headless discovery (vgi_discover_faces): the GPU's per-pixel first hits
word for word against the oracle, its face list equal to the distinct
faces of the oracle's pixels, and the discovered faces driving frames that
match the oracle's."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal, run_frames, terrain_case

pytestmark = pytest.mark.gpu

CAMERAS = [
    ((6.5, 52.25, 8.75), (0.6, -0.45, 0.7), (0.0, 1.0, 0.0), 0.6, 96, 64),   # inside the scene, low and oblique
    ((48.5, 70.25, 47.75), (0.2, -1.0, 0.3), (0.0, 0.0, 1.0), 0.45, 80, 80),  # above the scene's box, looking down
    ((-20.0, 30.5, 40.0), (1.0, 0.02, 0.0), (0.0, 1.0, 0.0), 0.8, 33, 17),    # outside the box, odd sizes
]


def unit(v):
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


@pytest.mark.parametrize("eye,forward,up,tan_half,w,h", CAMERAS)
def test_discovery_matches_oracle(gpu, eye, forward, up, tan_half, w, h):
    case = terrain_case()
    case.load(gpu, with_faces=False)
    geometry = gpu.geometry()
    params = case.params_fn(geometry)(1, 1)
    f = unit(forward)
    pixels, faces = gpu.discover_faces(eye, f, up, tan_half, w, h)
    want = O.discover(geometry, params, np.float32(eye), f, np.float32(up), tan_half, w, h)
    assert_words_equal(pixels, want, "pixel records")
    assert (want[..., 3] < 6).any()
    np.testing.assert_array_equal(faces, O.discovered_faces(want))


def test_discovery_reports_a_short_list(gpu):
    case = terrain_case()
    case.load(gpu, with_faces=False)
    eye, forward, up, tan_half, w, h = CAMERAS[0]
    _, faces = gpu.discover_faces(eye, unit(forward), up, tan_half, w, h)
    with pytest.raises(vgi.VgiError) as err:
        gpu.discover_faces(eye, unit(forward), up, tan_half, w, h, capacity=len(faces) - 1)
    assert err.value.status == vgi.ERR_CAPACITY
    # Enough room: the same list.
    _, again = gpu.discover_faces(eye, unit(forward), up, tan_half, w, h, capacity=len(faces))
    np.testing.assert_array_equal(again, faces)


def test_discovered_faces_drive_frames(gpu):
    terrain_case(bounces=2).load(gpu, with_faces=False)
    eye, forward, up, tan_half, w, h = CAMERAS[1]
    _, faces = gpu.discover_faces(eye, unit(forward), up, tan_half, w, h)
    case = terrain_case(bounces=2)
    case.faces = faces
    ref = run_frames(gpu, case, 3, 4)
    assert_words_equal(gpu.read_results(), ref.results, "frame results")
