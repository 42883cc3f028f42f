"""Reconstruction and presentation of the view receivers on the GPU against
the oracle word for word: reconstruct_view + publish_view over receivers
found by discovery, traced by view frames and placed in screen tiles by
their witness pixels, then corner_irradiance per pixel."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import Case, assert_words_equal, terrain_case
from test_oracle_far import floor_scene

pytestmark = pytest.mark.gpu


def unit(v):
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def prepare(gpu, case, cam, frames=3, grid=4):
    case.load(gpu, with_faces=False)
    pixels, faces = gpu.discover_faces(*cam)
    gpu.view_set_receivers(faces)
    for k in range(frames):
        gpu.view_frame(clock_ms=10 * k)
    w, h = cam[4], cam[5]
    gx, gy = max(w // grid, 1), max(h // grid, 1)
    tiles = vgi.witness_tiles(pixels, faces, gx, gy)
    tx, ty = (gx + 1) // 2, (gy + 1) // 2
    gpu.view_set_tiles(tiles, tx, ty)
    return faces, tiles, tx, ty


def reconstruct_pair(gpu, case, tiles, tx, ty, display):
    before = gpu.view_read()
    gpu.view_reconstruct(*display)
    after = gpu.view_read()
    published, stats = gpu.view_read_published()
    geometry = gpu.geometry()
    params = case.params_fn(geometry)(1, 1)
    custom = bool(case.lights.size and np.any(case.lights.reshape(-1, 12)[:, 9:12] != 0))
    want_est, want_pub, want_stats = O.reconstruct(geometry, params, case.materials, case.lights, case.emitters, case.pipe(1),
                                                   before["receivers"], before["estimates"], before["continuations"], tiles, tx, ty,
                                                   display, custom)
    assert_words_equal(after["estimates"], want_est, "estimates after reconstruction")
    assert_words_equal(published, want_pub, "published pixels")
    np.testing.assert_array_equal(stats, want_stats)
    return after, published


def test_reconstruction_and_presentation_match_oracle_on_terrain(gpu):
    case = terrain_case(bounces=2)
    cam = ((48.5, 80.25, 47.75), unit((0.2, -1.0, 0.3)), (0.0, 0.0, 1.0), 0.45, 96, 72)
    faces, tiles, tx, ty = prepare(gpu, case, cam)
    assert (tiles != 0xFFFFFFFF).all()
    after, published = reconstruct_pair(gpu, case, tiles, tx, ty, (0.031, 1.0, 1.0))
    shown = after["estimates"].view(np.float32)[:, 8:12]
    assert np.all(shown[:, 3] == 1.0)
    # A second pass blends the shown value over time.
    gpu.view_frame(clock_ms=40)
    reconstruct_pair(gpu, case, tiles, tx, ty, (0.031, 1.0, 0.25))
    published, _ = gpu.view_read_published()
    geometry = gpu.geometry()
    params = case.params_fn(geometry)(1, 1)
    for corners in (True, False):
        image = gpu.view_present(*cam, corners=corners)
        want = O.present(geometry, params, published, *cam, corners=corners)
        assert_words_equal(image.view(np.uint32), want.view(np.uint32), f"presented image, corners={corners}")
    assert (image[..., 3] > 0).mean() > 0.5
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))


def test_publish_adds_custom_direct_light(gpu):
    coords, vox = floor_scene(slab=True)
    m = vgi.VoxelGiMaterials()
    m.set(0, vgi.MaterialTransport(diffuse=(0.6, 0.6, 0.6)))
    m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(8.0, 8.0, 8.0)))
    point = vgi.PointTransportLight((16.0, 12.0, 16.0), (2.0, 2.0, 2.0), 64.0, custom_visible=(10.0, 10.0, 10.0))
    case = Case(coords, vox, m, lights=[point], env=(0.3, 0.4, 0.5), faces=np.zeros((0, 5), np.int32))
    cam = ((16.0, 20.0, 16.0), np.float32([0, -1, 0]), (0.0, 0.0, -1.0), 0.5, 48, 40)
    faces, tiles, tx, ty = prepare(gpu, case, cam, frames=2)
    after, published = reconstruct_pair(gpu, case, tiles, tx, ty, (0.031, 1.0, 1.0))
    irradiance = published.view(np.float32)[:, 4:7]
    shown = after["estimates"].view(np.float32)[:, 8:11]
    lit = published[:, 3] == 2
    assert lit.any() and np.all(irradiance[lit] >= shown[lit])
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))
