"""Headless discovery's oracle (orc_discover): one primary ray per pixel of a
pinhole camera, the first hit's voxel and face. Properties on CPU: every
hit voxel is solid, nearly every hit face is an exposed face turned towards
the camera (a ray that meets an edge or corner exactly may report the other
face of the edge), and the pixel's distance places the hit on its ray."""
import numpy as np

import oracle_lib as O
import vgi

OFFSETS = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])


AIR = 256


def small_terrain():
    coords, vox = vgi.terrain(6, 4, 6, seed=5, base_height=30.0, falloff=18.0, emitters=48)
    scene = O.Scene(coords, vox)
    geometry = scene.arrays()
    params = O.params_words(1, 1, geometry[0].size // 4, 0, geometry[3], 0)
    return coords, vox, geometry, params


def dense(coords, vox):
    lo = coords.min(0) * 16
    size = (coords.max(0) - coords.min(0) + 1) * 16
    grid = np.full(size[::-1], AIR, np.uint16)  # z, y, x
    for r, (x, y, z) in enumerate(coords * 16 - lo):
        grid[z:z + 16, y:y + 16, x:x + 16] = vox[r * 4096:(r + 1) * 4096].reshape(16, 16, 16)
    return grid, lo


def camera():
    eye = np.array([6.5, 52.25, 8.75], np.float32)
    forward = np.array([0.6, -0.45, 0.7])
    forward = (forward / np.linalg.norm(forward)).astype(np.float32)
    return eye, forward, np.array([0.0, 1.0, 0.0], np.float32), 0.6


def test_discovered_hits_are_exposed_faces_towards_the_camera():
    coords, vox, geometry, params = small_terrain()
    eye, forward, up, tan_half = camera()
    w, h = 96, 64
    pixels = O.discover(geometry, params, eye, forward, up, tan_half, w, h)
    hit = pixels[..., 3] < 6
    assert hit.mean() > 0.5
    assert np.all(pixels[~hit][:, 3] == 6) and np.all(pixels[hit][:, 5] == 1)
    grid, lo = dense(coords, vox)
    p = pixels[hit]
    v = p[:, :3].view(np.int32) - lo
    assert np.all(grid[v[:, 2], v[:, 1], v[:, 0]] != AIR), "every hit voxel is solid"
    faces = O.discovered_faces(pixels)
    exposed = {tuple(r) for r in vgi.exposed_faces(coords, vox, facing=eye)}
    inside = np.array([tuple(r) in exposed for r in faces])
    assert inside.mean() > 0.99, inside.mean()
    # The hit lies on the voxel's face: its distance along the ray reaches the face's plane.
    normal = OFFSETS[p[:, 3]]
    centre = p[:, :3].view(np.int32) + 0.5 + 0.5 * normal
    distance = p[:, 6].view(np.float32)
    ys, xs = np.nonzero(hit)
    sx = (2.0 * (xs + 0.5) / w - 1.0) * tan_half * (w / h)
    sy = (1.0 - 2.0 * (ys + 0.5) / h) * tan_half
    right = np.cross(forward, up)
    right /= np.linalg.norm(right)
    dirs = forward + right * sx[:, None] + np.cross(right, forward) * sy[:, None]
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    points = eye + dirs * distance[:, None]
    plane_gap = np.abs(((points - centre) * normal).sum(1))
    assert np.median(plane_gap) < 1e-3 and np.quantile(plane_gap, 0.97) < 1e-2


def test_discovery_looking_out_of_the_scene_hits_nothing():
    coords, vox, geometry, params = small_terrain()
    eye, forward, up, tan_half = camera()
    # Looking up from above the terrain: every ray leaves the scene.
    pixels = O.discover(geometry, params, eye, np.array([0, 1, 0], np.float32), np.array([0, 0, 1], np.float32), tan_half, 8, 4)
    assert np.all(pixels[..., 3] == 6) and np.all(pixels[..., 6] == 0)
    assert O.discovered_faces(pixels).shape == (0, 5)
