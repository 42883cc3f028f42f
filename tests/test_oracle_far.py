"""The far tier's oracle (orc_far_frame with the host side restated in
oracle_lib.FarTier) against the behaviour the reference's far-tier tests
state (src/gpu/view/pixel_tests.rs): a still camera adds one sample per cell
per frame, every cell visits each of its pixels, a cell's path index
advances by one per traced path, a one-cell pan keeps the history, and the
transport reach bounds what a cell sees."""
import numpy as np

import oracle_lib as O
import vgi

AIR = 256


def f16(bits):
    return np.asarray(bits, np.uint16).view(np.float16).astype(np.float32)


def floor_scene(slab=True):
    """A 32 x 32 floor of material 0 at y = 0 (regions 0..1 in x and z), and
    an emissive slab of material 1 at y = 24 over its middle."""
    coords = np.array([[x, y, z] for z in range(2) for y in range(2) for x in range(2)], np.int32)
    vox = np.full(len(coords) * 4096, AIR, np.uint16)
    for r, (x, y, z) in enumerate(coords):
        page = vox[r * 4096:(r + 1) * 4096].reshape(16, 16, 16)  # z, y, x
        if y == 0:
            page[:, 0, :] = 0
        if slab and y == 1:
            page[4:12, 8, 4:12] = 1 if (x, z) != (5, 5) else 0
    return coords, vox


class Scene:
    def __init__(self, slab=True, emission=(8.0, 8.0, 8.0), env=(0.3, 0.4, 0.5), lights=(), reach=768.0):
        self.coords, self.vox = floor_scene(slab)
        m = vgi.VoxelGiMaterials()
        m.set(0, vgi.MaterialTransport(diffuse=(0.6, 0.6, 0.6)))
        m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=emission))
        self.materials = m.words()
        self.lights = np.concatenate([l.words() for l in lights]) if len(lights) else np.zeros(0, np.float32)
        self.custom = any(np.any(l.custom_visible) for l in lights) if len(lights) else False
        self.emitters, self.n_emit, self.total = vgi.host_emitters(self.coords, self.vox, self.materials)
        self.geometry = O.Scene(self.coords, self.vox).arrays()
        self.params = O.params_words(1, 1, self.geometry[0].size // 4, len(self.lights) // 12, self.geometry[3], 0, env, self.total,
                                     self.n_emit, reach)
        self.reach = reach

    def pipe(self, settings):
        return O.Pipeline(3, 1 if self.reach < 768.0 else 0, min(max(settings.steps, 16), 2048), 1, 1)


def top_camera(shift=0.0, w=16, h=16):
    """Looking straight down at the floor from y = 20: a voxel of the floor
    is 16 / 19 of a pixel wide."""
    eye = (16.0 + shift, 20.0, 16.0)
    return (eye, np.float32([0.0, -1.0, 0.0]), (0.0, 0.0, -1.0), 0.5, w, h)


def run(scene, settings, frames, camera=top_camera, far=None):
    far = far or O.FarTier()
    out = []
    for f in range(frames):
        cells, output, stats = far.frame(scene.geometry, scene.params, scene.materials, scene.lights, scene.emitters, scene.pipe(settings),
                                         camera(f) if callable(camera) else camera, settings, f, scene.custom)
        out.append((cells.copy(), output.copy(), stats.copy()))
    return far, out


def counts(output, n):
    c = output[16:].reshape(-1, 4)[:n]
    return f16(c[:, 1] >> 16)


def test_still_camera_adds_a_sample_per_frame_and_pan_keeps_history():
    scene = Scene(slab=False)
    settings = vgi.FarTierSettings(voxel_pixels=64.0, cell=2, rate=1)
    far, frames = run(scene, settings, 6, lambda f: top_camera())
    n = 64
    for f, (cells, output, stats) in enumerate(frames):
        assert list(output[8:12]) == [8, 8, 2, 1] and output[15] == f
        c = output[16:].reshape(-1, 4)
        assert np.all(c[:, 2] & 7 == 2), "owned top faces"
        assert np.all(c[:, 2] >> 3 == f), "stamped with this frame"
        assert np.allclose(counts(output, n), f + 1, atol=0.01), (f, counts(output, n))
        assert np.all(f16(c[:, 0] & 0xFFFF) > 0.0), "the floor sees the sky"
        assert stats[0] == n and stats[1] == n
    # A pan by one voxel, under one cell: the history follows the world point.
    cells, output, stats = far.frame(scene.geometry, scene.params, scene.materials, scene.lights, scene.emitters, scene.pipe(settings),
                                     top_camera(1.0), settings, 6, False)
    kept = int((counts(output, n) > 1.0).sum())
    assert kept >= 48, kept
    assert stats[3] == kept


def test_cells_visit_every_pixel_and_index_paths_in_order():
    scene = Scene(slab=False)
    settings = vgi.FarTierSettings(voxel_pixels=64.0, cell=3, rate=4)
    far, frames = run(scene, settings, 36, lambda f: top_camera(w=16, h=16))
    width = 6  # ceil(16 / 3)
    interior = [i for i in range(36) if i % width < width - 1 and i // width < width - 1]
    visited = {i: set() for i in interior}
    sequences = {i: [] for i in interior}
    for f, (cells, output, stats) in enumerate(frames):
        assert np.all(counts(output, 36)[interior] > 0.0)
        for i in interior:
            x, z = cells[i, 4:7:2].view(np.float32)
            visited[i].add((round((x - 8.0 + 4.0) * 2), round((z - 8.0 + 4.0) * 2)))
            sequences[i].append(int(cells[i, 8]))
    for i in interior:
        assert len(visited[i]) == 9, (i, visited[i])
        seq = sequences[i]
        assert all(b - a in (0, 1) for a, b in zip(seq, seq[1:])), seq
        # Four warm-up paths, then one frame in four: 8 or 9 more in 32 frames.
        assert seq[-1] in (12, 13), seq


def test_far_tier_honours_transport_reach():
    settings = vgi.FarTierSettings(voxel_pixels=64.0, cell=3, rate=1)

    def light(reach):
        scene = Scene(slab=True, env=(0.0, 0.0, 0.0), reach=reach)
        _, frames = run(scene, settings, 4, lambda f: top_camera(w=16, h=16))
        output = frames[-1][1]
        middle = 2 * 6 + 2
        return float(f16(output[16 + middle * 4] & 0xFFFF))

    assert light(768.0) > 0.01
    assert light(16.0) == 0.0


def test_custom_light_is_shown_outside_the_history():
    point = vgi.PointTransportLight((16.0, 12.0, 16.0), (0.0, 0.0, 0.0), 64.0, custom_visible=(100.0, 100.0, 100.0))
    scene = Scene(slab=False, lights=[point])
    settings = vgi.FarTierSettings(voxel_pixels=64.0, cell=3, rate=4)
    far, frames = run(scene, settings, 8, lambda f: top_camera(w=16, h=16))
    interior = [i for i in range(36) if i % 6 < 5 and i // 6 < 5]
    for cells, output, stats in frames:
        shown = f16(output[16:].reshape(-1, 4)[:, 0] & 0xFFFF)
        mean = cells[:, 0].view(np.float32)
        assert np.all(shown[interior] > mean[interior] + 0.05)


def test_far_faces_outside_the_interest_are_not_owned():
    scene = Scene(slab=False)
    inside = vgi.FarTierSettings(voxel_pixels=64.0, cell=2, interest=((0, 0, 0), (1, 1, 1)))
    outside = vgi.FarTierSettings(voxel_pixels=64.0, cell=2, interest=((4, 4, 4), (5, 5, 5)))
    assert run(scene, inside, 1, top_camera())[1][0][2][0] == 64
    assert run(scene, outside, 1, top_camera())[1][0][2][0] == 0
    # Too large on screen: a 0.84-pixel voxel is not under a half-pixel threshold.
    near = vgi.FarTierSettings(voxel_pixels=0.5, cell=2)
    assert run(scene, near, 1, top_camera())[1][0][2][0] == 0
