"""The oracle library makes the benchmark inputs without libvgi: the seeded
scene generators compiled into liboracle write the same voxels and face
lists as libvgi's, and the numpy restatements of the model records equal
libvgi's GpuMaterial and GpuLight encoders (src/world.rs:166-173,
src/gpu.rs:713-744). bench.py's CPU arm relies on this to time the oracle
on the GPU arm's workload without loading the product library."""
import numpy as np

import oracle_lib as O
import vgi


def test_terrain_and_faces_equal_libvgi():
    c1, v1 = O.terrain(4, 3, 5, seed=3, base_height=24.0, falloff=20.0, emitters=16)
    c2, v2 = vgi.terrain(4, 3, 5, seed=3, base_height=24.0, falloff=20.0, emitters=16)
    assert (c1 == c2).all() and (v1 == v2).all()
    assert (v1 >= 8).any() and (v1 < 256).any() and (v1 == 256).any()
    for facing in (None, (30.0, 40.0, 30.0)):
        f1 = O.exposed_faces(c1, v1, facing=facing)
        f2 = vgi.exposed_faces(c2, v2, facing=facing)
        assert f1.shape[0] > 0 and (f1 == f2).all()
    r1, r2 = O.stone_room(), vgi.stone_room()
    assert (r1[0] == r2[0]).all() and (r1[1] == r2[1]).all()


def test_record_encoders_equal_libvgi():
    rng = np.random.default_rng(1)
    m = vgi.VoxelGiMaterials()
    entries = []
    for k in range(256):
        d = tuple(rng.uniform(-0.5, 1.5, 3))
        e = tuple(rng.uniform(-1.0, 20.0, 3))
        if k == 5:
            e = (float("inf"), float("nan"), 3.0)
        if k == 6:
            d = (float("nan"), 2.0, -1.0)
        m.set(k, vgi.MaterialTransport(diffuse=d, emission=e))
        entries.append((d, e))
    assert (m.words().view(np.uint32) == O.material_words(entries).view(np.uint32)).all()
    for direction in [(0.4, 0.8, 0.3), (1.0, 0.0, 0.0), (0.0, 0.0, 0.0), (1e-30, 2e-30, 0.0), (3.0, -4.0, 12.0)]:
        a = vgi.DirectionalTransportLight(direction, (3.0, 2.0, 1.0), (0.1, 0.2, 0.3)).words()
        b = O.directional_light_words(direction, (3.0, 2.0, 1.0), (0.1, 0.2, 0.3))
        assert (a.view(np.uint32) == b.view(np.uint32)).all(), direction


def test_frame_slots_equals_a_whole_frame_on_its_slots():
    # frame_slots over every slot in order is the whole frame.
    coords, vox = O.stone_room()
    words = O.material_words([((0.5, 0.5, 0.5), (0.0, 0.0, 0.0)), ((0.5, 0.5, 0.5), (8.0, 4.0, 1.5))] +
                             [((0.45, 0.45, 0.45), (0.0, 0.0, 0.0))] * 254)
    faces = O.exposed_faces(coords, vox)
    scene = O.Scene(coords, vox)
    geometry = scene.arrays()
    emitters, n_emit, total = O.emitters(coords, vox, words)
    d = geometry[0]

    def params(n, samples):
        return O.params_words(n, samples, d.size // 4, 0, geometry[3], 0, (0, 0, 0), total, n_emit)

    t = O.transport_settings(bounces=1, path_steps=64, history_limit=64)
    a = O.Frames(geometry, params, words, np.zeros(0, np.float32), emitters, faces, t, O.Pipeline(1, 0, 64, 0, 4))
    b = O.Frames(geometry, params, words, np.zeros(0, np.float32), emitters, faces, t, O.Pipeline(1, 0, 64, 0, 4))
    for f in range(3):
        a.frame(4, 16 * f)
        b.frame_slots(4, 16 * f, np.arange(faces.shape[0]))
    assert (a.state == b.state).all() and (a.results == b.results).all()
