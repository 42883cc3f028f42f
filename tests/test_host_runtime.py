"""CPU tests of libvgi's host side: the library loads without a GPU, exports
every symbol the public headers declare, and its host runtime (top-level
growth, face index, emitter distribution and light tree) matches the oracle
word for word."""
import os
import re

import numpy as np
import pytest

import oracle_lib as O
import vgi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(vgi_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    lib = vgi.library()
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name


def test_context_creation_without_a_device_reports_unavailable():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(vgi.TransportUnavailable):
        vgi.GpuTracer(0)


def random_regions(seed, nx=6, ny=3, nz=5, drop=0.2, solid=0.35):
    rng = np.random.default_rng(seed)
    coords, solids = [], []
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                if rng.random() < drop:
                    continue
                coords.append((x - 2, y, z - 1))
                solids.append(1 if rng.random() < solid else 0)
    return np.array(coords, np.int32), np.array(solids, np.uint8)


@pytest.mark.parametrize("seed", range(6))
def test_top_level_growth_matches_oracle(seed):
    coords, solids = random_regions(seed)
    vox = np.full((len(coords), 4096), 256, np.uint16)
    vox[solids == 1, 100] = 2
    product = vgi.host_top_level(coords, solids)
    scene = O.Scene(coords, vox.reshape(-1), top_mode=0)
    assert product is not None
    assert (product == scene.top_level()).all()


def test_top_level_disabled_beyond_size_limits():
    coords = np.array([(0, 0, 0), (300, 0, 0)], np.int32)
    assert vgi.host_top_level(coords, np.zeros(2, np.uint8)) is None


def test_face_index_matches_oracle():
    coords, vox = vgi.terrain(4, 4, 4, seed=9, base_height=30.0, falloff=16.0, emitters=8)
    faces = vgi.exposed_faces(coords, vox)
    assert faces.shape[0] > 2000
    got = vgi.host_face_index(faces[:, :4])
    want = O.face_index(faces[:, :4])
    assert got.shape == want.shape
    assert (got == want).all()


def materials_with_emitters(n_emit=248):
    m = vgi.VoxelGiMaterials()
    rng = np.random.default_rng(11)
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(n_emit):
        r = float(rng.uniform(1, 10))
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(r, r, r)))
    return m


@pytest.mark.parametrize("scene", ["stone_room", "furnace", "terrain"])
def test_emitter_words_match_oracle(scene):
    if scene == "stone_room":
        coords, vox = vgi.stone_room()
        m = vgi.VoxelGiMaterials()
        m.set(0, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5)))
        m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(8.0, 4.0, 1.5)))
    elif scene == "furnace":
        coords, vox = vgi.furnace()
        m = vgi.VoxelGiMaterials()
        m.set(4, vgi.MaterialTransport(diffuse=(0.3, 0.55, 0.7), emission=(0.7, 1.3, 0.2)))
    else:
        coords, vox = vgi.terrain(6, 4, 6, seed=4, base_height=32.0, falloff=20.0, emitters=40)
        m = materials_with_emitters()
    words = m.words()
    got, faces, total = vgi.host_emitters(coords, vox, words)
    want, ofaces, ototal = O.emitters(coords, vox, words)
    assert faces == ofaces and total == ototal
    assert (got == want).all()
    if scene != "stone_room":
        assert faces >= 32  # light tree present
        assert got.view(np.float32)[7] == float(2 * faces - 1)


def test_terrain_generator_is_deterministic():
    a = vgi.terrain(3, 2, 3, seed=7)[1]
    b = vgi.terrain(3, 2, 3, seed=7)[1]
    c = vgi.terrain(3, 2, 3, seed=8)[1]
    assert (a == b).all() and not (a == c).all()


def test_stone_room_faces():
    coords, vox = vgi.stone_room()
    faces = vgi.exposed_faces(coords, vox)
    # 6 * 30^2 interior shell faces, the emitter's 5 exposed faces, minus the floor face it covers.
    assert faces.shape[0] == 6 * 30 * 30 + 5 - 1
