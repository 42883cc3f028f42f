"""CPU tests of libvgi's host side: the library loads without a GPU, exports
every symbol the public headers declare, and its host runtime (top-level
growth, face index, emitter distribution and light tree) matches the oracle
word for word."""
import ctypes
import os
import re
import subprocess
import sys

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
    # transport_failure_missing_device_does_not_select_cpu_implicitly
    # (src/tests.rs:10-37): with no visible device vgi_create returns
    # VGI_UNAVAILABLE and no context, the Python mirror raises
    # TransportUnavailable, and no call runs anything (there is no CPU path).
    # A child process hides every device, so this holds on a GPU box too.
    code = r"""
import ctypes, sys
sys.path.insert(0, sys.argv[1])
import vgi
lib = vgi.library()
h = ctypes.c_void_p(12345)
cfg = vgi._Config(0, 0)
rc = lib.vgi_create(ctypes.byref(cfg), ctypes.byref(h))
assert rc == vgi.UNAVAILABLE, rc
assert h.value is None, h.value
assert lib.vgi_frame(None, 8, 0) == vgi.ERR_INVALID
try:
    vgi.GpuTracer(0)
except vgi.TransportUnavailable:
    print("idle")
"""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code, os.path.join(ROOT, "global-illumination_b200")], env=env, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "idle"


def test_failure_injection_refuses_unknown_kinds():
    lib = vgi.library()
    assert lib.vgi_inject_failure(None, 7, 1) == vgi.ERR_INVALID
    assert lib.vgi_inject_failure(None, vgi.INJECT_ALLOC, 0) == vgi.OK
    assert lib.vgi_inject_failure(None, vgi.INJECT_UPLOAD, 0) == vgi.OK


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


def test_light_selection_frequencies_match_reported_probabilities():
    # Restates emission/tree.rs:199-262 on the oracle's light-tree walk (the
    # shader's choose_emitter and tree_probability): at a few receivers, the
    # frequencies of 262,144 independent uniforms' choices, pooled into 64
    # bins by emitter index, pass the reference's Pearson gate against the
    # reported probabilities, which sum to one.
    O.lib().orc_choose_emitters.restype = ctypes.c_int
    O.lib().orc_choose_emitters.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
    O.lib().orc_emitter_probability.restype = ctypes.c_float
    O.lib().orc_emitter_probability.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_uint32]
    coords, vox = vgi.terrain(6, 4, 6, seed=5, base_height=30.0, falloff=18.0, emitters=200)
    words, n_emit, total = O.emitters(coords, vox, materials_with_emitters().words())
    assert n_emit >= 32  # the tree, not the CDF
    records = words[: n_emit * 8].reshape(n_emit, 8)
    lookup = {(int(r[0]), int(r[1]), int(r[2]), int(r[3])): i for i, r in enumerate(records.view(np.int32))}
    faces = vgi.exposed_faces(coords, vox)
    normals = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    N = 262144
    state = np.uint64(0x243F6A8885A308D3)
    with np.errstate(over="ignore"):
        steps = np.arange(1, N + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15) + state
        w = steps
        w = (w ^ (w >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        w = (w ^ (w >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        w ^= w >> np.uint64(31)
    uniforms = ((w >> np.uint64(40)).astype(np.float32) / np.float32(16777216.0)).astype(np.float32)
    for probe in faces[::max(1, len(faces) // 3)][:3]:
        n = normals[probe[3]]
        position = (probe[:3].view(np.int32).astype(np.float32) + np.float32(0.5) + n * np.float32(0.5)).astype(np.float32)
        expected = np.zeros(64)
        for i, r in enumerate(records.view(np.int32)):
            expected[i % 64] += O.lib().orc_emitter_probability(O.ptr(words), n_emit, total, O.ptr(position), O.ptr(n), O.ptr(r[:3].copy()),
                                                                int(r[3]))
        assert abs(expected.sum() - 1.0) < 2e-5
        out = np.zeros((N, 5), np.uint32)
        O.lib().orc_choose_emitters(O.ptr(words), n_emit, total, O.ptr(position), O.ptr(n), O.ptr(uniforms), N, O.ptr(out))
        observed = np.zeros(64)
        for row in out.view(np.int32)[:, :4]:
            observed[lookup[tuple(int(v) for v in row)] % 64] += 1
        bins, rare_o, rare_e = [], 0.0, 0.0
        for o, p in zip(observed, expected):
            e = p * N
            if e >= 8.0:
                bins.append([o, e])
            else:
                rare_o += o
                rare_e += e
        if rare_e >= 8.0:
            bins.append([rare_o, rare_e])
        else:
            bins[0][0] += rare_o
            bins[0][1] += rare_e
        df = len(bins) - 1
        chi2 = sum((o - e) ** 2 / e for o, e in bins)
        assert chi2 < df + 10.0 * (2.0 * df) ** 0.5 + 50.0, (chi2, df, position)


def test_edit_events_encode_like_the_reference_planner():
    """vgi.encode_edit_events packs measured edits as encode_events does
    (src/gpu/resident.rs:1320-1414): event headers (union min, union max,
    (cap 0, 0, first bound, bounds)), then bounds (min, flux) (max, kind 6),
    and per bound a measure record (bound record, first position, margin
    count, changed voxels) (min - 1, flux) (size + margin)."""
    words, n, measures = vgi.encode_edit_events([((1, 2, 3), (4, 5, 6), 17, 40.0), ((10, 0, 0), (10, 1, 2), 3, 2.5)])
    assert n == 2
    w = words.reshape(-1, 4)
    assert w.shape == (2 * 3 + 2 * 2, 4)
    assert w[0].tolist() == [1, 2, 3, 0] and w[1].tolist() == [4, 5, 6, 0] and w[2].tolist() == [0, 0, 0, 1]
    assert w[5].tolist() == [0, 0, 1, 1]
    f40 = int(np.float32(40.0).view(np.uint32))
    assert w[6].tolist() == [1, 2, 3, f40] and w[7].tolist() == [4, 5, 6, 6]
    assert w[8].tolist()[:3] == [10, 0, 0] and w[9].tolist() == [10, 1, 2, 6]
    m = measures.reshape(-1, 3, 4)
    assert m[0].tolist() == [[6, 0, 6 * 6 * 6, 17], [0, 1, 2, f40], [6, 6, 6, 0]]
    assert m[1][0].tolist() == [8, 216, 3 * 4 * 5, 3]
    assert m[1][1][:3].tolist() == [9, 4294967295, 4294967295]


def test_cave_generator_stays_inside_its_volume():
    """Skylight shafts reach the top voxel row and no further: the generator
    writes nothing past the volume it fills (padding after it is untouched),
    for caves whose shafts land on the last rows of regions."""
    import ctypes

    nx, ny, nz = 6, 4, 6
    n = nx * ny * nz * 4096
    for seed in range(12):
        p = vgi.CaveParams(seed, 6, 60, 3.0, 8.0, 6, 16, 6.0, 20)
        buf = np.full(n + 2 * 4096 * nx * ny, 777, np.uint16)
        vgi.library().vgi_scene_cave(ctypes.byref(p), nx, ny, nz, buf.ctypes.data_as(ctypes.c_void_p))
        assert (buf[n:] == 777).all(), seed
        assert (buf[:n] == 256).any() and (buf[:n] != 256).any()


def _one_region(voxels_materials):
    vox = np.full(4096, 256, np.uint16)
    for (x, y, z), m in voxels_materials:
        vox[x + 16 * (y + 16 * z)] = m
    return np.zeros((1, 3), np.int32), vox


def test_emission_distribution_holds_exposed_faces_with_normalised_power():
    # emission.rs:400-433: two adjacent emissive voxels have 10 exposed faces
    # of equal power; the probabilities sum to 1; the CDF's first entry is
    # 0.1 and its last 1.0, so a choice of 0 takes the first face and 0.999
    # the last (choose_emitter's search).
    coords, vox = _one_region([((4, 4, 4), 10), ((5, 4, 4), 10)])
    entries = [((0.5, 0.5, 0.5), (0.0, 0.0, 0.0))] * 256
    entries[10] = ((0.5, 0.5, 0.5), (5.0, 5.0, 5.0))
    words, n_emit, total = O.emitters(coords, vox, O.material_words(entries))
    assert n_emit == 10
    records = words[: n_emit * 8].reshape(n_emit, 8)
    cumulative = records[:, 4].view(np.float32)
    probability = records[:, 5].view(np.float32)
    assert abs(float(probability.astype(np.float64).sum()) - 1.0) < 1e-6
    assert cumulative[0] == np.float32(0.1) and cumulative[-1] == np.float32(1.0)
    assert (np.diff(cumulative) > 0).all()
    # The library's host build (vgi_build_emitters) writes the same words.
    assert (vgi.host_emitters(coords, vox, O.material_words(entries))[0] == words).all()


def test_light_tree_keeps_weak_emitters_selectable():
    # emission/tree.rs:266-293: one emitter a 1e18 times brighter than 63
    # others in a row; the tree's selection probability of every face, seen
    # from above the row, stays positive and finite and they sum to 1.
    O.lib().orc_emitter_probability.restype = ctypes.c_float
    O.lib().orc_emitter_probability.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_uint32]
    coords = np.array([[x, 0, 0] for x in range(4)], np.int32)
    vox = np.full((4, 4096), 256, np.uint16)
    for x in range(64):
        vox[x // 16][(x % 16) + 16 * (0 + 16 * 0)] = 4 if x == 0 else 5
    entries = [((0.5, 0.5, 0.5), (0.0, 0.0, 0.0))] * 256
    entries[4] = ((0.5, 0.5, 0.5), (1.0, 1.0, 1.0))
    entries[5] = ((0.5, 0.5, 0.5), (1e-18, 1e-18, 1e-18))
    words, n_emit, total = O.emitters(coords, vox, O.material_words(entries))
    assert n_emit >= 32  # the tree, not the CDF
    records = words[: n_emit * 8].reshape(n_emit, 8).view(np.int32)
    position = np.array([0.5, 2.0, 0.5], np.float32)
    normal = np.array([0.0, -1.0, 0.0], np.float32)
    probabilities = np.array([O.lib().orc_emitter_probability(O.ptr(words), n_emit, total, O.ptr(position), O.ptr(normal),
                                                              O.ptr(r[:3].copy()), int(r[3])) for r in records], np.float64)
    assert np.isfinite(probabilities).all() and (probabilities > 0.0).all()
    assert abs(probabilities.sum() - 1.0) < 1e-5
    assert (vgi.host_emitters(coords, vox, O.material_words(entries))[0] == words).all()
