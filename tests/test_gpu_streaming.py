"""Page streaming on the GPU geometry (vgi_update_regions, vgi_load_regions,
vgi_unload_regions: page_loaded, page_changed and page_unloaded,
src/input.rs:54-70) against the oracle's restatement of
TransportScene::with_page_contents with the same region deltas
(orc_scene_regions).

A terrain streams in and out across frames: regions load, unload, load
again, loaded ones are replaced with carved copies, and some are sent again
unchanged (also while being unloaded in the same change). Odd deltas are one
scene change (vgi_update_regions), even ones an unload then a load, and the
oracle takes the same changes. After every delta:
- the GPU's packed geometry equals the oracle's in canonical form (every
  region of the terrain, resident or not, with its top-level extents);
- without the top-level extents, it also equals a fresh pack of the same
  region set (O.Scene), since only the incremental top-level field may take
  another fixed point than a full build (src/world.rs:465-472);
- the world-cache frames traced over it (the faces set once, before any
  delta) give the oracle's results and resident state word for word.
"""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal

pytestmark = pytest.mark.gpu

N = (8, 4, 8)


def materials():
    rng = np.random.default_rng(3)
    m = vgi.VoxelGiMaterials()
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(248):
        r = float(rng.uniform(1, 10))
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(r, r, r)))
    return m.words()


def carved(vox, seed):
    """A copy of a region's voxels with a seeded ball carved out (a page change)."""
    out = vox.reshape(4096).copy()
    rng = np.random.default_rng(seed)
    c = rng.integers(2, 14, size=3)
    z, y, x = np.meshgrid(np.arange(16), np.arange(16), np.arange(16), indexing="ij")
    ball = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= 16
    out.reshape(16, 16, 16)[ball] = 256
    return out


def test_streamed_pages_match_the_oracle():
    coords, vox = vgi.terrain(*N, seed=11, base_height=30.0, falloff=18.0, emitters=24)
    vox = vox.reshape(-1, 4096)
    words = materials()
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0)).words()
    key = {tuple(c): i for i, c in enumerate(coords)}
    # Faces of the whole terrain, kept as the world cache throughout; while
    # their regions are out their paths start in unloaded space.
    faces = vgi.exposed_faces(coords, vox)[::4].copy()
    transport = vgi.TransportSettings(bounces=2, path_steps=256)
    pipe = O.Pipeline(2, 0, 256, 0, 8)

    resident = {tuple(c) for c in coords if c[0] < 5}
    current = {k: vox[key[k]] for k in resident}
    first = np.array(sorted(resident, key=lambda k: (k[2], k[1], k[0])), np.int32)

    g = vgi.GpuTracer(0)
    try:
        g.load_regions(first, np.stack([current[tuple(k)] for k in first]))
        ref = O.Scene(first, np.stack([current[tuple(k)] for k in first]), top_mode=0)
        g.set_materials(words)
        g.set_lights(sun, 1)
        g.set_environment((0.0, 0.0, 0.0))
        g.set_transport(transport)
        g.set_faces(faces)
        frames = None
        rng = np.random.default_rng(5)
        clock = 0
        for step in range(6):
            if step:
                out = [k for k in resident if rng.random() < 0.25]
                back = [tuple(c) for c in coords if tuple(c) not in resident and rng.random() < 0.5]
                change = [k for k in resident if k not in out and rng.random() < 0.1]
                # Pages sent again with the same voxels, some also unloaded in
                # the same change: the same regions, so not touched.
                same = [k for k in resident if k not in change and rng.random() < 0.1]
                loads = back + change + same
                for k in back:
                    current[k] = vox[key[k]]
                for i, k in enumerate(change):
                    current[k] = carved(current[k], 100 * step + i)
                load_coords = np.array(loads, np.int32).reshape(-1, 3)
                load_vox = np.stack([current[k] for k in loads]) if loads else np.zeros((0, 4096), np.uint16)
                out_coords = np.array(out, np.int32).reshape(-1, 3)
                if step % 2:
                    # One scene change per frame, as with_page_contents takes
                    # the frame's changed and removed pages together.
                    g.update_regions(load_coords, load_vox, out_coords)
                    ref.regions(load_coords, load_vox, removed=out_coords)
                else:
                    # Unload, then load: two scene changes on both sides.
                    if out:
                        g.unload_regions(out_coords)
                    if loads:
                        g.load_regions(load_coords, load_vox)
                    ref.regions(removed=out_coords)
                    ref.regions(load_coords, load_vox)
                resident.update(same)
                for k in out:
                    if k not in same:
                        resident.discard(k)
                        current.pop(k, None)
                resident.update(back)
            # Geometry: canonical form over every region of the terrain.
            d, h, cl, bounds = g.geometry()
            rd, rh, rcl, rbounds = ref.arrays()
            assert (bounds == rbounds).all(), (step, bounds, rbounds)
            got = O.canonical(d, h, cl, coords)
            assert_words_equal(got, O.canonical(rd, rh, rcl, coords), f"geometry after delta {step}")
            live = np.array(sorted(resident, key=lambda k: (k[2], k[1], k[0])), np.int32)
            fresh = O.Scene(live, np.stack([current[tuple(k)] for k in live]), top_mode=0).arrays()
            want = O.canonical(*fresh[:3], coords)
            got[:, 2:4] = 0
            want[:, 2:4] = 0
            assert_words_equal(got, want, f"geometry after delta {step} against a fresh pack")
            assert ((got[:, 0] == 0) == [tuple(c) not in resident for c in coords]).all()
            # Frames over the streamed geometry.
            g.build_emitters()
            emitters, n_emit, total = O.emitters(live, np.stack([current[tuple(k)] for k in live]), words)
            geometry = ref.arrays()

            def params(n, samples, geometry=geometry, total=total, n_emit=n_emit):
                return O.params_words(n, samples, geometry[0].size // 4, 1, geometry[3], 1, (0, 0, 0), total, n_emit)

            if frames is None:
                frames = O.Frames(geometry, params, words, sun, emitters, faces, transport, pipe)
            frames.geometry, frames.params_fn, frames.emitter_words = geometry, params, emitters
            for _ in range(2):
                g.frame(8, clock_ms=clock)
                frames.frame(8, clock_ms=clock)
                clock += 16
            assert_words_equal(g.read_results(), frames.results, f"frame results after delta {step}")
            assert_words_equal(g.read_state(), frames.state, f"resident state after delta {step}")
    finally:
        g.close()


def test_region_loads_refuse_bad_input_and_keep_the_scene():
    coords, vox = vgi.stone_room()
    with vgi.GpuTracer(0) as g:
        g.load_regions(coords, vox)
        before = g.geometry()
        dup = np.concatenate([coords[:2], coords[:1]])
        with pytest.raises(vgi.VgiError) as err:
            g.load_regions(dup, np.zeros((3, 4096), np.uint16))
        assert err.value.status == vgi.ERR_INVALID
        bad = np.full((1, 4096), 257, np.uint16)
        with pytest.raises(vgi.VgiError) as err:
            g.load_regions(np.array([[5, 5, 5]], np.int32), bad)
        assert err.value.status == vgi.ERR_INVALID
        after = g.geometry()
        for a, b in zip(before, after):
            assert (np.asarray(a) == np.asarray(b)).all()
        # Unloading what is not loaded changes nothing; unloading all leaves
        # an empty scene that frames can still trace (every path escapes or
        # reaches unloaded space).
        g.unload_regions(np.array([[9, 9, 9]], np.int32))
        g.unload_regions(coords)
        d, h, cl, bounds = g.geometry()
        assert (O.canonical(d, h, cl, coords)[:, 0] == 0).all()


def test_one_scene_change_refuses_bad_input_and_handles_reloads():
    """vgi_update_regions: a refused change (a duplicate loaded coordinate, a
    voxel above 256) leaves the scene as it was, even with removals in the
    same call; a region unloaded and loaded again with the same voxels in one
    change is the same region (geometry and top-level field unchanged), and
    with other voxels it is replaced."""
    coords, vox = vgi.stone_room()
    vox = vox.reshape(-1, 4096)
    with vgi.GpuTracer(0) as g:
        g.update_regions(coords, vox, np.zeros((0, 3), np.int32))
        before = g.geometry()
        dup = np.concatenate([coords[:2], coords[:1]])
        with pytest.raises(vgi.VgiError) as err:
            g.update_regions(dup, np.zeros((3, 4096), np.uint16), coords[3:4])
        assert err.value.status == vgi.ERR_INVALID
        bad = np.full((1, 4096), 257, np.uint16)
        with pytest.raises(vgi.VgiError) as err:
            g.update_regions(coords[:1], bad, coords[3:4])
        assert err.value.status == vgi.ERR_INVALID
        for a, b in zip(before, g.geometry()):
            assert (np.asarray(a) == np.asarray(b)).all()
        want = O.canonical(*before[:3], coords)
        # Unloaded and sent again unchanged in the same change: untouched.
        g.update_regions(coords[2:4], vox[2:4], coords[2:4])
        assert (O.canonical(*g.geometry()[:3], coords) == want).all()
        # Sent again with other voxels: replaced, as the oracle replaces it.
        changed = vox[2:3].copy()
        changed[0, :2048] = 256
        g.update_regions(coords[2:3], changed, coords[2:3])
        ref = O.Scene(coords, vox, top_mode=0)
        ref.regions(coords[2:3], changed, removed=coords[2:3])
        rd, rh, rcl, _ = ref.arrays()
        assert (O.canonical(*g.geometry()[:3], coords) == O.canonical(rd, rh, rcl, coords)).all()
