"""Sparse updates of host-packed geometry (vgi_patch_packed), the staging of
GpuTracer::synchronize_geometry (src/gpu/geometry.rs:19-124) for a
SceneDelta (src/gpu_scene.rs:49-60): element ranges of the directory,
headers and cells, a whole directory when its capacity changes, and arrays
that grow or shrink with the scene.

The oracle packs a terrain, then the same terrain after voxel edits, after
more regions load (new bounds, more cells, a larger directory) and after
regions unload. Each change goes to the GPU as the delta between the two
packings: the runs of elements that differ, plus any grown tail. After each
delta the GPU's arrays equal the oracle's word for word, and frames traced
over them give the oracle's results and resident state word for word.
"""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal

pytestmark = pytest.mark.gpu


def runs(old, new, width):
    """(start, elements) for every run of rows of `new` that differ from
    `old`, rows past the end of `old` included."""
    a = np.asarray(old).reshape(-1, width)
    b = np.asarray(new).reshape(-1, width)
    m = min(a.shape[0], b.shape[0])
    diff = np.ones(b.shape[0], bool)
    diff[:m] = (a[:m] != b[:m]).any(axis=1)
    out = []
    i = 0
    while i < b.shape[0]:
        if not diff[i]:
            i += 1
            continue
        j = i
        while j < b.shape[0] and diff[j]:
            j += 1
        out.append((i, b[i:j].copy()))
        i = j
    return out


def send_delta(g, old, new):
    d0, h0, c0, _ = old
    d1, h1, c1, b1 = new
    rebuilt = d0.size != d1.size
    lengths = (d1.size // 4, h1.size // 4, c1.size)
    directory = d1 if rebuilt else runs(d0, d1, 4)
    g.patch_packed(lengths, b1, rebuilt, directory, runs(h0, h1, 4), runs(c0, c1, 1))
    moved = sum(e.size for _, e in runs(h0, h1, 4)) + sum(e.size for _, e in runs(c0, c1, 1))
    return rebuilt, moved


def materials():
    rng = np.random.default_rng(3)
    m = vgi.VoxelGiMaterials()
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(248):
        r = float(rng.uniform(1, 10))
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(r, r, r)))
    return m.words()


def test_packed_deltas_match_the_oracle():
    coords, vox = vgi.terrain(6, 4, 6, seed=23, base_height=30.0, falloff=18.0, emitters=16)
    vox = vox.reshape(-1, 4096)
    words = materials()
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0)).words()
    transport = vgi.TransportSettings(bounces=2, path_steps=256)
    pipe = O.Pipeline(2, 0, 256, 0, 8)
    # Start from the regions with x < 4; the others load later.
    first = coords[:, 0] < 4
    ref = O.Scene(coords[first], vox[first], top_mode=0)
    faces = vgi.exposed_faces(coords, vox)[::3].copy()
    with vgi.GpuTracer(0) as g:
        packed = ref.arrays()
        g.upload_packed(*packed)
        g.set_materials(words)
        g.set_lights(sun, 1)
        g.set_environment((0.0, 0.0, 0.0))
        g.set_transport(transport)
        g.set_faces(faces)
        live = (coords[first], vox[first])
        frames = None
        clock = 0
        rng = np.random.default_rng(9)
        seen = {"rebuilt": False, "grown": False, "shrunk": False}
        for step in range(4):
            if step == 1:
                # Voxel edits: a carved ball and a placed block.
                e = []
                for x in range(20, 27):
                    for y in range(20, 27):
                        for z in range(20, 27):
                            if (x - 23) ** 2 + (y - 23) ** 2 + (z - 23) ** 2 <= 9:
                                e.append((x, y, z, 256))
                e += [(40, 50, 40 + k, 3) for k in range(5)]
                ref.edit(np.array(e, np.int32))
                live_coords, live_vox = live
                live_vox = live_vox.copy()
                key = {tuple(c): i for i, c in enumerate(live_coords)}
                for x, y, z, v in e:
                    r = key.get((x >> 4, y >> 4, z >> 4))
                    if r is not None:
                        live_vox[r][((z & 15) * 16 + (y & 15)) * 16 + (x & 15)] = v
                live = (live_coords, live_vox)
            elif step == 2:
                # The other regions load: new bounds, more headers and cells.
                ref.regions(coords[~first], vox[~first])
                live = (coords, vox)
            elif step == 3:
                # A third of the regions unload.
                out = rng.random(coords.shape[0]) < 0.33
                ref.regions(removed=coords[out])
                live = (coords[~out], vox[~out])
            if step:
                new = ref.arrays()
                rebuilt, moved = send_delta(g, packed, new)
                seen["rebuilt"] |= rebuilt
                seen["grown"] |= new[2].size > packed[2].size
                seen["shrunk"] |= new[1].size < packed[1].size
                assert moved > 0
                packed = new
            got = g.geometry()
            for a, b, what in zip(got, packed, ("directory", "headers", "cells", "bounds")):
                assert_words_equal(np.asarray(a).reshape(-1), np.asarray(b).reshape(-1), f"{what} after delta {step}")
            emitters, n_emit, total = O.emitters(*live, words)
            g.set_emitters(emitters, n_emit, total)

            def params(n, samples, geometry=packed, total=total, n_emit=n_emit):
                return O.params_words(n, samples, geometry[0].size // 4, 1, geometry[3], 1, (0, 0, 0), total, n_emit)

            if frames is None:
                frames = O.Frames(packed, params, words, sun, emitters, faces, transport, pipe)
            frames.geometry, frames.params_fn, frames.emitter_words = packed, params, emitters
            for _ in range(2):
                g.frame(8, clock_ms=clock)
                frames.frame(8, clock_ms=clock)
                clock += 16
            assert_words_equal(g.read_results(), frames.results, f"frame results after delta {step}")
            assert_words_equal(g.read_state(), frames.state, f"resident state after delta {step}")
        assert seen["grown"] and seen["shrunk"], seen


def test_refused_packed_deltas_change_nothing():
    coords, vox = vgi.stone_room()
    ref = O.Scene(coords, vox)
    packed = ref.arrays()
    with vgi.GpuTracer(0) as g:
        # Without packed geometry there is nothing to patch.
        g.upload_regions(coords, vox)
        with pytest.raises(vgi.VgiError) as err:
            g.patch_packed((packed[0].size // 4, packed[1].size // 4, packed[2].size), packed[3], False, [], [], [])
        assert err.value.status == vgi.ERR_STATE
        g.upload_packed(*packed)
        lengths = (packed[0].size // 4, packed[1].size // 4, packed[2].size)
        bad = [
            # a header of kind 7
            dict(headers=[(0, np.array([[7, 0, 0, 0]], np.uint32))]),
            # a mixed header whose brick table runs past the cells
            dict(headers=[(0, np.array([[3, packed[2].size - 8, 0, 0]], np.uint32))]),
            # a directory entry naming a header past the end
            dict(directory=[(0, np.array([[0, 0, 0, lengths[1] + 5]], np.int32))]),
            # a range past its array
            dict(cells=[(lengths[2], np.zeros(4, np.uint32))]),
        ]
        for case in bad:
            with pytest.raises(vgi.VgiError) as err:
                g.patch_packed(lengths, packed[3], False, case.get("directory", []), case.get("headers", []), case.get("cells", []))
            assert err.value.status == vgi.ERR_INVALID, case
            for a, b in zip(g.geometry(), packed):
                assert (np.asarray(a).reshape(-1) == np.asarray(b).reshape(-1)).all()
        # A directory of another capacity has to come whole.
        with pytest.raises(vgi.VgiError) as err:
            g.patch_packed((lengths[0] * 2, lengths[1], lengths[2]), packed[3], False, [], [], [])
        assert err.value.status == vgi.ERR_INVALID


def page_regions(page, voxels32):
    """The eight 16^3 regions of a 32^3 page (x fastest) at page coordinate
    `page` (region coordinates page * 2 + offset)."""
    v = np.asarray(voxels32, np.uint16).reshape(32, 32, 32)  # z, y, x
    coords, vox = [], []
    for oz in range(2):
        for oy in range(2):
            for ox in range(2):
                coords.append([page[0] * 2 + ox, page[1] * 2 + oy, page[2] * 2 + oz])
                vox.append(v[oz * 16:(oz + 1) * 16, oy * 16:(oy + 1) * 16, ox * 16:(ox + 1) * 16].reshape(4096))
    return np.array(coords, np.int32), np.stack(vox)


def test_sparse_uploads_survive_growth_and_residency_changes():
    """The reference's sparse-upload scenario (src/gpu/upload_tests.rs:22-80)
    on both geometry paths: a page with a floor at y = 4; fifteen more pages
    along x; those unloaded; a page at x = -1; one floor voxel carved; the
    first page emptied. After every stage the page events
    (vgi_update_regions) and the sparse packed delta (vgi_patch_packed) give
    the oracle's geometry, and frames over each give the oracle's results."""
    floor = np.full((32, 32, 32), 256, np.uint16)
    floor[:, 4, :] = 1
    m = vgi.VoxelGiMaterials()
    m.set(1, vgi.MaterialTransport(diffuse=(0.6, 0.6, 0.6)))
    m.set(2, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(4.0, 4.0, 4.0)))
    words = m.words()
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0)).words()
    transport = vgi.TransportSettings(bounces=1, path_steps=128)
    pipe = O.Pipeline(1, 0, 128, 0, 4)
    probes = np.array([[x, 4, 8, 2, 1] for x in range(12, 20)], np.int32)  # +Y faces of the floor
    first_coords, first_vox = page_regions((0, 0, 0), floor)
    ref = O.Scene(first_coords, first_vox, top_mode=0)
    streamed, patched = vgi.GpuTracer(0), vgi.GpuTracer(0)
    try:
        streamed.update_regions(first_coords, first_vox, np.zeros((0, 3), np.int32))
        packed = ref.arrays()
        patched.upload_packed(*packed)
        for g in (streamed, patched):
            g.set_materials(words)
            g.set_lights(sun, 1)
            g.set_environment((0.1, 0.1, 0.1))
            g.set_transport(transport)
        resident = {(0, 0, 0): floor.copy()}
        for stage in range(6):
            loads, removed = [], []
            if stage == 1:
                loads = [((x, 0, 0), floor) for x in range(1, 16)]
            elif stage == 2:
                removed = [(x, 0, 0) for x in range(1, 16)]
            elif stage == 3:
                loads = [((-1, 0, 0), floor)]
            elif stage == 4:
                carved = resident[(0, 0, 0)].copy()
                carved[8, 4, 8] = 256
                loads = [((0, 0, 0), carved)]
            elif stage == 5:
                loads = [((0, 0, 0), np.full((32, 32, 32), 256, np.uint16))]
            if stage:
                lc = [page_regions(p, v) for p, v in loads]
                load_coords = np.concatenate([c for c, _ in lc]) if lc else np.zeros((0, 3), np.int32)
                load_vox = np.concatenate([v for _, v in lc]) if lc else np.zeros((0, 4096), np.uint16)
                rm = np.concatenate([page_regions(p, floor)[0] for p in removed]) if removed else np.zeros((0, 3), np.int32)
                streamed.update_regions(load_coords, load_vox, rm)
                ref.regions(load_coords, load_vox, removed=rm)
                new = ref.arrays()
                send_delta(patched, packed, new)
                packed = new
                for p in removed:
                    resident.pop(p, None)
                for p, v in loads:
                    resident[p] = v
            live = [page_regions(p, v) for p, v in resident.items()]
            live_coords = np.concatenate([c for c, _ in live])
            live_vox = np.concatenate([v for _, v in live])
            got_stream = streamed.geometry()
            got_patch = patched.geometry()
            for a, b, what in zip(got_patch, packed, ("directory", "headers", "cells", "bounds")):
                assert_words_equal(np.asarray(a).reshape(-1), np.asarray(b).reshape(-1), f"patched {what}, stage {stage}")
            assert_words_equal(O.canonical(*got_stream[:3], live_coords), O.canonical(*packed[:3], live_coords),
                               f"streamed geometry, stage {stage}")
            emitters, n_emit, total = O.emitters(live_coords, live_vox, words)

            def params(n, samples, geometry=packed, total=total, n_emit=n_emit):
                return O.params_words(n, samples, geometry[0].size // 4, 1, geometry[3], 1, (0.1, 0.1, 0.1), total, n_emit)

            want = O.Frames(packed, params, words, sun, emitters, probes, transport, pipe)
            for g in (streamed, patched):
                g.set_emitters(emitters, n_emit, total)
                g.set_faces(probes)
                g.frame(4, clock_ms=0)
                g.frame(4, clock_ms=16)
            want.frame(4, clock_ms=0)
            want.frame(4, clock_ms=16)
            assert_words_equal(patched.read_results(), want.results, f"patched results, stage {stage}")
            assert_words_equal(streamed.read_results(), want.results, f"streamed results, stage {stage}")
    finally:
        streamed.close()
        patched.close()
