"""The allocation-free region packer (vgi_pack_regions_static) against the
regular upload path.

vgi_pack_regions_static exists for callers that must not allocate device
memory themselves. Examples are an engine that owns all GPU memory through
its own allocator, or a frame-critical thread where cudaMalloc's implicit
synchronisation would stall. Such a caller passes its own device buffers.

This test plays that caller. It places voxels, headers and cells in device
memory it already holds, calls the entry point through the C ABI twice in a
row on different scenes, and checks each result against what
vgi_upload_regions packs. The checks are exact: region kinds, materials and
every brick word and payload, compared in the layout-free canonical form.
"""
import ctypes

import numpy as np
import pytest

import oracle_lib as O
import vgi

pytestmark = pytest.mark.gpu


def _pack_static(coords, vox, capacity_words, with_used=False):
    import torch

    lib = vgi.library()
    fn = lib.vgi_pack_regions_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
    n = coords.shape[0]
    voxels = torch.from_numpy(vox.view(np.int16).copy()).cuda()
    headers = torch.zeros(n * 4, dtype=torch.int32, device="cuda")
    cells = torch.zeros(capacity_words, dtype=torch.int32, device="cuda")
    used = ctypes.c_uint64(0)
    stream = torch.cuda.current_stream()
    rc = fn(voxels.data_ptr(), n, headers.data_ptr(), cells.data_ptr(), capacity_words, ctypes.byref(used), stream.cuda_stream)
    out = (rc, headers.cpu().numpy().view(np.uint32), cells.cpu().numpy().view(np.uint32)[: used.value])
    return out + (used.value,) if with_used else out


def _reference_geometry(coords, vox):
    with vgi.GpuTracer(0) as g:
        g.upload_regions(coords, vox)
        return g.geometry()


def _check_scene(coords, vox):
    d, h, cl, _ = _reference_geometry(coords, vox)
    rc, sh, scl = _pack_static(coords, vox, capacity_words=coords.shape[0] * (64 + 64 * 32))
    assert rc == vgi.OK
    h = h.reshape(-1, 4)
    sh = sh.reshape(-1, 4).copy()
    assert (sh[:, 0] == h[:, 0]).all(), "region kinds"
    uniform = h[:, 0] != 3
    assert (sh[uniform, 1] == h[uniform, 1]).all(), "uniform materials"
    # The top-level extents and stride (header z, w) come from the host runtime.
    sh[:, 2:] = h[:, 2:]
    got = O.canonical(d, sh.reshape(-1), scl, coords)
    want = O.canonical(d, h.reshape(-1), cl, coords)
    assert (got == want).all(), "canonical geometry"
    # Cells follow region order: the first mixed region's table starts at 0.
    mixed = np.flatnonzero(h[:, 0] == 3)
    if mixed.size:
        assert sh[mixed[0], 1] == 0
    return scl.size


def test_static_pack_matches_upload_path_on_two_calls_in_a_row():
    coords_a, vox_a = vgi.terrain(6, 4, 6, seed=21, base_height=30.0, falloff=18.0, emitters=16)
    coords_b, vox_b = vgi.stone_room()
    used_a = _check_scene(coords_a, vox_a)
    used_b = _check_scene(coords_b, vox_b)
    assert used_a > 0 and used_b > 0


def test_static_pack_rejects_more_regions_than_its_scratch_holds():
    lib = vgi.library()
    fn = lib.vgi_pack_regions_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
    used = ctypes.c_uint64(7)
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    rc = fn(fake, 65537, fake, fake, 1 << 20, ctypes.byref(used), None)
    assert rc == vgi.ERR_CAPACITY and used.value == 0


def test_static_pack_reports_a_cell_buffer_too_small_and_recovers():
    # A cell buffer smaller than the scene needs: VGI_ERR_CAPACITY, nothing
    # counted as used. The next call with room packs the same scene exactly,
    # since each call clears the shared array's total and error words.
    coords, vox = vgi.terrain(6, 4, 6, seed=21, base_height=30.0, falloff=18.0, emitters=16)
    rc, _, _, used = _pack_static(coords, vox, capacity_words=100, with_used=True)
    assert rc == vgi.ERR_CAPACITY and used == 0
    assert _check_scene(coords, vox) > 100


def test_static_pack_rejects_voxel_values_above_air():
    # 256 is air; 257 is no voxel value: VGI_ERR_INVALID, then a good call works.
    coords, vox = vgi.stone_room()
    bad = vox.copy()
    bad[4096 * 3 + 100] = 257
    rc, _, _, used = _pack_static(coords, bad, capacity_words=coords.shape[0] * (64 + 64 * 32), with_used=True)
    assert rc == vgi.ERR_INVALID and used == 0
    assert _check_scene(coords, vox) > 0
