"""ctypes binding of the CPU oracle (oracle/liboracle.so).

Test infrastructure only: the oracle is the checker the CUDA path is compared
with; nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I64 = ctypes.c_int64
_INT = ctypes.c_int
_F = ctypes.c_float


class Counters(ctypes.Structure):
    _fields_ = [("rays", _U64), ("paths", _U64), ("steps", _U64), ("bytes", _U64), ("unknown", _U64),
                ("cache_hits", _U64), ("status", _U64 * 4), ("traverse_bytes", _U64)]

    def as_dict(self):
        d = {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "status"}
        d["status"] = [int(v) for v in self.status]
        return d


class Pipeline(ctypes.Structure):
    _fields_ = [("diffuse_hits", _U32), ("limited_reach", _U32), ("path_steps", _U32), ("budgeted", _U32), ("lanes", _U32)]


_SIG = {
    "orc_build_aadf": (_INT, [_U32, _U32, _U32, _P, _P]),
    "orc_scene_create": (_INT, [_P, _U32, _P, _P, _INT, _P]),
    "orc_scene_free": (None, [_P]),
    "orc_scene_edit": (_INT, [_P, _P, _U32]),
    "orc_scene_regions": (_INT, [_P, _P, _U32, _P, _P, _P, _U32]),
    "orc_scene_info": (_INT, [_P, _P, _P]),
    "orc_scene_copy": (_INT, [_P, _P, _P, _P]),
    "orc_scene_top_level": (_INT, [_P, _P]),
    "orc_canonical": (_INT, [_P, _U64, _P, _P, _U64, _P, _U32, _P]),
    "orc_trace_faces": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _P, _P, _P, _INT]),
    "orc_trace_faces_predicted": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _P, _P, _P, _U32, _P, _P, _INT]),
    "orc_predicted_misses": (_U64, [_P]),
    "orc_accumulate_picks": (_INT, [_P, _P, _P, _P, _P, _U32, _P, _P]),
    "orc_footprints": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _U32, _P, _P]),
    "orc_discover": (_INT, [_P, _U64, _P, _P, _P, _P, _U32, _U32, _P, _INT]),
    "orc_far_frame": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _P, _P, _P, _P, _INT]),
    "orc_reconstruct": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _U32, _U32, _P, _U32, _P, _P]),
    "orc_corner_value": (_INT, [_P, _P, _P, _P, _P]),
    "orc_present": (_INT, [_P, _U64, _P, _P, _P, _P, _U32, _P, _U32, _U32, _INT, _P, _INT]),
    "orc_classify": (_INT, [_P, _P, _U32, _P]),
    "orc_select": (_INT, [_P, _P, _P, _U32, _P, _P, _P, _P, _P]),
    "orc_trace_ray": (_INT, [_P, _U64, _P, _P, _P, _P, _U32, _U32, _P]),
    "orc_advance_box": (_INT, [_P, _P]),
    "orc_sample_1d": (_F, [_U32, _U32, _U32]),
    "orc_hemisphere": (None, [_P, _F, _F, _P]),
    "orc_sincos": (None, [_F, _P, _P]),
    "orc_exp": (_F, [_F]),
    "orc_pcg": (_U32, [_U32]),
    "orc_curve_limit": (_U32, [_U32]),
    "orc_resolve_retention": (_INT, [_P, _U32, _P, _U32, _INT, _P, _P, _P]),
    "orc_begin_trace": (_INT, [_P, _P, _P, _P, _U32, _P]),
    "orc_mark_changed": (_INT, [_P, _P, _P, _U32, _P]),
    "orc_accumulate": (_INT, [_P, _P, _P, _P, _P, _U32, _P]),
    "orc_apply_events": (_INT, [_P, _P, _P, _P, _U32, _P]),
    "orc_measure_edits": (_INT, [_P, _P, _P, _P, _P, _U32, _P]),
    "orc_trace_view_paths": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _U32, _P]),
    "orc_view_frame": (_INT, [_P, _U64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "orc_face_index": (_I64, [_P, _U32, _P, _U64]),
    "orc_emitters": (_I64, [_P, _U32, _P, _P, _P, _U64, _P]),
    "orc_sun_flip_log": (_U64, [_P, _U64]),
    "orc_sun_flip_log_clear": (None, []),
    # Seeded scene generators (input synthesis, compiled into liboracle from
    # the package's vgi_scenes.cpp), so CPU-only callers need no libvgi.
    "vgi_scene_grid_coords": (_U32, [_U32, _U32, _U32, _P]),
    "vgi_scene_stone_room": (None, [_P]),
    "vgi_scene_terrain": (None, [_P, _U32, _U32, _U32, _P]),
    "vgi_scene_cave": (None, [_P, _U32, _U32, _U32, _P]),
    "vgi_scene_faces": (_U64, [_P, _U32, _P, _P, _P, _U64]),
}

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_PATH):
            build()
        l = ctypes.CDLL(ORACLE_PATH)
        for name, (res, args) in _SIG.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def f2u(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


# ---- geometry -------------------------------------------------------------

def build_aadf(size, blocked):
    sx, sy, sz = size
    b = c(blocked, np.uint8).reshape(-1)
    out = np.zeros(b.size * 6, np.uint8)
    lib().orc_build_aadf(sx, sy, sz, ptr(b), ptr(out))
    return out.reshape(-1, 6)


class Scene:
    """The reference's packing of a region list (PackedScene over a scene
    built from nothing): directory, headers, cells and region bounds."""

    def __init__(self, coords, voxels, top_mode: int = 0, strides=None):
        coords = c(coords, np.int32).reshape(-1, 3)
        voxels = c(voxels, np.uint16).reshape(-1)
        st = None if strides is None else c(strides, np.uint8)
        h = ctypes.c_void_p()
        rc = lib().orc_scene_create(ptr(coords), coords.shape[0], ptr(voxels), ptr(st), top_mode, ctypes.byref(h))
        assert rc == 0, rc
        self._h = h
        self.coords = coords

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_scene_free(self._h)
            self._h = None

    def edit(self, edits) -> None:
        e = c(edits, np.int32).reshape(-1, 4)
        assert lib().orc_scene_edit(self._h, ptr(e), e.shape[0]) == 0

    def regions(self, coords=None, voxels=None, removed=None, strides=None) -> None:
        """Loads (or replaces) regions and unloads others (orc_scene_regions)."""
        co = c(np.zeros((0, 3)) if coords is None else coords, np.int32).reshape(-1, 3)
        vx = c(np.zeros(0) if voxels is None else voxels, np.uint16).reshape(-1)
        assert vx.size == co.shape[0] * 4096
        rm = c(np.zeros((0, 3)) if removed is None else removed, np.int32).reshape(-1, 3)
        st = None if strides is None else c(strides, np.uint8)
        assert lib().orc_scene_regions(self._h, ptr(co) if co.size else None, co.shape[0], ptr(vx) if vx.size else None, ptr(st),
                                       ptr(rm) if rm.size else None, rm.shape[0]) == 0

    def arrays(self):
        sizes = np.zeros(3, np.uint64)
        bounds = np.zeros(6, np.int32)
        lib().orc_scene_info(self._h, ptr(sizes), ptr(bounds))
        d = np.zeros(int(sizes[0]) * 4, np.int32)
        h = np.zeros(int(sizes[1]) * 4, np.uint32)
        cl = np.zeros(max(int(sizes[2]), 1), np.uint32)
        lib().orc_scene_copy(self._h, ptr(d), ptr(h), ptr(cl))
        return d, h, cl[: int(sizes[2])], bounds

    def top_level(self):
        bounds = self.arrays()[3]
        n = int(np.prod(bounds[3:] - bounds[:3] + 1))
        out = np.zeros(n * 6, np.uint8)
        rc = lib().orc_scene_top_level(self._h, ptr(out))
        return None if rc == 1 else out.reshape(-1, 6)


def canonical(directory, headers, cells, coords):
    d = c(directory, np.int32).reshape(-1)
    h = c(headers, np.uint32).reshape(-1)
    cl = c(cells, np.uint32).reshape(-1)
    if cl.size == 0:
        cl = np.zeros(1, np.uint32)
    co = c(coords, np.int32).reshape(-1, 3)
    out = np.zeros((co.shape[0], 4 + 64 * 33), np.uint32)
    rc = lib().orc_canonical(ptr(d), d.size // 4, ptr(h), ptr(cl), cells.size, ptr(co), co.shape[0], ptr(out))
    assert rc == 0, rc
    return out


def discover(geometry, params, eye, forward, up, tan_half_fov, width, height, threads=0):
    """orc_discover: (height, width, 8) per-pixel first-hit records, as the
    GPU's vgi_discover_faces writes them."""
    d, h, cl, _ = geometry
    d = c(d, np.int32)
    cl = c(cl, np.uint32) if len(cl) else np.zeros(1, np.uint32)
    cam = np.array([*eye, *forward, *up, tan_half_fov], np.float32)
    out = np.zeros((height, width, 8), np.uint32)
    rc = lib().orc_discover(ptr(d), d.size // 4, ptr(c(h, np.uint32)), ptr(cl), ptr(c(params, np.float32)), ptr(cam), width, height,
                            ptr(out), threads)
    assert rc == 0
    return out


def discovered_faces(pixels):
    """The distinct hit faces of per-pixel records as (n, 5) rows voxel xyz,
    face, material, sorted by voxel z, y, x and face."""
    p = np.asarray(pixels, np.uint32).reshape(-1, 8)
    p = p[p[:, 3] < 6]
    rows = np.stack([p[:, 0].view(np.int32), p[:, 1].view(np.int32), p[:, 2].view(np.int32), p[:, 3].astype(np.int32),
                     p[:, 4].astype(np.int32)], 1)
    rows = np.unique(rows, axis=0)
    return rows[np.lexsort((rows[:, 3], rows[:, 0], rows[:, 1], rows[:, 2]))]


SUN_FLIP_WORDS = 4 + 2048 * 4 + 7  # the view queue's sun-flip reports


class FarTier:
    """The far tier's host side restated (vgi_far_frame): settings
    normalisation, cell size, the view words, the previous camera and the
    ping-pong of cell histories, with the frame itself run by orc_far_frame."""

    def __init__(self):
        self.cells = [None, None]
        self.output = None
        self.current = 0
        self.shape = None
        self.size = None
        self.previous = None  # (camera words, frame)

    def view_words(self, camera, settings, frame, custom):
        eye, forward, up, tan_half, w, h = camera
        s = settings
        vp = float(np.clip(s.voxel_pixels, 0.0, 4096.0)) if np.isfinite(s.voxel_pixels) else 0.0
        history = float(np.clip(s.history, 1.0, 1024.0)) if np.isfinite(s.history) else 32.0
        rate = min(max(s.rate, 1), 8)
        ratio = np.float32(h) / np.float32(480.0)
        size = min(s.cell, 4) or min(max(int(np.floor(ratio)) + (1 if ratio - np.floor(ratio) >= 0.5 else 0), 1), 4)
        cx, cy = -(-w // size), -(-h // size)
        flags = (1 if vp > 0 else 0) | (s.measure << 1)
        cam = np.array([*eye, *forward, *up, tan_half], np.float32)
        if self.shape != (cx, cy) or self.size != (w, h):
            self.cells = [np.zeros((cx * cy, 12), np.uint32), np.zeros((cx * cy, 12), np.uint32)]
            self.output = np.zeros(16 + 4 * cx * cy, np.uint32)
            self.previous = None
            self.shape, self.size = (cx, cy), (w, h)
        prev_ok = self.previous is not None and ((frame - self.previous[1]) & 0xFFFFFFFF) <= 1
        words = np.zeros(44, np.uint32)
        f = words.view(np.float32)
        f[0:10] = cam
        f[10:20] = self.previous[0] if prev_ok else cam
        words[20:22] = (w, h)
        words[22:26] = (cx, cy, size, flags)
        f[26:29] = (vp, history, float(rate))
        words[29] = self.previous[1] if prev_ok else 0xFFFFFFFF
        f[30:33] = forward
        f[33] = np.float32(np.float32(np.float32(1.0) / np.float32(tan_half)) * np.float32(h)) * np.float32(0.5)
        if s.interest is not None:
            words[34:37] = np.asarray(s.interest[0], np.int32).view(np.uint32)
            words[38:41] = np.asarray(s.interest[1], np.int32).view(np.uint32)
            words[37] = words[41] = 1
        words[42] = frame & 0xFFFFFFFF
        words[43] = 1 if custom else 0
        return words, cam

    def frame(self, geometry, params, materials, lights, emitter_words, pipe, camera, settings, frame, custom=False,
              receivers=None, estimates=None, state=None, index=None, threads=0):
        words, cam = self.view_words(camera, settings, frame, custom)
        d, h, cl, _ = geometry
        d = c(d, np.int32)
        cl = c(cl, np.uint32) if len(cl) else np.zeros(1, np.uint32)
        lights = c(lights, np.float32).reshape(-1)
        if lights.size == 0:
            lights = np.zeros(12, np.float32)
        previous = self.cells[self.current]
        self.current ^= 1
        current = self.cells[self.current]
        stats = np.zeros(8, np.uint32)
        n_recv = 0 if receivers is None else len(receivers)
        rc = lib().orc_far_frame(ptr(d), d.size // 4, ptr(c(h, np.uint32)), ptr(cl), ptr(c(params, np.float32)), ptr(c(materials, np.float32)),
                                 ptr(lights), ptr(c(emitter_words, np.uint32)), ptr(None if state is None else c(state, np.uint32)),
                                 ptr(None if index is None else c(index, np.uint32)), ctypes.byref(pipe), ptr(words),
                                 ptr(None if receivers is None else c(receivers, np.uint32)),
                                 ptr(None if estimates is None else c(estimates, np.uint32)), n_recv, ptr(previous), ptr(current),
                                 ptr(self.output), ptr(stats), threads)
        assert rc == 0
        self.previous = (cam, frame & 0xFFFFFFFF)
        return current, self.output, stats


def _geometry_args(geometry):
    d, h, cl, _ = geometry
    d = c(d, np.int32)
    cl = c(cl, np.uint32) if len(cl) else np.zeros(1, np.uint32)
    return d, c(h, np.uint32), cl


def reconstruct(geometry, params, materials, lights, emitter_words, pipe, receivers, estimates, conts, tile_of, tiles_x, tiles_y,
                display=(0.031, 1.0, 1.0), custom=False):
    """orc_reconstruct: (estimates after, published (n, 12), counters (5,))."""
    d, h, cl = _geometry_args(geometry)
    lights = c(lights, np.float32).reshape(-1)
    if lights.size == 0:
        lights = np.zeros(12, np.float32)
    est = np.array(estimates, np.uint32).reshape(-1, 16).copy()
    n = est.shape[0]
    published = np.zeros((n, 12), np.uint32)
    stats = np.zeros(5, np.uint32)
    rc = lib().orc_reconstruct(ptr(d), d.size // 4, ptr(h), ptr(cl), ptr(c(params, np.float32)), ptr(c(materials, np.float32)), ptr(lights),
                               ptr(c(emitter_words, np.uint32)), ctypes.byref(pipe), ptr(c(receivers, np.uint32)), ptr(est),
                               ptr(c(conts, np.uint32)), ptr(c(tile_of, np.uint32)), tiles_x, tiles_y, n,
                               ptr(np.asarray(display, np.float32)), 1 if custom else 0, ptr(published), ptr(stats))
    assert rc == 0
    return est, published, stats


def corner_value(center, edge_u=None, edge_v=None, diagonal=None):
    """orc_corner_value on (rgb, weight) pairs; None = no face (weight 0)."""
    def w(x):
        if x is None:
            return np.zeros(4, np.float32)
        value, weight = x
        rgb = np.broadcast_to(np.float32(value), 3) if np.ndim(value) == 0 else np.asarray(value, np.float32)
        return np.array([*rgb, weight], np.float32)

    out = np.zeros(3, np.float32)
    lib().orc_corner_value(ptr(w(center)), ptr(w(edge_u)), ptr(w(edge_v)), ptr(w(diagonal)), ptr(out))
    return out


def present(geometry, params, published, eye, forward, up, tan_half_fov, width, height, corners=True, threads=0):
    d, h, cl = _geometry_args(geometry)
    p = c(published, np.uint32).reshape(-1, 12)
    cam = np.array([*eye, *forward, *up, tan_half_fov], np.float32)
    out = np.zeros((height, width, 4), np.float32)
    rc = lib().orc_present(ptr(d), d.size // 4, ptr(h), ptr(cl), ptr(c(params, np.float32)), ptr(p if p.size else np.zeros(12, np.uint32)),
                           p.shape[0], ptr(cam), width, height, 1 if corners else 0, ptr(out), threads)
    assert rc == 0
    return out


# ---- model words ------------------------------------------------------------

def params_words(n_tasks, samples, dir_slots, n_lights, bounds, n_directional, environment=(0, 0, 0), emitter_total=0.0,
                 emitter_count=0, reach=768.0):
    """GpuParams (src/gpu.rs:771-791) as 24 little-endian words in a float32 array."""
    w = np.zeros(24, np.uint32)
    w[0:4] = [n_tasks, samples, dir_slots - 1, n_lights]
    w[4:7] = np.asarray(bounds[:3], np.int32).view(np.uint32)
    w[8:11] = np.asarray(bounds[3:6], np.int32).view(np.uint32)
    w[11] = n_directional
    f = w.view(np.float32)
    f[12:15] = environment
    f[15] = 0.0
    f[16] = 0.0
    f[17] = 768.0
    f[18] = emitter_total
    f[19] = float(emitter_count)
    f[20] = min(max(reach, 1.0), 768.0)
    return f


def emitters(coords, voxels, materials):
    co = c(coords, np.int32).reshape(-1, 3)
    vx = c(voxels, np.uint16).reshape(-1)
    m = c(materials, np.float32).reshape(-1)
    info = np.zeros(3, np.uint32)
    n = lib().orc_emitters(ptr(co), co.shape[0], ptr(vx), ptr(m), None, 0, ptr(info))
    out = np.zeros(n, np.uint32)
    lib().orc_emitters(ptr(co), co.shape[0], ptr(vx), ptr(m), ptr(out), n, ptr(info))
    return out, int(info[0]), float(info[2:3].view(np.float32)[0])


class _TerrainParams(ctypes.Structure):
    _fields_ = [("seed", _U32), ("octaves", _U32), ("period", _F), ("base_height", _F), ("falloff", _F), ("emitters", _U32)]


class _FaceFilter(ctypes.Structure):
    _fields_ = [("use_frustum", _U32), ("eye", _F * 3), ("forward", _F * 3), ("tan_half", _F), ("use_box", _U32),
                ("box_min", ctypes.c_int32 * 3), ("box_max", ctypes.c_int32 * 3), ("use_facing", _U32)]


def grid_coords(nx, ny, nz):
    out = np.zeros((nx * ny * nz, 3), np.int32)
    lib().vgi_scene_grid_coords(nx, ny, nz, ptr(out))
    return out


def stone_room():
    vox = np.zeros(8 * 4096, np.uint16)
    lib().vgi_scene_stone_room(ptr(vox))
    return grid_coords(2, 2, 2), vox


def terrain(nx, ny, nz, seed=2, octaves=4, period=64.0, base_height=96.0, falloff=48.0, emitters=256):
    """The seeded fBm terrain (vgi_scene_terrain), made without libvgi."""
    p = _TerrainParams(seed, octaves, period, base_height, falloff, emitters)
    vox = np.zeros(nx * ny * nz * 4096, np.uint16)
    lib().vgi_scene_terrain(ctypes.byref(p), nx, ny, nz, ptr(vox))
    return grid_coords(nx, ny, nz), vox


def exposed_faces(coords, voxels, facing=None):
    """Exposed faces (voxel xyz, face, material), optionally only those turned
    towards the eye `facing` (vgi_scene_faces), made without libvgi."""
    co = c(coords, np.int32).reshape(-1, 3)
    vx = c(voxels, np.uint16).reshape(-1)
    flt = _FaceFilter()
    if facing is not None:
        flt.use_facing = 1
        flt.eye[:] = list(map(float, facing))
    n = lib().vgi_scene_faces(ptr(co), co.shape[0], ptr(vx), ctypes.byref(flt), None, 0)
    out = np.zeros((max(n, 1), 5), np.int32)
    lib().vgi_scene_faces(ptr(co), co.shape[0], ptr(vx), ctypes.byref(flt), ptr(out), n)
    return out[:n]


def material_words(entries):
    """GpuMaterial words for 256 (diffuse, emission) pairs: the reference's
    VoxelGiMaterials::bounded (src/world.rs:166-173) clamps diffuse to [0, 1]
    and emission to [0, 1e12] (non-finite -> 0); GpuMaterial
    (src/gpu.rs:713-723) puts diffuse in words 0-2, emission in 8-10 and the
    largest emission channel in word 13."""
    out = np.zeros((256, 16), np.float32)
    for m, (diffuse, emission) in enumerate(entries):
        d = np.asarray(diffuse, np.float32)
        e = np.asarray(emission, np.float32)
        d = np.where(np.isfinite(d), np.minimum(np.maximum(d, np.float32(0)), np.float32(1)), np.float32(0))
        e = np.where(np.isfinite(e), np.minimum(np.maximum(e, np.float32(0)), np.float32(1e12)), np.float32(0))
        out[m, 0:3] = d
        out[m, 8:11] = e
        out[m, 13] = max(e[0], max(e[1], e[2]))
    return out.reshape(-1)


def directional_light_words(direction, radiance, custom=(0.0, 0.0, 0.0)):
    """GpuLight words of a directional source (src/gpu.rs:733-744): the
    direction times 1 / length in float32 (glam's normalize_or_zero), range
    -1, radiance, custom visible RGB in words 9-11."""
    d = np.asarray(direction, np.float32)
    length = np.sqrt(np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1])) + np.float32(d[2] * d[2]), dtype=np.float32)
    with np.errstate(divide="ignore"):
        rcp = np.float32(1.0) / np.float32(length)
    out = np.zeros(12, np.float32)
    if np.isfinite(rcp) and rcp > 0:
        out[0:3] = d * rcp
    out[3] = -1.0
    out[4:7] = np.asarray(radiance, np.float32)
    out[9:12] = np.asarray(custom, np.float32)
    return out


def face_index(faces):
    f = c(faces, np.int32).reshape(-1, 4)
    cap = 1024
    while f.shape[0] * 2 > cap:
        cap *= 2
    out = np.zeros((cap * 4 + 1) * 4, np.uint32)
    n = lib().orc_face_index(ptr(f), f.shape[0], ptr(out), out.size // 4)
    assert n > 0
    return out[: n * 4].reshape(-1, 4)


def trace_faces(geometry, params, materials, lights, emitter_words, tasks, pipe: Pipeline, state=None, index=None, threads=0,
                predicted=None):
    """orc_trace_faces; with predicted = (keys (n, 4): voxel xyz, face;
    values (n, 3) rgb), an uncached hit takes the predicted value and ends
    the path (the GPU's MLP cache mode)."""
    if predicted is not None:
        return _trace_faces_predicted(geometry, params, materials, lights, emitter_words, tasks, pipe, state, index, threads,
                                      predicted)
    d, h, cl, _ = geometry
    d = c(d, np.int32)
    h = c(h, np.uint32)
    cl = c(cl, np.uint32) if len(cl) else np.zeros(1, np.uint32)
    t = c(tasks, np.uint32).reshape(-1, 8)
    out = np.zeros((t.shape[0], 24), np.uint32)
    cnt = Counters()
    lights = c(lights, np.float32).reshape(-1)
    if lights.size == 0:
        lights = np.zeros(12, np.float32)
    rc = lib().orc_trace_faces(ptr(d), d.size // 4, ptr(h), ptr(cl), ptr(c(params, np.float32)), ptr(c(materials, np.float32)),
                               ptr(lights), ptr(c(emitter_words, np.uint32)),
                               ptr(None if state is None else c(state, np.uint32)), ptr(None if index is None else c(index, np.uint32)),
                               ptr(t), t.shape[0], ctypes.byref(pipe), ptr(out), ctypes.byref(cnt), threads)
    assert rc == 0
    return out, cnt.as_dict()


def _trace_faces_predicted(geometry, params, materials, lights, emitter_words, tasks, pipe, state, index, threads, predicted):
    d, h, cl, _ = geometry
    d = c(d, np.int32)
    h = c(h, np.uint32)
    cl = c(cl, np.uint32) if len(cl) else np.zeros(1, np.uint32)
    t = c(tasks, np.uint32).reshape(-1, 8)
    keys = c(predicted[0], np.int32).reshape(-1, 4)
    values = c(predicted[1], np.float32).reshape(-1, 3)
    assert keys.shape[0] == values.shape[0]
    out = np.zeros((t.shape[0], 24), np.uint32)
    cnt = Counters()
    lights = c(lights, np.float32).reshape(-1)
    if lights.size == 0:
        lights = np.zeros(12, np.float32)
    rc = lib().orc_trace_faces_predicted(ptr(d), d.size // 4, ptr(h), ptr(cl), ptr(c(params, np.float32)),
                                         ptr(c(materials, np.float32)), ptr(lights), ptr(c(emitter_words, np.uint32)),
                                         ptr(None if state is None else c(state, np.uint32)),
                                         ptr(None if index is None else c(index, np.uint32)), ptr(t), t.shape[0], ctypes.byref(pipe),
                                         ptr(keys), ptr(values), keys.shape[0], ptr(out), ctypes.byref(cnt), threads)
    assert rc == 0
    d = cnt.as_dict()
    last = ctypes.c_uint64(0)
    d["predicted_misses"] = int(lib().orc_predicted_misses(ctypes.byref(last)))
    k = last.value
    d["last_miss"] = (k & 0xffff, (k >> 16) & 0xffff, (k >> 32) & 0xffff, k >> 48)
    return out, d


class OracleShardTracer:
    """The oracle as a face-sharding tracer (the CPU stand-in for a GPU rank
    in the sharding tests). Its gather reads the slots' state rows, so its
    records are whole 36-word state rows."""

    record_words = 36

    def __init__(self, frames: "Frames"):
        self.frames = frames
        self.cache_hits = 0

    def frame_shard(self, samples, clock_ms, first, n):
        self.cache_hits += self.frames.frame_shard(samples, clock_ms, first, n)["cache_hits"]

    def read_cache(self, first, n):
        return self.frames.state[first:first + n].copy()

    def write_cache(self, first, n, records):
        self.frames.state[first:first + n] = np.asarray(records, np.uint32).reshape(n, 36)


def transport_settings(**overrides):
    """The transport fields controls_words reads, with the defaults of
    TransportSettings and TraceWork (src/settings.rs:393-428,
    src/work.rs:11-47), for callers that do not load libvgi."""
    t = types.SimpleNamespace(reach=768.0, bounces=3, path_steps=2048, budgeted=False, history_limit=0, recency=1.0,
                              measured_retention=1.0, response_seconds=0.075, lanes=0, transport_revision=0, stable_error=0.12,
                              stable_samples=32)
    for k, v in overrides.items():
        if not hasattr(t, k):
            raise KeyError(k)
        setattr(t, k, v)
    return t


def controls_words(n, samples, clock_ms, transport, batch_id=1, n_events=0):
    """The Controls words the product's frame uses (src/gpu/resident.rs:708-760)."""
    w = np.zeros(36, np.uint32)
    w[0] = n
    w[1] = samples
    w[2] = clock_ms
    hl = transport.history_limit
    w[3] = 65536 if hl == 0 else min(hl, 65536)
    w[4] = f2u(max(transport.response_seconds, 0.001))
    w[5] = n
    w[10] = f2u(transport.recency if transport.recency >= 1.0 else 1.0)
    w[11] = f2u(max(transport.measured_retention, 0.0))
    w[13] = n_events
    w[14] = n
    w[15] = 192 * 192
    w[16] = transport.transport_revision
    w[17] = f2u(transport.stable_error)
    w[18] = transport.stable_samples
    w[24] = n
    w[25] = batch_id
    w[30] = 64 * 64
    w[31] = 48 * 48
    return w


class Frames:
    """The product's per-frame sequence on the CPU: begin_trace, mark_changed,
    trace (with cache gather), accumulate; state laid out as the reference's
    resident records."""

    def __init__(self, geometry, params_fn, materials, lights, emitter_words, faces, transport, pipe: Pipeline, threads=0):
        self.geometry = geometry
        self.params_fn = params_fn
        self.materials = materials
        self.lights = lights
        self.emitter_words = emitter_words
        self.faces = np.asarray(faces, np.int32).reshape(-1, 5)
        n = self.faces.shape[0]
        self.n = n
        self.transport = transport
        self.pipe = pipe
        self.threads = threads
        self.state = np.zeros((n, 36), np.uint32)
        self.state[:, 28] = np.arange(1, n + 1, dtype=np.uint32)  # slot incarnations
        self.meta = np.zeros((n, 12), np.uint32)
        self.meta[:, 0:3] = self.faces[:, 0:3].view(np.uint32)
        self.meta[:, 3] = self.faces[:, 3].astype(np.uint32) | 8 | (self.faces[:, 4].astype(np.uint32) << 16)
        self.checkpoint = np.zeros((n, 12), np.uint32)
        self.index = face_index(self.faces[:, :4])
        self.tasks = np.zeros((n, 8), np.uint32)
        self.tasks[:, 0:3] = self.faces[:, 0:3].view(np.uint32)
        self.tasks[:, 3] = self.faces[:, 3]
        self.slots = np.arange(n, dtype=np.uint32)
        self.batch_id = 1
        self.results = np.zeros((n, 24), np.uint32)
        self.far_stats = np.zeros(8, np.uint32)

    def frame(self, samples, clock_ms=0, predicted=None, pipe=None):
        """One frame; `predicted` and `pipe` as trace_faces takes them (the
        MLP cache mode's termination and its one-hit pipeline)."""
        ctl = controls_words(self.n, samples, clock_ms, self.transport, self.batch_id)
        L = lib()
        L.orc_begin_trace(ptr(self.state), ptr(self.meta), ptr(self.tasks), ptr(self.slots), self.n, ptr(ctl))
        L.orc_mark_changed(ptr(self.state), ptr(self.meta), ptr(self.slots), self.n, ptr(ctl))
        params = self.params_fn(self.n, samples)
        out, cnt = trace_faces(self.geometry, params, self.materials, self.lights, self.emitter_words, self.tasks, pipe or self.pipe,
                               self.state, self.index, self.threads, predicted)
        L.orc_accumulate(ptr(self.state), ptr(self.meta), ptr(self.checkpoint), ptr(out), ptr(self.slots), self.n, ptr(ctl))
        self.results = out
        self.batch_id = (self.batch_id + 1) & 0x0FFFFFFF or 1
        return cnt

    def frame_slots(self, samples, clock_ms, slots):
        """frame() over the listed slots only (begin_trace, mark_changed,
        trace with the gather over every slot's state, accumulate); the
        other slots keep their state. Returns the counters and the results
        of the listed slots."""
        slots = c(slots, np.uint32)
        n = slots.size
        ctl = controls_words(n, samples, clock_ms, self.transport, self.batch_id)
        L = lib()
        tasks = np.ascontiguousarray(self.tasks[slots])
        L.orc_begin_trace(ptr(self.state), ptr(self.meta), ptr(tasks), ptr(slots), n, ptr(ctl))
        L.orc_mark_changed(ptr(self.state), ptr(self.meta), ptr(slots), n, ptr(ctl))
        params = self.params_fn(n, samples)
        out, cnt = trace_faces(self.geometry, params, self.materials, self.lights, self.emitter_words, tasks, self.pipe, self.state,
                               self.index, self.threads)
        L.orc_accumulate(ptr(self.state), ptr(self.meta), ptr(self.checkpoint), ptr(out), ptr(slots), n, ptr(ctl))
        self.tasks[slots] = tasks
        self.results[slots] = out
        self.batch_id = (self.batch_id + 1) & 0x0FFFFFFF or 1
        return cnt, out

    def frame_shard(self, samples, clock_ms, first, n):
        """frame() over slots [first, first + n) only (vgi_frame_shard)."""
        ctl = controls_words(n, samples, clock_ms, self.transport, self.batch_id)
        L = lib()
        slots = np.arange(first, first + n, dtype=np.uint32)
        tasks = np.ascontiguousarray(self.tasks[first:first + n])
        L.orc_begin_trace(ptr(self.state), ptr(self.meta), ptr(tasks), ptr(slots), n, ptr(ctl))
        L.orc_mark_changed(ptr(self.state), ptr(self.meta), ptr(slots), n, ptr(ctl))
        params = self.params_fn(n, samples)
        out, cnt = trace_faces(self.geometry, params, self.materials, self.lights, self.emitter_words, tasks, self.pipe, self.state,
                               self.index, self.threads)
        L.orc_accumulate(ptr(self.state), ptr(self.meta), ptr(self.checkpoint), ptr(out), ptr(slots), n, ptr(ctl))
        self.tasks[first:first + n] = tasks
        self.results[first:first + n] = out
        self.batch_id = (self.batch_id + 1) & 0x0FFFFFFF or 1
        return cnt

    def view_trace_paths(self, receivers, samples):
        """trace_view_paths over receivers (8 words each) x samples."""
        r = c(receivers, np.uint32).reshape(-1, 8)
        out = np.zeros((r.shape[0] * samples, 32), np.uint32)
        d, h, cl, _ = self.geometry
        params = self.params_fn(self.n, samples)
        lib().orc_trace_view_paths(ptr(d), d.size // 4, ptr(h), ptr(cl), ptr(params), ptr(self.materials), ptr(self.lights),
                                   ptr(self.emitter_words), ptr(self.state), ptr(self.index), ctypes.byref(self.pipe), ptr(r),
                                   r.shape[0], samples, ptr(out))
        return out

    def view_start(self, receivers, materials):
        """A view tier over `receivers` (8 words each, as vgi_view_read
        returns them) with empty estimates of the given materials."""
        n = receivers.shape[0]
        self.view = {"receivers": c(receivers, np.uint32).copy(), "paths": np.zeros((n, 32), np.uint32),
                     "continuations": np.zeros((n, 32), np.uint32), "estimates": np.zeros((n, 16), np.uint32),
                     "queue": np.zeros(12 + 2 * n + SUN_FLIP_WORDS, np.uint32)}
        self.view["estimates"][:, 13] = materials
        self.view_frames = 0
        lib().orc_sun_flip_log_clear()

    def view_read_sun_flips(self):
        """vgi_view_read_sun_flips on the oracle: (records (up to 2048, 4),
        overflow (7,), every flip since the last read (n, 4)), clearing the
        region and the log as the library's read does."""
        n = self.view["receivers"].shape[0]
        region = self.view["queue"][12 + 2 * n:]
        count = int(region[0])
        records = region[4:4 + 4 * min(count, 2048)].reshape(-1, 4).copy()
        overflow = region[4 + 2048 * 4:].copy()
        total = int(lib().orc_sun_flip_log(None, 0))
        log = np.zeros((total, 4), np.uint32)
        lib().orc_sun_flip_log(ptr(log), total)
        assert total == count, (total, count)
        region[:] = 0
        lib().orc_sun_flip_log_clear()
        return records, overflow, log

    def view_frame(self, first=0, invocations=0, max_hits=8, depth=0, ticket=(0, 0, 0, 0), view_first=False, shared=True,
                   clock_ms=0, events=None, n_events=0, measured_retention=1.0, far=None, topology=False):
        """far = (44 far-tier view words, cells (n, 12)) turns on the far
        handoff; self.far_stats[5] counts the receivers it seeds."""
        v = self.view
        n = v["receivers"].shape[0]
        wave = np.array([first, invocations or n, max_hits, depth, *ticket], np.uint32)
        frames = getattr(self, "view_frames", 0)
        view = np.array([int(view_first), int(shared and self.n > 0), clock_ms, n_events, 192 * 192, 0, int(topology), frames,
                         int(frames > 0)], np.uint32)
        self.view_frames = frames + 1
        view[5] = np.float32(max(measured_retention, 0.0)).view(np.uint32)
        ev = np.zeros(4, np.uint32) if events is None else c(events, np.uint32)
        d, h, cl, _ = self.geometry
        params = self.params_fn(self.n, 1)
        lib().orc_view_frame(ptr(d), d.size // 4, ptr(h), ptr(cl), ptr(params), ptr(self.materials), ptr(self.lights),
                             ptr(self.emitter_words), ptr(self.state), ptr(self.meta), ptr(self.index), ctypes.byref(self.pipe),
                             ptr(v["receivers"]), n, ptr(v["paths"]), ptr(v["continuations"]), ptr(v["estimates"]), ptr(v["queue"]),
                             ptr(wave), ptr(view), ptr(ev), ptr(None if far is None else c(far[0], np.uint32)),
                             ptr(None if far is None else c(far[1], np.uint32)), ptr(self.far_stats))

    def measure_edits(self, words, measures, n_entries, material_light):
        """measure_edits + finish_edits on a copy of the event words."""
        w = c(words, np.uint32).copy()
        m = c(measures, np.uint32)
        ml = c(material_light, np.float32)
        lib().orc_measure_edits(ptr(self.state), ptr(self.meta), ptr(self.index), ptr(ml), ptr(m), n_entries, ptr(w))
        return w

    def apply_events(self, words, n_events):
        ctl = controls_words(self.n, 0, 0, self.transport, self.batch_id, n_events)
        w = c(words, np.uint32)
        lib().orc_apply_events(ptr(self.state), ptr(self.meta), ptr(self.checkpoint), ptr(w), self.n, ptr(ctl))


def resolve_retention(events, receiver, reach=192 * 192, measured=True):
    """orc_resolve_retention: (history cap, predicted change or None when some
    change in range has unknown flux, woken) for one receiver voxel over
    events in the encode_events layout (words, count)."""
    words, n = events
    w = c(words, np.uint32).reshape(-1) if len(words) else np.zeros(4, np.uint32)
    p = c(receiver, np.int32).reshape(3)
    lim = ctypes.c_uint32()
    change = ctypes.c_float()
    flags = ctypes.c_uint32()
    assert lib().orc_resolve_retention(ptr(w), n, ptr(p), reach, 1 if measured else 0, ctypes.byref(lim), ctypes.byref(change),
                                       ctypes.byref(flags)) == 0
    return lim.value, (change.value if flags.value & 1 else None), bool(flags.value & 2)
