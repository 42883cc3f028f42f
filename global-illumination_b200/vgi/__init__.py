"""Python binding of libvgi (include/vgi.h) for tests, benchmarks and tools.

The host-side names mirror bevy_voxel_gi's interface for this path
(crates/bevy_voxel_gi/src/): ``MaterialTransport`` / ``VoxelGiMaterials``
(world.rs:59-175), ``TransportSettings`` (settings.rs:393-428),
``DirectionalTransportLight`` (sources.rs:38-45) and ``GpuTracer``
(gpu.rs:309-1240), whose methods map one-to-one onto the C ABI. Every call
goes through the CUDA library; there is no CPU fallback, and loading fails
loudly when libvgi.so has not been built.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(os.path.dirname(_HERE), "libvgi.so")

OK = 0
UNAVAILABLE = 1
ERR_INVALID = -1
ERR_CUDA = -2
ERR_STATE = -3
ERR_CAPACITY = -4

INJECT_ALLOC = 1
INJECT_UPLOAD = 2
MLP_WAIT_DEFAULT = 0xFFFFFFFF

AIR = 256
FACE_OFFSETS = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


class VgiError(RuntimeError):
    """A libvgi call returned a failure status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libvgi status {status}: {message}")
        self.status = status


class TransportUnavailable(VgiError):
    """No usable CUDA device: the reference idles transport in this case
    (src/lib.rs:355-357); it never falls back to the CPU."""


class Camera(ctypes.Structure):
    """vgi_camera."""
    _fields_ = [("eye", ctypes.c_float * 3), ("forward", ctypes.c_float * 3), ("up", ctypes.c_float * 3), ("tan_half_fov", ctypes.c_float),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class ViewDisplay(ctypes.Structure):
    """vgi_view_display."""
    _fields_ = [("evidence_goal", ctypes.c_float), ("spatial", ctypes.c_float), ("temporal", ctypes.c_float)]


def witness_tiles(pixels: np.ndarray, faces: np.ndarray, grid_x: int, grid_y: int) -> np.ndarray:
    """Each receiver's screen tile from discovery's per-pixel records (h, w,
    8): the first pixel in raster order that saw its face is its witness;
    its cell is pixel * grid / viewport and its tile the 2 x 2-cell tile
    (tile_of_pixel, voxel_view_discovery.wgsl:160-165). All ones: never
    seen. Tiles are ((grid_x + 1) // 2) x ((grid_y + 1) // 2)."""
    h, w = pixels.shape[:2]
    p = np.asarray(pixels, np.uint32).reshape(-1, 8)

    def key(x, y, z, f):
        m = np.uint64(0xFFFFF)
        return ((x.astype(np.uint64) & m) | ((y.astype(np.uint64) & m) << np.uint64(20)) | ((z.astype(np.uint64) & m) << np.uint64(40))
                | (f.astype(np.uint64) << np.uint64(60)))

    hit = np.nonzero(p[:, 3] < 6)[0]
    seen, first = np.unique(key(p[hit, 0], p[hit, 1], p[hit, 2], p[hit, 3]), return_index=True)
    first = hit[first]  # np.unique keeps each key's first occurrence: the first pixel in raster order
    f = np.asarray(faces, np.int32).reshape(-1, 5).view(np.uint32)
    k = key(f[:, 0], f[:, 1], f[:, 2], f[:, 3])
    at = np.minimum(np.searchsorted(seen, k), max(len(seen) - 1, 0))
    found = (len(seen) > 0) & (seen[at] == k) if len(seen) else np.zeros(len(k), bool)
    out = np.full(len(k), 0xFFFFFFFF, np.uint32)
    i = first[at[found]]
    cx = np.minimum((i % w) * grid_x // w, grid_x - 1)
    cy = np.minimum((i // w) * grid_y // h, grid_y - 1)
    out[found] = ((cy // 2) * ((grid_x + 1) // 2) + cx // 2).astype(np.uint32)
    return out


class FarSettingsStruct(ctypes.Structure):
    """vgi_far_settings."""
    _fields_ = [("voxel_pixels", ctypes.c_float), ("measure", ctypes.c_uint32), ("cell", ctypes.c_uint32), ("history", ctypes.c_float),
                ("rate", ctypes.c_uint32), ("steps", ctypes.c_uint32), ("interest_min", ctypes.c_int32 * 3),
                ("interest_max", ctypes.c_int32 * 3), ("bounded", ctypes.c_uint32)]


@dataclasses.dataclass
class FarTierSettings:
    """FarTierSettings (src/settings.rs:95-137) with its defaults; measure
    0 = voxel side, 1 = voxel area, 2 = block area; interest = (min, max)
    region coordinates or None."""

    voxel_pixels: float = 8.0
    measure: int = 0
    cell: int = 0
    history: float = 32.0
    rate: int = 4
    steps: int = 128
    interest: Optional[tuple] = None

    def struct(self) -> FarSettingsStruct:
        lo, hi = self.interest if self.interest is not None else ((0, 0, 0), (0, 0, 0))
        return FarSettingsStruct(self.voxel_pixels, self.measure, self.cell, self.history, self.rate, self.steps,
                                 (ctypes.c_int32 * 3)(*lo), (ctypes.c_int32 * 3)(*hi), 1 if self.interest is not None else 0)


class Schedule(ctypes.Structure):
    """vgi_schedule."""
    _fields_ = [("focus", ctypes.c_int32 * 3), ("budget", ctypes.c_uint32), ("classify_first", ctypes.c_uint32),
                ("classify_end", ctypes.c_uint32), ("audit_ms", ctypes.c_uint32)]


class MlpStatus(ctypes.Structure):
    """vgi_mlp_status."""
    _fields_ = [("frames", ctypes.c_uint32), ("steps", ctypes.c_uint32), ("terminating", ctypes.c_uint32),
                ("queries", ctypes.c_uint32), ("loss", ctypes.c_float), ("error", ctypes.c_uint32),
                ("query_ms", ctypes.c_float), ("train_ms", ctypes.c_float)]


class Counters(ctypes.Structure):
    _fields_ = [
        ("rays", ctypes.c_uint64),
        ("paths", ctypes.c_uint64),
        ("steps", ctypes.c_uint64),
        ("bytes", ctypes.c_uint64),
        ("unknown", ctypes.c_uint64),
        ("cache_hits", ctypes.c_uint64),
        ("status", ctypes.c_uint64 * 4),
        ("traverse_bytes", ctypes.c_uint64),
        ("warp_passes", ctypes.c_uint64 * 2),
        ("lane_passes", ctypes.c_uint64 * 2),
    ]

    def as_dict(self) -> dict:
        d = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            d[k] = int(v) if isinstance(v, int) else [int(x) for x in v]
        return d


class ViewWave(ctypes.Structure):
    """vgi_view_wave: one view frame's ViewWave range, ticket and view controls."""
    _fields_ = [
        ("first", ctypes.c_uint32),
        ("invocations", ctypes.c_uint32),
        ("max_hits", ctypes.c_uint32),
        ("depth", ctypes.c_uint32),
        ("ticket", ctypes.c_uint32 * 4),
        ("view_first", ctypes.c_uint32),
        ("shared", ctypes.c_uint32),
        ("clock_ms", ctypes.c_uint32),
    ]


class _Transport(ctypes.Structure):
    _fields_ = [
        ("reach", ctypes.c_float),
        ("bounces", ctypes.c_uint32),
        ("path_steps", ctypes.c_uint32),
        ("budgeted", ctypes.c_uint32),
        ("history_limit", ctypes.c_uint32),
        ("recency", ctypes.c_float),
        ("measured_retention", ctypes.c_float),
        ("response_seconds", ctypes.c_float),
        ("lanes", ctypes.c_uint32),
        ("transport_revision", ctypes.c_uint32),
        ("stable_error", ctypes.c_float),
        ("stable_samples", ctypes.c_uint32),
    ]


class _Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("flags", ctypes.c_uint32)]


class TerrainParams(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint32),
        ("octaves", ctypes.c_uint32),
        ("period", ctypes.c_float),
        ("base_height", ctypes.c_float),
        ("falloff", ctypes.c_float),
        ("emitters", ctypes.c_uint32),
    ]


class FaceFilter(ctypes.Structure):
    _fields_ = [
        ("use_frustum", ctypes.c_uint32),
        ("eye", ctypes.c_float * 3),
        ("forward", ctypes.c_float * 3),
        ("tan_half", ctypes.c_float),
        ("use_box", ctypes.c_uint32),
        ("box_min", ctypes.c_int32 * 3),
        ("box_max", ctypes.c_int32 * 3),
        ("use_facing", ctypes.c_uint32),
    ]


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I64 = ctypes.c_int64
_INT = ctypes.c_int
_F = ctypes.c_float

_SIGNATURES = {
    "vgi_create": (_INT, [_P, _P]),
    "vgi_destroy": (_INT, [_P]),
    "vgi_last_error": (ctypes.c_char_p, [_P]),
    "vgi_stream": (_INT, [_P, _P]),
    "vgi_sync": (_INT, [_P]),
    "vgi_upload_regions": (_INT, [_P, _P, _U32, _P, _P]),
    "vgi_upload_packed": (_INT, [_P, _P, _U64, _P, _U32, _P, _U64, _P]),
    "vgi_patch_packed": (_INT, [_P, _U64, _U32, _U64, _P, _INT, _P, _U32, _P, _P, _U32, _P, _P, _U32, _P]),
    "vgi_edit_voxels": (_INT, [_P, _P, _U32]),
    "vgi_load_regions": (_INT, [_P, _P, _U32, _P, _P]),
    "vgi_unload_regions": (_INT, [_P, _P, _U32]),
    "vgi_update_regions": (_INT, [_P, _P, _U32, _P, _P, _P, _U32]),
    "vgi_geometry_info": (_INT, [_P, _P, _P]),
    "vgi_read_geometry": (_INT, [_P, _P, _P, _P]),
    "vgi_set_materials": (_INT, [_P, _P]),
    "vgi_set_lights": (_INT, [_P, _P, _U32, _U32]),
    "vgi_set_environment": (_INT, [_P, _P]),
    "vgi_set_emitters": (_INT, [_P, _P, _U64, _U32, _F]),
    "vgi_build_emitters": (_INT, [_P]),
    "vgi_set_transport": (_INT, [_P, _P]),
    "vgi_set_faces": (_INT, [_P, _P, _U32]),
    "vgi_frame": (_INT, [_P, _U32, _U32]),
    "vgi_set_timing": (_INT, [_P, _INT]),
    "vgi_set_graph": (_INT, [_P, _INT]),
    "vgi_autotune": (_INT, [_P, _U32, _P, _P, _P]),
    "vgi_set_layout": (_INT, [_P, _U32, _U32]),
    "vgi_pack_regions_static": (_INT, [_P, _U32, _P, _P, _U64, _P, _P]),
    "vgi_frame_times": (_INT, [_P, _P]),
    "vgi_trace_batch": (_INT, [_P, _P, _U32, _U32, _U32, _P]),
    "vgi_census": (_INT, [_P, _U32, _P]),
    "vgi_trace_tasks": (_INT, [_P, _P, _U32, _U32, _P, _P]),
    "vgi_apply_events": (_INT, [_P, _P, _U32, _U64]),
    "vgi_apply_events_measured": (_INT, [_P, _P, _U32, _U64, _P, _U32]),
    "vgi_read_events": (_INT, [_P, _P, _U64]),
    "vgi_view_set_receivers": (_INT, [_P, _P, _U32]),
    "vgi_view_frame": (_INT, [_P, _P, _P, _U32, _U64]),
    "vgi_view_read": (_INT, [_P, _P, _P, _P, _P, _P]),
    "vgi_view_trace_paths": (_INT, [_P, _U32, _P]),
    "vgi_reference_fp64": (_INT, [_P, _P, _U32, _U32, _U64, _P, _P, _P]),
    "vgi_mlp_set_weights": (_INT, [_P, _P, _U32]),
    "vgi_mlp_get_weights": (_INT, [_P, _P, _U32]),
    "vgi_mlp_forward": (_INT, [_P, _P, _U32, _P]),
    "vgi_mlp_gradients": (_INT, [_P, _P, _P, _U32, _P, _P]),
    "vgi_mlp_train": (_INT, [_P, _P, _P, _U32, ctypes.c_float, _P]),
    "vgi_mlp_apply_gradients": (_INT, [_P, _P, ctypes.c_float, ctypes.c_float, _INT]),
    "vgi_mlp_encode": (_INT, [_P, _P, _U32, _P]),
    "vgi_set_mlp_cache": (_INT, [_P, ctypes.c_int, _U32, _U32, _U32, ctypes.c_float]),
    "vgi_set_mlp_schedule": (_INT, [_P, _U32, ctypes.c_float]),
    "vgi_mlp_stats": (_INT, [_P, _P]),
    "vgi_frame_shard": (_INT, [_P, _U32, _U32, _U32, _U32]),
    "vgi_submit_batch": (_INT, [_P, _P, _U32, _U32, _U32, _P, _P]),
    "vgi_frame_scheduled": (_INT, [_P, _U32, _U32, _P]),
    "vgi_discover_faces": (_INT, [_P, _P, _P, _P, _U32, _P]),
    "vgi_scene_cave": (None, [_P, _U32, _U32, _U32, _P]),
    "vgi_far_frame": (_INT, [_P, _P, _P, _U32]),
    "vgi_far_read": (_INT, [_P, _P, _P, _P, _P]),
    "vgi_far_reset": (_INT, [_P]),
    "vgi_set_far_handoff": (_INT, [_P, _INT]),
    "vgi_set_topology_prior": (_INT, [_P, _INT]),
    "vgi_view_read_sun_flips": (_INT, [_P, _P]),
    "vgi_mlp_set_wait_limit": (_INT, [_P, _U32]),
    "vgi_inject_failure": (_INT, [_P, _U32, _U32]),
    "vgi_view_set_tiles": (_INT, [_P, _P, _U32, _U32, _U32]),
    "vgi_view_reconstruct": (_INT, [_P, _P]),
    "vgi_view_read_published": (_INT, [_P, _P, _P]),
    "vgi_view_present": (_INT, [_P, _P, _INT, _P]),
    "vgi_apply_events_footprints": (_INT, [_P, _P, _U32, _U64, _P, _U32, _P, _U32]),
    "vgi_read_selection": (_INT, [_P, _P, _P, _P, _P, _P]),
    "vgi_complete_batch": (_INT, [_P, _U64]),
    "vgi_read_cache": (_INT, [_P, _U32, _U32, _P, ctypes.c_int]),
    "vgi_write_cache": (_INT, [_P, _U32, _U32, _P, ctypes.c_int]),
    "vgi_batch_create": (_INT, [_P, _U32, _P]),
    "vgi_batch_destroy": (_INT, [_P]),
    "vgi_batch_last_error": (ctypes.c_char_p, [_P]),
    "vgi_batch_frame": (_INT, [_P, _U32, _U32]),
    "vgi_batch_set_graph": (_INT, [_P, ctypes.c_int]),
    "vgi_batch_sync": (_INT, [_P]),
    "vgi_batch_autotune": (_INT, [_P, _U32, _P, _P, _P]),
    "vgi_read_results": (_INT, [_P, _U32, _U32, _P]),
    "vgi_read_state": (_INT, [_P, _U32, _U32, _P]),
    "vgi_write_state": (_INT, [_P, _U32, _U32, _P]),
    "vgi_read_slot_meta": (_INT, [_P, _U32, _U32, _P]),
    "vgi_material_record": (None, [_P, _P, _P]),
    "vgi_directional_light_record": (None, [_P, _P, _P, _P]),
    "vgi_host_emitters": (_I64, [_P, _U32, _P, _P, _P, _U64, _P]),
    "vgi_host_face_index": (_I64, [_P, _U32, _P, _U64]),
    "vgi_host_top_level": (_INT, [_P, _P, _U32, _P, _U64]),
    "vgi_scene_grid_coords": (_U32, [_U32, _U32, _U32, _P]),
    "vgi_scene_stone_room": (None, [_P]),
    "vgi_scene_furnace": (None, [_P]),
    "vgi_scene_terrain": (None, [_P, _U32, _U32, _U32, _P]),
    "vgi_scene_faces": (_U64, [_P, _U32, _P, _P, _P, _U64]),
}

_lib = None


def library() -> ctypes.CDLL:
    """Loads libvgi.so (built in-tree by ``make -C global-illumination_b200``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise FileNotFoundError(f"{LIBRARY_PATH} is missing: build it with make -C {os.path.dirname(LIBRARY_PATH)}")
        lib = ctypes.CDLL(LIBRARY_PATH)
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to libvgi must be contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


# ---- host-side mirror of the reference's model types --------------------------

def encode_edit_events(edits):
    """Retention events for voxel edits, as encode_events packs them
    (src/gpu/resident.rs:1320-1414): one event per edited box, `edits` a
    list of (lo xyz, hi xyz, changed voxels, flux). Each bound is a measured
    edit (kind 6): its measure record asks measure_edits for the one-voxel
    margin scan around the box, which sets the flux. Returns (event words,
    event count, measure records) for GpuTracer.apply_events_measured."""
    head, bounds, measures = [], [], []
    n = len(edits)
    positions = 0
    for k, (lo, hi, voxels, flux) in enumerate(edits):
        lo = [int(v) for v in lo]
        hi = [int(v) for v in hi]
        head += [[lo[0], lo[1], lo[2], 0], [hi[0], hi[1], hi[2], 0], [0, 0, k, 1]]
        f = int(np.float32(flux).view(np.uint32))
        bounds += [[lo[0], lo[1], lo[2], f], [hi[0], hi[1], hi[2], 6]]
        size = [hi[a] - lo[a] + 3 for a in range(3)]
        count = size[0] * size[1] * size[2]
        measures += [[3 * n + 2 * k, positions, count, int(voxels)], [lo[0] - 1, lo[1] - 1, lo[2] - 1, f], [*size, 0]]
        positions += count
    words = np.array(head + bounds, np.int64).reshape(-1).astype(np.uint32)
    return words, n, np.array(measures, np.int64).reshape(-1, 4).astype(np.uint32).reshape(-1, 12) if measures else np.zeros((0, 12), np.uint32)


@dataclasses.dataclass
class MaterialTransport:
    """A transport material's optics (src/world.rs:59-79)."""

    diffuse: Sequence[float] = (0.45, 0.45, 0.45)
    emission: Sequence[float] = (0.0, 0.0, 0.0)


class VoxelGiMaterials:
    """The 256 transport materials (src/world.rs:90-175); unassigned ones keep
    the default optics. ``words()`` is the GpuMaterial table the GPU reads."""

    def __init__(self):
        self.entries = [MaterialTransport() for _ in range(256)]
        self.assigned = [False] * 256

    def set(self, material: int, transport: MaterialTransport) -> None:
        self.entries[material] = transport
        self.assigned[material] = True

    def get(self, material: int) -> MaterialTransport:
        return self.entries[material]

    def insert(self, transport: MaterialTransport) -> int:
        for m in range(256):
            if self.assigned[m] and self.words_of(self.entries[m]).tobytes() == self.words_of(transport).tobytes():
                return m
        for m in range(256):
            if not self.assigned[m]:
                self.set(m, transport)
                return m
        raise ValueError("MaterialsFull: all 256 materials are assigned")

    @staticmethod
    def words_of(t: MaterialTransport) -> np.ndarray:
        out = np.zeros(16, np.float32)
        library().vgi_material_record(_ptr(_c(t.diffuse, np.float32)), _ptr(_c(t.emission, np.float32)), _ptr(out))
        return out

    def words(self) -> np.ndarray:
        return np.concatenate([self.words_of(e) for e in self.entries]).astype(np.float32)


@dataclasses.dataclass
class DirectionalTransportLight:
    """A directional source (src/sources.rs:38-45): direction towards the light."""

    direction: Sequence[float]
    radiance: Sequence[float]
    custom_visible: Sequence[float] = (0.0, 0.0, 0.0)

    def words(self) -> np.ndarray:
        out = np.zeros(12, np.float32)
        library().vgi_directional_light_record(_ptr(_c(self.direction, np.float32)), _ptr(_c(self.radiance, np.float32)),
                                               _ptr(_c(self.custom_visible, np.float32)), _ptr(out))
        return out


@dataclasses.dataclass
class PointTransportLight:
    """A point source (src/gpu.rs:745-753): position and range, intensity,
    custom visible RGB in extra.yzw."""

    position: Sequence[float]
    intensity: Sequence[float]
    range: float
    custom_visible: Sequence[float] = (0.0, 0.0, 0.0)

    def words(self) -> np.ndarray:
        out = np.zeros(12, np.float32)
        out[0:3] = self.position
        out[3] = self.range
        out[4:7] = self.intensity
        out[9:12] = self.custom_visible
        return out


@dataclasses.dataclass
class TransportSettings:
    """TransportSettings (src/settings.rs:393-428) plus the accumulation
    fields of TraceWork (src/work.rs:11-47) and the shader overrides."""

    reach: float = 768.0
    bounces: int = 3
    path_steps: int = 2048
    budgeted: bool = False
    history_limit: int = 0
    recency: float = 1.0
    measured_retention: float = 1.0
    response_seconds: float = 0.075
    lanes: int = 0
    transport_revision: int = 0
    stable_error: float = 0.12
    stable_samples: int = 32

    def _c(self) -> _Transport:
        return _Transport(self.reach, self.bounces, self.path_steps, int(self.budgeted), self.history_limit, self.recency,
                          self.measured_retention, self.response_seconds, self.lanes, self.transport_revision,
                          self.stable_error, self.stable_samples)


class GpuTracer:
    """One libvgi context: the B200 counterpart of the reference's GpuTracer."""

    def __init__(self, device: int = 0):
        lib = library()
        handle = ctypes.c_void_p()
        cfg = _Config(device, 0)
        rc = lib.vgi_create(ctypes.byref(cfg), ctypes.byref(handle))
        if rc == UNAVAILABLE:
            raise TransportUnavailable(rc, "no CUDA device")
        if rc != OK:
            raise VgiError(rc, "vgi_create failed")
        self._h = handle
        self._lib = lib
        self.n_slots = 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.vgi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        if rc != OK:
            raise VgiError(rc, self._lib.vgi_last_error(self._h).decode())

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.vgi_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def sync(self) -> None:
        self._check(self._lib.vgi_sync(self._h))

    # geometry
    def upload_regions(self, coords: np.ndarray, voxels: np.ndarray, strides: Optional[np.ndarray] = None) -> None:
        coords = _c(coords, np.int32).reshape(-1, 3)
        voxels = _c(voxels, np.uint16).reshape(-1)
        assert voxels.size == coords.shape[0] * 4096
        st = None if strides is None else _c(strides, np.uint8)
        self._check(self._lib.vgi_upload_regions(self._h, _ptr(coords), coords.shape[0], _ptr(voxels), _ptr(st)))

    def upload_packed(self, directory, headers, cells, bounds) -> None:
        d = _c(directory, np.int32).reshape(-1)
        h = _c(headers, np.uint32).reshape(-1)
        c = _c(cells, np.uint32).reshape(-1)
        b = _c(bounds, np.int32).reshape(-1)
        self._check(self._lib.vgi_upload_packed(self._h, _ptr(d), d.size // 4, _ptr(h), h.size // 4, _ptr(c), c.size, _ptr(b)))

    def patch_packed(self, lengths, bounds, directory_rebuilt: bool, directory, headers, cells) -> None:
        """A SceneDelta on packed geometry (synchronize_geometry): `lengths`
        = (directory slots, headers, cells) after the change; `directory`,
        `headers`, `cells` are lists of (start, elements) with elements
        shaped (k, 4) int32, (k, 4) uint32 and (k,) uint32; with
        directory_rebuilt, `directory` is the whole new directory instead."""

        def pack(parts, dtype, width):
            ranges = np.array([[start, len(np.asarray(e).reshape(-1, width))] for start, e in parts], np.uint64).reshape(-1)
            data = np.concatenate([_c(e, dtype).reshape(-1) for _, e in parts]) if parts else np.zeros(0, dtype)
            return ranges, data

        b = _c(bounds, np.int32).reshape(-1)
        if directory_rebuilt:
            d_ranges, d_data = np.zeros(0, np.uint64), _c(directory, np.int32).reshape(-1)
            n_d = 0
        else:
            d_ranges, d_data = pack(directory, np.int32, 4)
            n_d = d_ranges.size // 2
        h_ranges, h_data = pack(headers, np.uint32, 4)
        c_ranges, c_data = pack(cells, np.uint32, 1)
        d_data, h_data, c_data = (np.ascontiguousarray(x) for x in (d_data, h_data, c_data))
        self._check(self._lib.vgi_patch_packed(
            self._h, int(lengths[0]), int(lengths[1]), int(lengths[2]), _ptr(b), 1 if directory_rebuilt else 0,
            _ptr(d_ranges), n_d, _ptr(d_data), _ptr(h_ranges), h_ranges.size // 2, _ptr(h_data),
            _ptr(c_ranges), c_ranges.size // 2, _ptr(c_data)))

    def load_regions(self, coords: np.ndarray, voxels: np.ndarray, strides: Optional[np.ndarray] = None) -> None:
        """page_loaded / page_changed: regions (coords n x 3, voxels n x 4096)
        loaded into the GPU geometry, replacing resident ones."""
        c = _c(coords, np.int32).reshape(-1, 3)
        v = _c(voxels, np.uint16).reshape(-1)
        assert v.size == c.shape[0] * 4096
        st = None if strides is None else _c(strides, np.uint8)
        self._check(self._lib.vgi_load_regions(self._h, _ptr(c), c.shape[0], _ptr(v), _ptr(st)))

    def unload_regions(self, coords: np.ndarray) -> None:
        """page_unloaded: regions removed from the GPU geometry."""
        c = _c(coords, np.int32).reshape(-1, 3)
        self._check(self._lib.vgi_unload_regions(self._h, _ptr(c), c.shape[0]))

    def update_regions(self, coords: np.ndarray, voxels: np.ndarray, removed: np.ndarray,
                       strides: Optional[np.ndarray] = None) -> None:
        """One frame's page events as one scene change (with_page_contents):
        `removed` regions unloaded, then `coords`/`voxels` loaded."""
        c = _c(coords, np.int32).reshape(-1, 3)
        v = _c(voxels, np.uint16).reshape(-1)
        assert v.size == c.shape[0] * 4096
        r = _c(removed, np.int32).reshape(-1, 3)
        st = None if strides is None else _c(strides, np.uint8)
        self._check(self._lib.vgi_update_regions(self._h, _ptr(c), c.shape[0], _ptr(v), _ptr(st), _ptr(r), r.shape[0]))

    def edit_voxels(self, edits: np.ndarray) -> None:
        e = _c(edits, np.int32).reshape(-1, 4)
        self._check(self._lib.vgi_edit_voxels(self._h, _ptr(e), e.shape[0]))

    def geometry(self):
        sizes = np.zeros(3, np.uint64)
        bounds = np.zeros(6, np.int32)
        self._check(self._lib.vgi_geometry_info(self._h, _ptr(sizes), _ptr(bounds)))
        d = np.zeros(int(sizes[0]) * 4, np.int32)
        h = np.zeros(int(sizes[1]) * 4, np.uint32)
        c = np.zeros(max(int(sizes[2]), 1), np.uint32)
        self._check(self._lib.vgi_read_geometry(self._h, _ptr(d), _ptr(h), _ptr(c)))
        return d, h, c[: int(sizes[2])], bounds

    # model
    def set_materials(self, words: np.ndarray) -> None:
        w = _c(words, np.float32).reshape(-1)
        assert w.size == 256 * 16
        self._check(self._lib.vgi_set_materials(self._h, _ptr(w)))

    def set_lights(self, words: np.ndarray, n_directional: int) -> None:
        w = _c(words, np.float32).reshape(-1)
        self._check(self._lib.vgi_set_lights(self._h, _ptr(w), w.size // 12, n_directional))

    def set_environment(self, rgb) -> None:
        self._check(self._lib.vgi_set_environment(self._h, _ptr(_c(rgb, np.float32))))

    def set_emitters(self, words: np.ndarray, n_faces: int, total_weight: float) -> None:
        w = _c(words, np.uint32).reshape(-1)
        self._check(self._lib.vgi_set_emitters(self._h, _ptr(w), w.size, n_faces, total_weight))

    def build_emitters(self) -> None:
        self._check(self._lib.vgi_build_emitters(self._h))

    def set_transport(self, t: TransportSettings) -> None:
        tc = t._c()
        self._check(self._lib.vgi_set_transport(self._h, ctypes.byref(tc)))

    # face cache
    def set_faces(self, faces: np.ndarray) -> None:
        f = _c(faces, np.int32).reshape(-1, 5)
        self._check(self._lib.vgi_set_faces(self._h, _ptr(f), f.shape[0]))
        self.n_slots = f.shape[0]

    def autotune(self, samples: int) -> dict:
        """Picks the fastest layout / refill threshold for the current faces."""
        layout, refill, ms = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_float()
        self._check(self._lib.vgi_autotune(self._h, samples, ctypes.byref(layout), ctypes.byref(refill), ctypes.byref(ms)))
        return {"layout": int(layout.value), "refill_min": int(refill.value), "trace_ms": float(ms.value)}

    def set_graph(self, enable: bool) -> None:
        """Replay frames from a captured CUDA graph (see include/vgi.h)."""
        self._check(self._lib.vgi_set_graph(self._h, int(enable)))

    def frame(self, samples: int, clock_ms: int = 0) -> None:
        self._check(self._lib.vgi_frame(self._h, samples, clock_ms))

    WAVEFRONT = 0
    SINGLE_KERNEL = 1

    def set_layout(self, layout: int, refill_min: int = 8) -> None:
        """Trace layout: GpuTracer.WAVEFRONT (default) or GpuTracer.SINGLE_KERNEL."""
        self._check(self._lib.vgi_set_layout(self._h, layout, refill_min))

    def set_timing(self, enable: bool) -> None:
        self._check(self._lib.vgi_set_timing(self._h, int(enable)))

    def frame_times(self) -> np.ndarray:
        """Device ms of the last frame's prepare, trace and accumulate, and the
        summed traversal launches of the wavefront layout."""
        out = np.zeros(4, np.float32)
        self._check(self._lib.vgi_frame_times(self._h, _ptr(out)))
        return out

    def trace_batch(self, tasks: np.ndarray, samples: int, clock_ms: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        t = _c(tasks, np.uint32).reshape(-1, 8)
        if out is None:
            out = np.zeros((t.shape[0], 24), np.uint32)
        self._check(self._lib.vgi_trace_batch(self._h, _ptr(t), t.shape[0], samples, clock_ms, _ptr(out)))
        return out

    def census(self, samples: int) -> dict:
        c = Counters()
        self._check(self._lib.vgi_census(self._h, samples, ctypes.byref(c)))
        return c.as_dict()

    def trace_tasks(self, tasks: np.ndarray, samples: int, count: bool = False):
        t = _c(tasks, np.uint32).reshape(-1, 8)
        out = np.zeros((t.shape[0], 24), np.uint32)
        c = Counters()
        self._check(self._lib.vgi_trace_tasks(self._h, _ptr(t), t.shape[0], samples, _ptr(out), ctypes.byref(c) if count else None))
        return (out, c.as_dict()) if count else out

    def apply_events(self, words: np.ndarray, n_events: int) -> None:
        w = _c(words, np.uint32).reshape(-1)
        self._check(self._lib.vgi_apply_events(self._h, _ptr(w), n_events, w.size))

    def apply_events_measured(self, words: np.ndarray, n_events: int, measures: np.ndarray, read: bool = True):
        """Retention events whose measured edits take their flux from the
        cache first; returns the event words as apply_events read them
        (None with read=False)."""
        w = _c(words, np.uint32).reshape(-1)
        m = _c(measures, np.uint32).reshape(-1, 12)
        self._check(self._lib.vgi_apply_events_measured(self._h, _ptr(w), n_events, w.size, _ptr(m), m.shape[0]))
        if not read:
            return None
        out = np.zeros_like(w)
        if self.n_slots:
            self._check(self._lib.vgi_read_events(self._h, _ptr(out), out.size))
        return out

    # ---- view tier -----------------------------------------------------------
    def apply_events_footprints(self, words: np.ndarray, n_events: int, footprints: np.ndarray, measures=None) -> np.ndarray:
        """Retention events whose reserved Light events take the changed boxes'
        shadow footprints first; returns the event words as retention read them."""
        w = _c(words, np.uint32).reshape(-1)
        fp = _c(footprints, np.int32).reshape(-1, 4)
        m = _c(measures if measures is not None else np.zeros((0, 12), np.uint32), np.uint32).reshape(-1, 12)
        n_fp = (fp.shape[0] - 1) // 3
        self._check(self._lib.vgi_apply_events_footprints(self._h, _ptr(w), n_events, w.size, _ptr(m) if m.size else None, m.shape[0],
                                                          _ptr(fp), n_fp))
        out = np.zeros_like(w)
        self._check(self._lib.vgi_read_events(self._h, _ptr(out), out.size))
        return out

    def view_set_receivers(self, faces: np.ndarray) -> None:
        """Visible unit faces (voxel xyz, face, material rows) as view receivers."""
        f = _c(faces, np.int32).reshape(-1, 5)
        self._check(self._lib.vgi_view_set_receivers(self._h, _ptr(f), f.shape[0]))
        self.n_view = f.shape[0]

    def view_frame(self, first: int = 0, invocations: int = 0, max_hits: int = 8, depth: int = 0, ticket=(0, 0, 0, 0),
                   view_first: bool = False, shared: bool = True, clock_ms: int = 0, events=None, n_events: int = 0) -> None:
        w = ViewWave(first, invocations, max_hits, depth, (ctypes.c_uint32 * 4)(*ticket), int(view_first), int(shared), clock_ms)
        ev = np.zeros(0, np.uint32) if events is None else _c(events, np.uint32).reshape(-1)
        self._check(self._lib.vgi_view_frame(self._h, ctypes.byref(w), _ptr(ev), n_events, ev.size))

    def view_read(self) -> dict:
        n = getattr(self, "n_view", 0)
        out = {"receivers": np.zeros((n, 8), np.uint32), "paths": np.zeros((n, 32), np.uint32),
               "continuations": np.zeros((n, 32), np.uint32), "estimates": np.zeros((n, 16), np.uint32),
               "queue": np.zeros(12 + 2 * n, np.uint32)}
        self._check(self._lib.vgi_view_read(self._h, _ptr(out["receivers"]), _ptr(out["paths"]), _ptr(out["continuations"]),
                                            _ptr(out["estimates"]), _ptr(out["queue"])))
        return out

    def view_trace_paths(self, samples: int) -> np.ndarray:
        n = getattr(self, "n_view", 0)
        out = np.zeros((n * samples, 32), np.uint32)
        self._check(self._lib.vgi_view_trace_paths(self._h, samples, _ptr(out)))
        return out

    MLP_WEIGHTS = 19456
    MLP_LAYERS = [(96, 64), (64, 64), (64, 64), (64, 64), (64, 16)]

    def mlp_set_weights(self, master: np.ndarray) -> None:
        w = _c(master, np.float32).reshape(-1)
        self._check(self._lib.vgi_mlp_set_weights(self._h, _ptr(w), w.size))

    def mlp_get_weights(self) -> np.ndarray:
        w = np.zeros(self.MLP_WEIGHTS, np.float32)
        self._check(self._lib.vgi_mlp_get_weights(self._h, _ptr(w), w.size))
        return w

    def mlp_forward(self, features: np.ndarray) -> np.ndarray:
        f = _c(features, np.float32).reshape(-1, 96)
        out = np.zeros((f.shape[0], 4), np.float32)
        self._check(self._lib.vgi_mlp_forward(self._h, _ptr(f), f.shape[0], _ptr(out)))
        return out[:, :3]

    @staticmethod
    def _mlp_batch(features, targets):
        f = _c(features, np.float32).reshape(-1, 96)
        y = np.zeros((f.shape[0], 4), np.float32)
        y[:, :3] = np.asarray(targets, np.float32).reshape(-1, 3)
        return f, y

    def mlp_gradients(self, features: np.ndarray, targets: np.ndarray):
        """(dLoss/dW in master order, loss) of the relative-luminance loss."""
        f, y = self._mlp_batch(features, targets)
        g = np.zeros(self.MLP_WEIGHTS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self._lib.vgi_mlp_gradients(self._h, _ptr(f), _ptr(y), f.shape[0], _ptr(g), _ptr(loss)))
        return g, float(loss[0])

    def mlp_train(self, features: np.ndarray, targets: np.ndarray, lr: float = 1e-2) -> float:
        """One Adam step; returns the loss before it."""
        f, y = self._mlp_batch(features, targets)
        loss = np.zeros(1, np.float32)
        self._check(self._lib.vgi_mlp_train(self._h, _ptr(f), _ptr(y), f.shape[0], float(lr), _ptr(loss)))
        return float(loss[0])

    def mlp_apply_gradients(self, grads, loss: float = 0.0, lr: float = 1e-2) -> None:
        """One Adam step from a given gradient (a host array, or a CUDA tensor
        on this context's device)."""
        if hasattr(grads, "data_ptr"):
            assert grads.numel() == self.MLP_WEIGHTS and grads.is_contiguous()
            self._check(self._lib.vgi_mlp_apply_gradients(self._h, ctypes.c_void_p(grads.data_ptr()), float(loss), float(lr), 1))
        else:
            g = _c(grads, np.float32).reshape(-1)
            assert g.size == self.MLP_WEIGHTS
            self._check(self._lib.vgi_mlp_apply_gradients(self._h, _ptr(g), float(loss), float(lr), 0))

    def mlp_encode(self, faces: np.ndarray) -> np.ndarray:
        """The network's inputs (n x 96) for face rows (voxel xyz, face, material)."""
        f = _c(faces, np.int32).reshape(-1, 5)
        out = np.zeros((f.shape[0], 96), np.float32)
        self._check(self._lib.vgi_mlp_encode(self._h, _ptr(f), f.shape[0], _ptr(out)))
        return out

    def submit_batch(self, tasks: np.ndarray, samples: int, clock_ms: int, out: np.ndarray) -> int:
        """vgi_submit_batch: returns a ticket; `tasks` and `out` (ideally
        pinned) must stay alive and unchanged until complete_batch(ticket)."""
        assert tasks.dtype == np.uint32 and tasks.flags.c_contiguous and out.dtype == np.uint32 and out.flags.c_contiguous
        ticket = ctypes.c_uint64()
        self._check(self._lib.vgi_submit_batch(self._h, _ptr(tasks), tasks.shape[0], samples, clock_ms, _ptr(out), ctypes.byref(ticket)))
        return ticket.value

    def complete_batch(self, ticket: int) -> None:
        self._check(self._lib.vgi_complete_batch(self._h, ticket))

    # headless discovery
    def discover_faces(self, eye, forward, up, tan_half_fov: float, width: int, height: int, capacity: Optional[int] = None,
                       pixels: bool = True):
        """Primary rays per pixel: (pixels (h, w, 8) u32 records or None,
        faces (n, 5) rows voxel xyz, face, material). The default capacity,
        one face per pixel, always suffices."""
        capacity = width * height if capacity is None else capacity
        f = np.asarray(forward, np.float64)
        f = (f / np.linalg.norm(f)).astype(np.float32)
        cam = Camera((ctypes.c_float * 3)(*map(float, eye)), (ctypes.c_float * 3)(*map(float, f)),
                     (ctypes.c_float * 3)(*map(float, up)), float(tan_half_fov), width, height)
        records = np.empty((height, width, 8), np.uint32) if pixels else None
        faces = np.empty((capacity, 5), np.int32)  # the library writes the first n rows
        n = ctypes.c_uint32()
        self._check(self._lib.vgi_discover_faces(self._h, ctypes.byref(cam), _ptr(records) if pixels else None, _ptr(faces), capacity,
                                                 ctypes.byref(n)))
        return records, faces[: n.value].copy()

    # reconstruction and presentation of the view receivers
    def view_set_tiles(self, tiles: np.ndarray, tiles_x: int, tiles_y: int) -> None:
        t = _c(tiles, np.uint32).reshape(-1)
        self._check(self._lib.vgi_view_set_tiles(self._h, _ptr(t), t.size, tiles_x, tiles_y))

    def view_reconstruct(self, evidence_goal: float = 0.031, spatial: float = 1.0, temporal: float = 1.0) -> None:
        d = ViewDisplay(evidence_goal, spatial, temporal)
        self._check(self._lib.vgi_view_reconstruct(self._h, ctypes.byref(d)))

    def view_read_published(self):
        """(FarPixel words (n, 12), counters (5,))."""
        n = getattr(self, "n_view", 0)
        pixels = np.zeros((n, 12), np.uint32)
        stats = np.zeros(5, np.uint32)
        self._check(self._lib.vgi_view_read_published(self._h, _ptr(pixels), _ptr(stats)))
        return pixels, stats

    def view_present(self, eye, forward, up, tan_half_fov: float, width: int, height: int, corners: bool = True) -> np.ndarray:
        """corner_irradiance at each pixel's first hit: (height, width, 4) f32."""
        cam = Camera((ctypes.c_float * 3)(*map(float, eye)), (ctypes.c_float * 3)(*map(float, forward)),
                     (ctypes.c_float * 3)(*map(float, up)), float(tan_half_fov), width, height)
        out = np.zeros((height, width, 4), np.float32)
        self._check(self._lib.vgi_view_present(self._h, ctypes.byref(cam), 1 if corners else 0, _ptr(out)))
        return out

    # far tier
    def far_frame(self, eye, forward, up, tan_half_fov: float, width: int, height: int, settings: Optional["FarTierSettings"] = None,
                  frame: int = 0) -> None:
        """One far-tier frame (classify, then trace the queue) for a camera;
        `forward` must be unit length."""
        cam = Camera((ctypes.c_float * 3)(*map(float, eye)), (ctypes.c_float * 3)(*map(float, forward)),
                     (ctypes.c_float * 3)(*map(float, up)), float(tan_half_fov), width, height)
        st = (settings or FarTierSettings()).struct()
        self._check(self._lib.vgi_far_frame(self._h, ctypes.byref(cam), ctypes.byref(st), frame & 0xFFFFFFFF))

    def mlp_set_wait_limit(self, polls: Optional[int] = None) -> None:
        """Polls per tensor-core wait of the MLP kernels (None: the default;
        0: every wait gives up at once, to exercise the run-out path)."""
        self._check(self._lib.vgi_mlp_set_wait_limit(self._h, MLP_WAIT_DEFAULT if polls is None else int(polls)))

    def inject_failure(self, what: int, count: int = 1) -> None:
        """vgi_inject_failure for this thread: INJECT_ALLOC or INJECT_UPLOAD."""
        inject_failure(what, count)

    def view_read_sun_flips(self):
        """The sun-flip reports since the last read, which this read clears:
        (records (up to 2048, 4): voxel xyz, flux bits; overflow (7,); count
        of all flips, records and overflow together)."""
        words = np.zeros(4 + 2048 * 4 + 7, np.uint32)
        self._check(self._lib.vgi_view_read_sun_flips(self._h, _ptr(words)))
        count = int(words[0])
        return words[4:4 + 4 * min(count, 2048)].reshape(-1, 4), words[4 + 2048 * 4:], count

    def set_topology_prior(self, enable: bool) -> None:
        self._check(self._lib.vgi_set_topology_prior(self._h, 1 if enable else 0))

    def set_far_handoff(self, enable: bool) -> None:
        self._check(self._lib.vgi_set_far_handoff(self._h, 1 if enable else 0))

    def far_reset(self) -> None:
        self._check(self._lib.vgi_far_reset(self._h))

    def far_read(self):
        """(shape (4,), output (16 + 4 cells,), cells (n, 12), stats (8,)) u32 words."""
        shape = np.zeros(4, np.uint32)
        self._check(self._lib.vgi_far_read(self._h, _ptr(shape), None, None, None))
        n = int(shape[0]) * int(shape[1])
        output = np.zeros(16 + 4 * n, np.uint32)
        cells = np.zeros((n, 12), np.uint32)
        stats = np.zeros(8, np.uint32)
        self._check(self._lib.vgi_far_read(self._h, None, _ptr(output), _ptr(cells), _ptr(stats)))
        return shape, output, cells, stats

    # scheduled frames
    def frame_scheduled(self, samples: int, clock_ms: int, budget: int, focus=(0, 0, 0), classify=None, audit_ms: int = 1000) -> None:
        """A frame that traces `budget` faces the GPU selection picks."""
        first, end = classify if classify is not None else (0, self.n_slots)
        sched = Schedule((ctypes.c_int32 * 3)(*[int(v) for v in focus]), budget, first, end, audit_ms)
        self._check(self._lib.vgi_frame_scheduled(self._h, samples, clock_ms, ctypes.byref(sched)))
        self._budget = budget

    def read_selection(self) -> dict:
        n, b = self.n_slots, getattr(self, "_budget", 0)
        keys = np.zeros(n, np.uint32)
        sel = np.zeros(1038, np.uint32)
        picks = np.zeros((b, 4), np.uint32)
        tasks = np.zeros((b, 8), np.uint32)
        results = np.zeros((b, 24), np.uint32)
        self._check(self._lib.vgi_read_selection(self._h, _ptr(keys), _ptr(sel), _ptr(picks), _ptr(tasks), _ptr(results)))
        return {"keys": keys, "selection": sel, "picks": picks, "tasks": tasks, "results": results}

    # face-sharded frames
    def frame_shard(self, samples: int, clock_ms: int, first: int, n: int) -> None:
        """prepare, trace and accumulate of slots [first, first + n) only."""
        self._check(self._lib.vgi_frame_shard(self._h, samples, clock_ms, first, n))

    def read_cache(self, first: int, n: int) -> np.ndarray:
        """Gather records of slots [first, first + n): (n, 4) u32 words."""
        out = np.zeros((n, 4), np.uint32)
        self._check(self._lib.vgi_read_cache(self._h, first, n, _ptr(out), 0))
        return out

    def write_cache(self, first: int, n: int, records: np.ndarray) -> None:
        r = _c(records, np.uint32).reshape(n, 4)
        self._check(self._lib.vgi_write_cache(self._h, first, n, _ptr(r), 0))

    def read_cache_device(self, first: int, n: int, device_ptr: int) -> None:
        """Enqueues a copy of the records into device memory (context stream)."""
        self._check(self._lib.vgi_read_cache(self._h, first, n, ctypes.c_void_p(device_ptr), 1))

    def write_cache_device(self, first: int, n: int, device_ptr: int) -> None:
        self._check(self._lib.vgi_write_cache(self._h, first, n, ctypes.c_void_p(device_ptr), 1))

    def set_mlp_cache(self, enable: bool = True, warm_frames: int = 8, samples: int = 65536, steps_per_frame: int = 16,
                      lr: float = 1e-2) -> None:
        """MLP cache mode of frame(): online training on `samples` faces a
        frame over `steps_per_frame` Adam steps, and after warm_frames
        frames the network ends uncached first hits."""
        self._check(self._lib.vgi_set_mlp_cache(self._h, 1 if enable else 0, warm_frames, samples, steps_per_frame, float(lr)))

    def set_mlp_schedule(self, rows_per_step: int = 0, history_share: float = 0.0) -> None:
        """MLP cache mode: rows of one Adam step (0: the frame's samples over
        its steps) and the averaging window, a share of the samples taken
        since the network began ending paths (0: the transport's limit)."""
        self._check(self._lib.vgi_set_mlp_schedule(self._h, int(rows_per_step), float(history_share)))

    def mlp_stats(self) -> dict:
        st = MlpStatus()
        self._check(self._lib.vgi_mlp_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in MlpStatus._fields_}

    def reference_fp64(self, tasks: np.ndarray, samples: int, seed: int = 1):
        """FP64 converged reference per FaceTask: (mean rgb, mean square rgb, known)."""
        t = _c(tasks, np.uint32).reshape(-1, 8)
        n = t.shape[0]
        mean = np.zeros((n, 3), np.float64)
        second = np.zeros((n, 3), np.float64)
        known = np.zeros(n, np.uint32)
        self._check(self._lib.vgi_reference_fp64(self._h, _ptr(t), n, samples, seed, _ptr(mean), _ptr(second), _ptr(known)))
        return mean, second, known

    def read_results(self, first: int = 0, n: Optional[int] = None) -> np.ndarray:
        n = self.n_slots - first if n is None else n
        out = np.zeros((n, 24), np.uint32)
        self._check(self._lib.vgi_read_results(self._h, first, n, _ptr(out)))
        return out

    def read_state(self, first: int = 0, n: Optional[int] = None) -> np.ndarray:
        n = self.n_slots - first if n is None else n
        out = np.zeros((n, 36), np.uint32)
        self._check(self._lib.vgi_read_state(self._h, first, n, _ptr(out)))
        return out

    def write_state(self, words: np.ndarray, first: int = 0) -> None:
        w = _c(words, np.uint32).reshape(-1, 36)
        self._check(self._lib.vgi_write_state(self._h, first, w.shape[0], _ptr(w)))

    def read_slot_meta(self, first: int = 0, n: Optional[int] = None) -> np.ndarray:
        n = self.n_slots - first if n is None else n
        out = np.zeros((n, 12), np.uint32)
        self._check(self._lib.vgi_read_slot_meta(self._h, first, n, _ptr(out)))
        return out


# ---- synthetic workloads and host-runtime helpers ----------------------------

def inject_failure(what: int, count: int = 1) -> None:
    """Makes the calling thread's next `count` device allocations
    (INJECT_ALLOC) or host-to-device copies (INJECT_UPLOAD) in libvgi fail
    without reaching the device (vgi_inject_failure); 0 cancels."""
    rc = library().vgi_inject_failure(None, what, count)
    if rc != OK:
        raise VgiError(rc, "vgi_inject_failure refused its arguments")


def grid_coords(nx: int, ny: int, nz: int) -> np.ndarray:
    out = np.zeros((nx * ny * nz, 3), np.int32)
    library().vgi_scene_grid_coords(nx, ny, nz, _ptr(out))
    return out


def stone_room():
    vox = np.zeros(8 * 4096, np.uint16)
    library().vgi_scene_stone_room(_ptr(vox))
    return grid_coords(2, 2, 2), vox


def furnace():
    vox = np.zeros(8 * 4096, np.uint16)
    library().vgi_scene_furnace(_ptr(vox))
    return grid_coords(2, 2, 2), vox


def terrain(nx: int, ny: int, nz: int, seed: int = 2, octaves: int = 4, period: float = 64.0, base_height: float = 96.0,
            falloff: float = 48.0, emitters: int = 256):
    p = TerrainParams(seed, octaves, period, base_height, falloff, emitters)
    vox = np.zeros(nx * ny * nz * 4096, np.uint16)
    library().vgi_scene_terrain(ctypes.byref(p), nx, ny, nz, _ptr(vox))
    return grid_coords(nx, ny, nz), vox


class CaveParams(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint32), ("worms", ctypes.c_uint32), ("steps", ctypes.c_uint32), ("radius_min", ctypes.c_float),
                ("radius_max", ctypes.c_float), ("roof", ctypes.c_uint32), ("skylights", ctypes.c_uint32),
                ("skylight_radius", ctypes.c_float), ("emitters", ctypes.c_uint32)]


def cave(nx: int, ny: int, nz: int, seed: int = 1, worms: int = 40, steps: int = 600, radius_min: float = 3.0, radius_max: float = 12.0,
         roof: int = 16, skylights: int = 16, skylight_radius: float = 6.0, emitters: int = 2000):
    """The worm-tunnel cave (vgi_scene_cave): (coords, voxels)."""
    p = CaveParams(seed, worms, steps, radius_min, radius_max, roof, skylights, skylight_radius, emitters)
    vox = np.zeros(nx * ny * nz * 4096, np.uint16)
    library().vgi_scene_cave(ctypes.byref(p), nx, ny, nz, _ptr(vox))
    return grid_coords(nx, ny, nz), vox


def exposed_faces(coords, voxels, frustum=None, box=None, facing=None) -> np.ndarray:
    """Exposed faces as (voxel xyz, face, material) rows. ``frustum`` =
    (eye, forward, tan_half); ``box`` = (min xyz, max xyz) on the air cell;
    ``facing`` = an eye position: faces turned towards it (a cube-map camera)."""
    coords = _c(coords, np.int32).reshape(-1, 3)
    voxels = _c(voxels, np.uint16).reshape(-1)
    flt = FaceFilter()
    if facing is not None:
        flt.use_facing = 1
        flt.eye[:] = list(map(float, facing))
    if frustum is not None:
        eye, fwd, tan_half = frustum
        fwd = np.asarray(fwd, np.float64)
        fwd = fwd / np.linalg.norm(fwd)
        flt.use_frustum = 1
        flt.eye[:] = list(map(float, eye))
        flt.forward[:] = list(map(float, fwd))
        flt.tan_half = tan_half
    if box is not None:
        flt.use_box = 1
        flt.box_min[:] = list(map(int, box[0]))
        flt.box_max[:] = list(map(int, box[1]))
    lib = library()
    n = lib.vgi_scene_faces(_ptr(coords), coords.shape[0], _ptr(voxels), ctypes.byref(flt), None, 0)
    out = np.zeros((max(n, 1), 5), np.int32)
    lib.vgi_scene_faces(_ptr(coords), coords.shape[0], _ptr(voxels), ctypes.byref(flt), _ptr(out), n)
    return out[:n]


def host_emitters(coords, voxels, material_words):
    coords = _c(coords, np.int32).reshape(-1, 3)
    voxels = _c(voxels, np.uint16).reshape(-1)
    m = _c(material_words, np.float32).reshape(-1)
    info = np.zeros(2, np.uint32)
    lib = library()
    n = lib.vgi_host_emitters(_ptr(coords), coords.shape[0], _ptr(voxels), _ptr(m), None, 0, _ptr(info))
    out = np.zeros(n, np.uint32)
    lib.vgi_host_emitters(_ptr(coords), coords.shape[0], _ptr(voxels), _ptr(m), _ptr(out), n, _ptr(info))
    return out, int(info[0]), float(info[1:2].view(np.float32)[0])


def host_face_index(faces) -> np.ndarray:
    f = _c(faces, np.int32).reshape(-1, 4)
    lib = library()
    n = lib.vgi_host_face_index(_ptr(f), f.shape[0], None, 0)
    out = np.zeros((n, 4), np.uint32)
    lib.vgi_host_face_index(_ptr(f), f.shape[0], _ptr(out), n)
    return out


def host_top_level(coords, solid) -> Optional[np.ndarray]:
    coords = _c(coords, np.int32).reshape(-1, 3)
    s = _c(solid, np.uint8)
    lo, hi = coords.min(0), coords.max(0)
    cells = int(np.prod(hi - lo + 1))
    out = np.zeros(cells * 6, np.uint8)
    rc = library().vgi_host_top_level(_ptr(coords), _ptr(s), coords.shape[0], _ptr(out), out.size)
    return None if rc == 1 else out.reshape(-1, 6)


class GpuBatch:
    """Several GpuTracer scenes traced together (vgi_batch_*): one frame of
    every scene, with each stage's traversal one launch over all their rays.
    The tracers must outlive the batch."""

    def __init__(self, tracers):
        self._lib = library()
        self.tracers = list(tracers)
        handles = (ctypes.c_void_p * len(self.tracers))(*[t._h.value for t in self.tracers])
        h = ctypes.c_void_p()
        rc = self._lib.vgi_batch_create(handles, len(self.tracers), ctypes.byref(h))
        if rc != OK:
            raise VgiError(rc, "vgi_batch_create failed")
        self._h = h

    def _check(self, rc: int) -> None:
        if rc != OK:
            raise VgiError(rc, self._lib.vgi_batch_last_error(self._h).decode())

    def frame(self, samples: int, clock_ms: int = 0) -> None:
        self._check(self._lib.vgi_batch_frame(self._h, samples, clock_ms))

    def set_graph(self, enable: bool) -> None:
        self._check(self._lib.vgi_batch_set_graph(self._h, 1 if enable else 0))

    def sync(self) -> None:
        self._check(self._lib.vgi_batch_sync(self._h))

    def autotune(self, samples: int) -> dict:
        refill, blocks, ms = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_float()
        self._check(self._lib.vgi_batch_autotune(self._h, samples, ctypes.byref(refill), ctypes.byref(blocks), ctypes.byref(ms)))
        return {"refill_min": refill.value, "blocks": blocks.value, "trace_ms": ms.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.vgi_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tasks_for(faces: np.ndarray, sequence: int = 0) -> np.ndarray:
    """FaceTask words (voxel xyz, face, sequence, 0, 0, 0) for face rows."""
    f = np.asarray(faces, np.int32).reshape(-1, 5)
    t = np.zeros((f.shape[0], 8), np.uint32)
    t[:, 0:3] = f[:, 0:3].astype(np.int64).astype(np.uint32)
    t[:, 3] = f[:, 3]
    t[:, 4] = sequence
    return t
