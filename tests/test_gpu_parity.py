"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Bar: geometry, hit records, face results, resident state and slot metadata
are bit-exact (integer and float words compared as u32). Workloads are the
reference's fixtures (stone room, furnace) and seeded terrain at sizes the
oracle finishes in seconds.
"""
import numpy as np
import pytest

import oracle_lib as O
import vgi

pytestmark = pytest.mark.gpu


class Case:
    def __init__(self, coords, vox, materials, lights=(), n_directional=0, env=(0.0, 0.0, 0.0), transport=None, faces=None):
        self.coords = np.asarray(coords, np.int32)
        self.vox = np.asarray(vox, np.uint16)
        self.materials = materials.words() if hasattr(materials, "words") else np.asarray(materials, np.float32)
        self.lights = np.concatenate([l.words() for l in lights]) if len(lights) else np.zeros(0, np.float32)
        self.n_directional = n_directional
        self.env = env
        self.transport = transport or vgi.TransportSettings()
        self.faces = vgi.exposed_faces(self.coords, self.vox) if faces is None else faces
        self.emitters, self.n_emit, self.total = vgi.host_emitters(self.coords, self.vox, self.materials)
        self.strides = None  # per-region stride log2 (coarse pages), or None

    def load(self, g: vgi.GpuTracer, with_faces=True, layout=vgi.GpuTracer.WAVEFRONT):
        g.set_layout(layout)
        g.upload_regions(self.coords, self.vox, self.strides)
        g.set_materials(self.materials)
        g.set_lights(self.lights, self.n_directional)
        g.set_environment(self.env)
        g.build_emitters()
        g.set_transport(self.transport)
        # Without faces the context's cache is emptied, so a trace never
        # gathers from an earlier test's faces (the context is shared).
        g.set_faces(self.faces if with_faces else np.zeros((0, 5), np.int32))

    def pipe(self, lanes):
        t = self.transport
        return O.Pipeline(t.bounces, 1 if min(max(t.reach, 1.0), 768.0) < 768.0 else 0, t.path_steps, int(t.budgeted), lanes)

    def params_fn(self, geometry):
        d, h, cl, bounds = geometry
        n_lights = self.lights.size // 12

        def fn(n, samples):
            return O.params_words(n, samples, d.size // 4, n_lights, bounds, self.n_directional, self.env, self.total, self.n_emit,
                                  self.transport.reach)

        return fn


def lanes_for(t: vgi.TransportSettings, samples):
    if t.lanes:
        return t.lanes
    lanes = 1
    while lanes < samples and lanes < 32:
        lanes <<= 1
    if lanes > samples and lanes > 1:
        lanes >>= 1
    return lanes


def stone_room_case(**kw):
    coords, vox = vgi.stone_room()
    m = vgi.VoxelGiMaterials()
    m.set(0, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5)))
    m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(8.0, 4.0, 1.5)))
    t = vgi.TransportSettings(bounces=1, path_steps=64, history_limit=64, **kw)
    return Case(coords, vox, m, transport=t)


def furnace_case(**kw):
    coords, vox = vgi.furnace()
    m = vgi.VoxelGiMaterials()
    m.set(4, vgi.MaterialTransport(diffuse=(0.3, 0.55, 0.7), emission=(0.7, 1.3, 0.2)))
    faces = vgi.exposed_faces(coords, vox, box=((9, 9, 9), (22, 22, 22)))
    return Case(coords, vox, m, faces=faces, transport=vgi.TransportSettings(**kw))


def terrain_case(seed=5, n=(6, 4, 6), emitters=48, **kw):
    coords, vox = vgi.terrain(*n, seed=seed, base_height=30.0, falloff=18.0, emitters=emitters)
    m = vgi.VoxelGiMaterials()
    rng = np.random.default_rng(seed)
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(248):
        r = float(rng.uniform(1, 10))
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(r, r, r)))
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0))
    faces = vgi.exposed_faces(coords, vox)
    return Case(coords, vox, m, lights=[sun], n_directional=1, env=kw.pop("env", (0.0, 0.0, 0.0)),
                transport=vgi.TransportSettings(**kw), faces=faces[::3].copy())


def assert_words_equal(got, want, what):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    bad = np.argwhere(got != want)
    if bad.size:
        r = bad[0][0]
        raise AssertionError(f"{what}: {len(bad)} words differ; first at {tuple(bad[0])}: got {got[r]} want {want[r]}")


@pytest.mark.parametrize("make", [stone_room_case, furnace_case, terrain_case])
def test_gpu_packing_matches_oracle(gpu, make):
    case = make()
    case.load(gpu, with_faces=False)
    d, h, cl, bounds = gpu.geometry()
    ref = O.Scene(case.coords, case.vox, top_mode=0)
    rd, rh, rcl, rbounds = ref.arrays()
    assert (bounds == rbounds).all()
    assert_words_equal(O.canonical(d, h, cl, case.coords), O.canonical(rd, rh, rcl, case.coords), "canonical geometry")


LAYOUTS = [vgi.GpuTracer.WAVEFRONT, vgi.GpuTracer.SINGLE_KERNEL]


def trace_pair(gpu, case, samples, lanes, sequence=0, layout=vgi.GpuTracer.WAVEFRONT):
    case.load(gpu, with_faces=False, layout=layout)
    geometry = gpu.geometry()
    tasks = vgi.tasks_for(case.faces, sequence)
    got, gcnt = gpu.trace_tasks(tasks, samples, count=True)
    params = case.params_fn(geometry)(tasks.shape[0], samples)
    want, wcnt = O.trace_faces(geometry, params, case.materials, case.lights, case.emitters, tasks, case.pipe(lanes))
    gcnt = {k: v for k, v in gcnt.items() if k not in ("warp_passes", "lane_passes")}
    return got, want, gcnt, wcnt


@pytest.mark.parametrize("make,samples,kw", [
    (stone_room_case, 4, {}),
    (furnace_case, 16, {"bounces": 3, "lanes": 8}),
    (furnace_case, 4, {"bounces": 3, "lanes": 1}),
    (terrain_case, 8, {"bounces": 2}),
    (terrain_case, 8, {"bounces": 3, "reach": 24.0}),
    (terrain_case, 4, {"bounces": 2, "budgeted": True, "path_steps": 48, "env": (0.16, 0.24, 0.38)}),
])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_trace_matches_oracle_bit_exact(gpu, make, samples, kw, layout):
    case = make(**kw)
    lanes = lanes_for(case.transport, samples)
    got, want, gcnt, wcnt = trace_pair(gpu, case, samples, lanes, sequence=12345, layout=layout)
    assert_words_equal(got, want, "face results")
    assert gcnt == wcnt
    assert wcnt["rays"] > 0 and wcnt["paths"] == case.faces.shape[0] * samples


def run_frames(gpu, case, frames, samples, layout=vgi.GpuTracer.WAVEFRONT):
    case.load(gpu, layout=layout)
    geometry = gpu.geometry()
    lanes = lanes_for(case.transport, samples)
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                   case.pipe(lanes))
    for f in range(frames):
        gpu.frame(samples, clock_ms=16 * f)
        ref.frame(samples, clock_ms=16 * f)
    return ref


@pytest.mark.parametrize("layout", LAYOUTS)
def test_stone_room_frames_match_oracle(gpu, layout):
    # Config 1 in full: 64 frames of 4 spp, 1 bounce via the cache, 64 DDA
    # steps, history 64 (alpha 1/16 once 64 samples are in).
    case = stone_room_case()
    ref = run_frames(gpu, case, 64, 4, layout)
    assert_words_equal(gpu.read_results(), ref.results, "frame results")
    assert_words_equal(gpu.read_state(), ref.state, "resident state")
    assert_words_equal(gpu.read_slot_meta(), ref.meta, "slot metadata")


def test_autotuned_layout_keeps_results_and_state(gpu):
    # The autotuner's trial traces change no slot; frames after it still
    # match the oracle in whatever layout it chose.
    case = terrain_case(bounces=2)
    ref = run_frames(gpu, case, 3, 8)
    state = gpu.read_state()
    choice = gpu.autotune(8)
    assert choice["layout"] in (0, 1) and 1 <= choice["refill_min"] <= 32 and choice["trace_ms"] > 0
    assert_words_equal(gpu.read_state(), state, "state after autotune")
    for f in range(3, 5):
        gpu.frame(8, clock_ms=16 * f)
        ref.frame(8, clock_ms=16 * f)
    assert_words_equal(gpu.read_results(), ref.results, "frames after autotune")
    gpu.set_layout(vgi.GpuTracer.WAVEFRONT)


def test_graph_replayed_frames_match_oracle(gpu):
    # Frames replayed from a captured graph, across a transport change that
    # drops and recaptures it.
    case = terrain_case(bounces=2)
    gpu.set_graph(True)
    try:
        ref = run_frames(gpu, case, 4, 8)
        case.transport.history_limit = 32
        gpu.set_transport(case.transport)
        ref.transport = case.transport
        for f in range(4, 8):
            gpu.frame(8, clock_ms=16 * f)
            ref.frame(8, clock_ms=16 * f)
        assert_words_equal(gpu.read_results(), ref.results, "graph frame results")
        assert_words_equal(gpu.read_state(), ref.state, "graph frame state")
    finally:
        gpu.set_graph(False)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_terrain_frames_with_cache_match_oracle(gpu, layout):
    case = terrain_case(bounces=2)
    ref = run_frames(gpu, case, 6, 8, layout)
    assert_words_equal(gpu.read_results(), ref.results, "frame results")
    assert_words_equal(gpu.read_state(), ref.state, "resident state")
    # The cache served paths once faces reached 16 samples.
    cnt = gpu.census(8)
    assert cnt["cache_hits"] > 0


@pytest.mark.parametrize("layout", LAYOUTS)
def test_census_counts_match_oracle(gpu, layout):
    case = terrain_case(bounces=2)
    ref = run_frames(gpu, case, 3, 8, layout)
    # Lane use is a property of the GPU layout; the oracle has no warps.
    got = {k: v for k, v in gpu.census(8).items() if k not in ("warp_passes", "lane_passes")}
    geometry = gpu.geometry()
    ctl = O.controls_words(ref.n, 8, 0, case.transport)
    tasks = ref.tasks.copy()
    O.lib().orc_begin_trace(O.ptr(ref.state), None, O.ptr(tasks), O.ptr(ref.slots), ref.n, O.ptr(ctl))
    _, want = O.trace_faces(geometry, case.params_fn(geometry)(ref.n, 8), case.materials, case.lights, case.emitters, tasks,
                            case.pipe(8), ref.state, ref.index)
    assert got == want


def encode_events(events):
    """encode_events (src/gpu/resident.rs:1326-1414) for box events:
    each event = (union lo, union hi, [(lo, hi, flux, kind_word)])."""
    head, bounds = [], []
    first = 0
    for lo, hi, items in events:
        head += [[lo[0], lo[1], lo[2], 0], [hi[0], hi[1], hi[2], 0], [0, 0, first, len(items)]]
        first += len(items)
        for blo, bhi, flux, kind in items:
            bounds += [[blo[0], blo[1], blo[2], int(np.float32(flux).view(np.uint32))], [bhi[0], bhi[1], bhi[2], kind]]
    words = np.array(head + bounds, np.int64).astype(np.uint32)
    return words.reshape(-1), len(events)


def test_events_and_discount_match_oracle(gpu):
    case = terrain_case(bounces=2, measured_retention=1.0)
    ref = run_frames(gpu, case, 4, 8)
    c = case.faces[len(case.faces) // 2, :3]
    events = [
        (c - 2, c + 2, [(c - 2, c + 2, 40.0, 3 | 8), (c + 5, c + 6, 0.0, 0)]),
        (c + 20, c + 22, [(c + 20, c + 22, 500.0, 3)]),
    ]
    words, n = encode_events(events)
    gpu.apply_events(words, n)
    ref.apply_events(words, n)
    assert_words_equal(gpu.read_state(), ref.state, "state after events")
    assert_words_equal(gpu.read_slot_meta(), ref.meta, "slot metadata after events")
    for f in range(2):
        gpu.frame(8, clock_ms=100 + f)
        ref.frame(8, clock_ms=100 + f)
    assert_words_equal(gpu.read_state(), ref.state, "state after discounted frames")
    assert_words_equal(gpu.read_results(), ref.results, "results after discounted frames")


def material_light(words):
    """(albedo, emission) luminance per material, as the host builds it for
    edit measurement (src/gpu/resident.rs:816-838)."""
    m = np.asarray(words, np.float32).reshape(256, 16)
    w = [np.float32(0.2126), np.float32(0.7152), np.float32(0.0722)]
    out = np.zeros((256, 2), np.float32)
    for col, first in ((0, 0), (1, 8)):
        out[:, col] = (w[0] * m[:, first] + w[1] * m[:, first + 1]) + w[2] * m[:, first + 2]
    return out


def test_measured_edits_match_oracle(gpu):
    # measure_edits + finish_edits (voxel_accumulate.wgsl:375-425) ahead of
    # apply_events: two edits next to traced faces take their flux from the
    # cache; one in open air above the terrain sees no face and turns unknown.
    case = terrain_case(bounces=2, measured_retention=1.0)
    ref = run_frames(gpu, case, 4, 8)
    a = case.faces[len(case.faces) // 2, :3]
    b = case.faces[len(case.faces) // 5, :3]
    sky = np.array([a[0], 120, a[2]], np.int32)
    bounds = [(a, a, 2.0, 1), (b - 1, b, 0.5, 8), (sky, sky + 1, 1.0, 8)]
    events = [(np.minimum(a, b - 1) - 1, np.maximum(a, b) + 1, [(lo, hi, flux, 6 | 8) for lo, hi, flux, _ in bounds[:2]]),
              (sky - 1, sky + 2, [(sky, sky + 1, 1.0, 6)])]
    words, n = encode_events(events)
    measures, first = [], 0
    for k, (lo, hi, flux, voxels) in enumerate(bounds):
        size = (hi - lo) + 3
        count = int(np.prod(size))
        measures += [[n * 3 + 2 * k, first, count, voxels], [*(lo - 1), int(np.float32(flux).view(np.uint32))], [*size, 0]]
        first += count
    measures = np.array(measures, np.int64).astype(np.uint32)
    got = gpu.apply_events_measured(words, n, measures)
    want = ref.measure_edits(words, measures, len(bounds), material_light(case.materials))
    assert_words_equal(got.reshape(-1, 4), want.reshape(-1, 4), "event words after measurement")
    kinds = want.reshape(-1, 4)[n * 3 + 1::2, 3] & 7
    assert list(kinds) == [3, 3, 0], kinds
    ref.apply_events(want, n)
    assert_words_equal(gpu.read_state(), ref.state, "state after measured events")
    assert_words_equal(gpu.read_slot_meta(), ref.meta, "slot metadata after measured events")
    for f in range(2):
        gpu.frame(8, clock_ms=100 + f)
        ref.frame(8, clock_ms=100 + f)
    assert_words_equal(gpu.read_results(), ref.results, "results after measured events")


def test_edits_match_oracle(gpu):
    case = terrain_case()
    case.load(gpu, with_faces=False)
    ref = O.Scene(case.coords, case.vox, top_mode=0)
    rng = np.random.default_rng(2)
    for step in range(3):
        centre = rng.integers((8, 8, 8), (88, 56, 88))
        r = int(rng.integers(1, 6))
        edits = []
        for dz in range(-r, r + 1):
            for dy in range(-r, r + 1):
                for dx in range(-r, r + 1):
                    if dx * dx + dy * dy + dz * dz <= r * r:
                        value = 256 if step != 1 else 3
                        edits.append((centre[0] + dx, centre[1] + dy, centre[2] + dz, value))
        edits = np.array(edits, np.int32)
        gpu.edit_voxels(edits)
        ref.edit(edits)
        d, h, cl, bounds = gpu.geometry()
        rd, rh, rcl, _ = ref.arrays()
        assert_words_equal(O.canonical(d, h, cl, case.coords), O.canonical(rd, rh, rcl, case.coords), f"geometry after edit {step}")


@pytest.mark.parametrize("samples", [1, 3, 8, 32])
def test_kept_light_tree_rows_follow_sample_counts_and_tree_changes(gpu, samples):
    """The begin kernel keeps each face's top light-tree probabilities across
    frames (filled by the face's lanes between them; not kept when the
    sample count does not divide 32). Frames with 1, 3, 8 and 32 samples
    match the oracle word for word, and so do frames after the emitters
    change (new emission, so a new tree and stale rows)."""
    case = terrain_case(bounces=1)
    ref = run_frames(gpu, case, 2, samples)
    assert_words_equal(gpu.read_results(), ref.results, f"frame results, {samples} samples")
    # New emission on the emissive materials: new emitter weights and tree.
    words = case.materials.copy().reshape(-1, 16)
    words[8:, 4:7] *= 1.5
    case.materials = words.reshape(-1)
    case.emitters, case.n_emit, case.total = vgi.host_emitters(case.coords, case.vox, case.materials)
    gpu.set_materials(case.materials)
    gpu.build_emitters()
    geometry = gpu.geometry()
    ref.params_fn, ref.emitter_words, ref.materials = case.params_fn(geometry), case.emitters, case.materials
    for f in range(2, 4):
        gpu.frame(samples, clock_ms=16 * f)
        ref.frame(samples, clock_ms=16 * f)
    assert_words_equal(gpu.read_results(), ref.results, f"frame results after the tree changed, {samples} samples")
    assert_words_equal(gpu.read_state(), ref.state, f"resident state after the tree changed, {samples} samples")
