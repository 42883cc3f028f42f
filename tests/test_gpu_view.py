"""View tier parity: trace_view_paths, and view frames (retain_view_history,
load_shared_faces, trace_visible_paths with paused paths, store_shared_faces)
interleaved with world-cache frames, bit for bit against the oracle."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal, encode_events, lanes_for, terrain_case

pytestmark = pytest.mark.gpu


def world(gpu, case, frames):
    case.load(gpu)
    geometry = gpu.geometry()
    lanes = lanes_for(case.transport, 8)
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                   case.pipe(lanes))
    for f in range(frames):
        gpu.frame(8, clock_ms=16 * f)
        ref.frame(8, clock_ms=16 * f)
    return ref


def receivers_for(faces):
    normals = np.array(vgi.FACE_OFFSETS, np.float32)
    r = np.zeros((faces.shape[0], 8), np.uint32)
    surface = (faces[:, 0:3].astype(np.float32) + np.float32(0.5)) + normals[faces[:, 3]] * np.float32(0.5)
    r[:, 0:3] = surface.astype(np.float32).view(np.uint32)
    r[:, 3] = faces[:, 3]
    r[:, 4:7] = faces[:, 0:3].view(np.uint32)
    return r


def compare_view(gpu, ref, what):
    got = gpu.view_read()
    for key in ("receivers", "paths", "continuations", "estimates", "queue"):
        want = ref.view[key][: got[key].size] if key == "queue" else ref.view[key]
        assert_words_equal(got[key], want, f"{what}: view {key}")
    assert_words_equal(gpu.read_state(), ref.state, f"{what}: world state")
    assert_words_equal(gpu.read_slot_meta(), ref.meta, f"{what}: world slot metadata")
    return compare_flips(gpu, ref, what)


def ordered(a):
    return a[np.lexsort(a.T[::-1])] if len(a) else a


def compare_flips(gpu, ref, what):
    """Reads, and so clears, both sides' sun-flip reports and compares them.
    The GPU takes its record slots by atomics, so which flips get the 2,048
    records is arbitrary: up to 2,048 flips the records compare as a set;
    past that, the GPU's records must be drawn from the oracle's full list
    and the rest must make up the overflow exactly (the biased min/max box
    and the summed round(flux * 64)). Returns the number of flips."""
    records, overflow, count = gpu.view_read_sun_flips()
    want_records, want_overflow, log = ref.view_read_sun_flips()
    assert count == log.shape[0], f"{what}: {count} sun flips, the oracle has {log.shape[0]}"
    if count <= 2048:
        assert_words_equal(ordered(records), ordered(log), f"{what}: sun flips")
        assert_words_equal(overflow, want_overflow, f"{what}: sun-flip overflow")
        return count
    # Multiset difference: the oracle's flips that are not among the GPU's records.
    keys = lambda a: [tuple(r) for r in a]
    pool = {}
    for k in keys(log):
        pool[k] = pool.get(k, 0) + 1
    for k in keys(records):
        assert pool.get(k, 0) > 0, f"{what}: GPU flip record {k} is not one of the oracle's flips"
        pool[k] -= 1
    rest = np.array([k for k, m in pool.items() for _ in range(m)], np.uint32).reshape(-1, 4)
    assert rest.shape[0] == count - 2048
    bias = np.int64(1 << 30)
    v = rest[:, 0:3].view(np.int32).astype(np.int64)
    flux = rest[:, 3].view(np.float32)
    rounded = ((flux * np.float32(64.0)) + np.float32(0.5)).astype(np.uint32)
    expect = np.zeros(7, np.uint32)
    expect[0:3] = (bias - v).max(axis=0).astype(np.uint32)
    expect[3:6] = (v + bias).max(axis=0).astype(np.uint32)
    expect[6] = np.uint32(rounded.astype(np.uint64).sum() & 0xFFFFFFFF)
    assert_words_equal(overflow, expect, f"{what}: sun-flip overflow")
    return count


def test_view_paths_match_oracle(gpu):
    case = terrain_case(bounces=2)
    ref = world(gpu, case, 3)
    faces = case.faces[::7].copy()
    gpu.view_set_receivers(faces)
    receivers = gpu.view_read()["receivers"]
    assert_words_equal(receivers, receivers_for(faces), "receivers")
    got = gpu.view_trace_paths(4)
    want = ref.view_trace_paths(receivers, 4)
    assert_words_equal(got, want, "view paths")
    # Some paths ended at cached faces, some traced on.
    assert (want[:, 23] == 1).any() and (want[:, 15] == 1).any()


@pytest.mark.parametrize("view_first", [False, True])
def test_view_frames_with_pauses_and_handoff_match_oracle(gpu, view_first):
    case = terrain_case(bounces=2, measured_retention=1.0)
    ref = world(gpu, case, 3)
    faces = case.faces[::5].copy()
    gpu.view_set_receivers(faces)
    ref.view_start(gpu.view_read()["receivers"], faces[:, 4])
    n = faces.shape[0]
    c = faces[n // 2, :3]
    events, n_events = encode_events([(c - 3, c + 3, [(c - 3, c + 3, 30.0, 3)])])
    plan = [
        dict(max_hits=1, invocations=n),                       # every path pauses after one hit
        dict(max_hits=1, invocations=n, first=7),              # resumes from a rotated owner
        dict(max_hits=2, invocations=n // 2, first=3),         # a partial wave
        dict(max_hits=8, invocations=2 * n, ticket=(1, 0, 0, 0)),  # a new ticket restarts paused paths
        dict(max_hits=3, invocations=n, depth=3),              # a finite depth
        dict(max_hits=8, invocations=n, events=events, n_events=n_events),  # retention on view history
    ]
    for k, wave in enumerate(plan):
        gpu.view_frame(view_first=view_first, clock_ms=100 + k, **wave)
        ref.view_frame(view_first=view_first, clock_ms=100 + k, measured_retention=1.0, **wave)
        compare_view(gpu, ref, f"view frame {k}")
        # The world cache keeps running between view frames and reads what the view stored.
        gpu.frame(8, clock_ms=200 + k)
        ref.frame(8, clock_ms=200 + k)
        assert_words_equal(gpu.read_results(), ref.results, f"world results after view frame {k}")
    q = ref.view["queue"]
    assert q[2] > 0 and q[3] > 0 and q[10] > 0  # completed, known, cache loads
    status = ref.view["continuations"][:, 19]
    assert set(np.unique(status)) <= {1, 2, 3}


def test_view_without_shared_cache_keeps_its_own_history(gpu):
    case = terrain_case(bounces=2)
    ref = world(gpu, case, 2)
    faces = case.faces[::9].copy()
    gpu.view_set_receivers(faces)
    ref.view_start(gpu.view_read()["receivers"], faces[:, 4])
    for k in range(3):
        gpu.view_frame(max_hits=8, shared=False, clock_ms=k)
        ref.view_frame(max_hits=8, shared=False, clock_ms=k)
        compare_view(gpu, ref, f"unshared view frame {k}")
    est = ref.view["estimates"]
    assert (est[:, 3].view(np.float32) > 0).any() and (est[:, 15] == 0).all()


def test_topology_prior_seeds_new_receivers_like_the_oracle(gpu):
    """bootstrap_face: new view receivers next to world-cache faces with at
    least 16 samples start from those faces' light; a view frame without
    tracing shows the priors, a traced one follows, both equal to the
    oracle's."""
    case = terrain_case(bounces=2)
    ref = world(gpu, case, 3)  # 24 samples a world face
    exposed = vgi.exposed_faces(case.coords, case.vox)
    world_keys = {tuple(r[:4]) for r in case.faces}
    fresh = np.array([r for r in exposed[1::3] if tuple(r[:4]) not in world_keys][:4000], np.int32)
    gpu.view_set_receivers(fresh)
    ref.view_start(gpu.view_read()["receivers"], fresh[:, 4])
    gpu.set_topology_prior(True)
    try:
        gpu.view_frame(max_hits=0, clock_ms=200)
        ref.view_frame(max_hits=0, clock_ms=200, topology=True)
        compare_view(gpu, ref, "priors")
        weights = gpu.view_read()["estimates"].view(np.float32)[:, 3]
        assert (weights == 1.0).sum() > len(fresh) // 2, (weights == 1.0).sum()
        gpu.view_frame(max_hits=4, clock_ms=216)
        ref.view_frame(max_hits=4, clock_ms=216, topology=True)
        compare_view(gpu, ref, "frame after the priors")
    finally:
        gpu.set_topology_prior(False)
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))


def test_sun_corners_are_traced_like_the_oracle(gpu):
    """reproject_paths' corner sun words: faces lit by the sun trace their
    four corners (some lit, some in shadow) and refresh one frame in 4."""
    case = terrain_case(bounces=2)
    ref = world(gpu, case, 1)
    faces = case.faces[::4].copy()
    gpu.view_set_receivers(faces)
    ref.view_start(gpu.view_read()["receivers"], faces[:, 4])
    for k in range(5):
        gpu.view_frame(max_hits=1, clock_ms=300 + k)
        ref.view_frame(max_hits=1, clock_ms=300 + k)
        compare_view(gpu, ref, f"sun corners, view frame {k}")
    corners = gpu.view_read()["estimates"][:, 14]
    traced = corners != 0x80808080
    assert traced.mean() > 0.3
    corner_bytes = np.stack([(corners[traced] >> (8 * k)) & 255 for k in range(4)]).ravel()
    valid = (corner_bytes & 128) != 0
    sees_sun = (corner_bytes & 1) != 0
    assert (valid & sees_sun).any() and (valid & ~sees_sun).any(), "corners in sun and in shadow"
    # The sun turns: as each face refreshes, corners that changed are reported as flips.
    sun = vgi.DirectionalTransportLight((-0.6, 0.5, -0.2), (3.0, 3.0, 3.0)).words()
    gpu.set_lights(sun, 1)
    ref.lights = sun
    flips = 0
    for k in range(4):
        gpu.view_frame(max_hits=1, clock_ms=310 + k)
        ref.view_frame(max_hits=1, clock_ms=310 + k)
        flips += compare_view(gpu, ref, f"sun corners after the sun turned, view frame {k}")
    assert flips > 0
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))


def test_sun_flips_build_up_until_read(gpu):
    """Sun-flip reports are kept across view frames until
    vgi_view_read_sun_flips delivers them (the reference clears its region
    only after a timing receipt copied it): two frames of a turning sun
    without a read in between deliver both frames' flips, past the 2,048
    records into the overflow box."""
    case = terrain_case(bounces=2)
    ref = world(gpu, case, 1)
    faces = case.faces.copy()
    gpu.view_set_receivers(faces)
    ref.view_start(gpu.view_read()["receivers"], faces[:, 4])
    for k in range(4):  # every receiver traces its corners at least once
        gpu.view_frame(max_hits=1, clock_ms=400 + k)
        ref.view_frame(max_hits=1, clock_ms=400 + k)
    compare_view(gpu, ref, "corners before the sun turns")
    counts = []
    for k, direction in enumerate([(-0.6, 0.5, -0.2), (0.1, 0.6, 0.8)]):
        sun = vgi.DirectionalTransportLight(direction, (3.0, 3.0, 3.0)).words()
        gpu.set_lights(sun, 1)
        ref.lights = sun
        for j in range(4):  # one frame in four refreshes each receiver
            gpu.view_frame(max_hits=1, clock_ms=410 + 4 * k + j)
            ref.view_frame(max_hits=1, clock_ms=410 + 4 * k + j)
        counts.append(int(ref.view["queue"][12 + 2 * faces.shape[0]]))
    assert counts[0] > 0 and counts[1] > counts[0], counts
    total = compare_view(gpu, ref, "flips of eight frames read at once")
    assert total == counts[1] > 2048, counts
    # Read: the region starts over.
    records, overflow, count = gpu.view_read_sun_flips()
    assert count == 0 and len(records) == 0 and not overflow.any()
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))


def test_sun_flips_of_faces_that_reenter_view(gpu):
    """A receiver that leaves the view keeps its corner words in its world
    slot; when it re-enters after the sun turned, its fresh corners are
    compared with the kept ones and the change is reported (the re-entry
    branch of report_sun_flips), in the first view frame after re-entry, when
    no refresh can report yet."""
    case = terrain_case(bounces=2)
    ref = world(gpu, case, 1)
    faces = case.faces.copy()
    gpu.view_set_receivers(faces)
    ref.view_start(gpu.view_read()["receivers"], faces[:, 4])
    for k in range(4):
        gpu.view_frame(max_hits=1, clock_ms=500 + k)
        ref.view_frame(max_hits=1, clock_ms=500 + k)
    compare_view(gpu, ref, "corners kept by the world slots")
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))
    sun = vgi.DirectionalTransportLight((-0.6, 0.5, -0.2), (3.0, 3.0, 3.0)).words()
    gpu.set_lights(sun, 1)
    ref.lights = sun
    gpu.view_set_receivers(faces)
    ref.view_start(gpu.view_read()["receivers"], faces[:, 4])
    gpu.view_frame(max_hits=1, clock_ms=520)
    ref.view_frame(max_hits=1, clock_ms=520)
    count = compare_view(gpu, ref, "first view frame after re-entry")
    assert count > 0
    gpu.view_set_receivers(np.zeros((0, 5), np.int32))
