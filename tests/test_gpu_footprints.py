"""Change footprints (trace_footprints / finish_footprints): where a changed
box's shadow lands along the sun becomes its reserved Light event, before
retention reads the events. GPU against the oracle, word for word."""
import numpy as np
import pytest

import oracle_lib as O
from test_gpu_parity import assert_words_equal, encode_events, run_frames, terrain_case

pytestmark = pytest.mark.gpu

EMPTY_LO, EMPTY_HI = np.full(3, 1 << 29), np.full(3, -(1 << 29))


def encode_footprints(boxes, events):
    """encode_footprints (src/gpu/resident.rs:1270-1310): the count, then per
    (box, event) its header record, bound record, first thread and grid."""
    first_bound, first = [], 0
    for _, _, items in events:
        first_bound.append(first)
        first += len(items)
    records = len(events) * 3
    words = [[len(boxes), 0, 0, 0]]
    threads = 0
    for (lo, hi), event in boxes:
        size = np.asarray(hi) - np.asarray(lo) + 1
        grid = int(min(max(np.ceil(np.sqrt(float((size.astype(np.float32) ** 2).sum()))), 1.0), 64.0))
        words += [[lo[0], lo[1], lo[2], event * 3], [hi[0], hi[1], hi[2], records + first_bound[event] * 2], [threads, grid, 0, 0]]
        threads += grid * grid
    return np.array(words, np.int32), threads


def events_with_footprints(boxes):
    """plan_footprints: one edit event per box, then one reserved Light event
    (empty union and bound) per box."""
    events = [(lo, hi, [(lo, hi, 40.0, 3)]) for lo, hi in boxes]
    events += [(EMPTY_LO, EMPTY_HI, [(EMPTY_LO, EMPTY_HI, 0.0, 4)]) for _ in boxes]
    plan = [((lo, hi), len(boxes) + k) for k, (lo, hi) in enumerate(boxes)]
    return events, plan


def test_footprints_fill_light_events_like_the_oracle(gpu):
    case = terrain_case(bounces=2, measured_retention=1.0)
    ref = run_frames(gpu, case, 3, 8)
    top = case.faces[case.faces[:, 3] == 2]  # +y faces: the ground seen from above
    c = top[len(top) // 2, :3]
    air = (c + np.array([-2, 6, -2]), c + np.array([2, 8, 2]))          # a block in the air: its shadow lands below
    buried = (c + np.array([-1, -6, -1]), c + np.array([1, -4, 1]))     # inside the ground: tubes land nowhere
    boxes = [air, buried]
    events, plan = events_with_footprints(boxes)
    words, n = encode_events(events)
    fp, threads = encode_footprints(plan, events)
    got = gpu.apply_events_footprints(words, n, fp)
    want = words.copy()
    sums = np.zeros((len(plan), 8), np.uint32)
    sums[:, 0:3] = 0xFFFFFFFF
    d, h, cl, bounds = ref.geometry
    params = ref.params_fn(ref.n, 8)
    cells = cl if len(cl) else np.zeros(1, np.uint32)
    lights = np.ascontiguousarray(case.lights, np.float32)
    rc = O.lib().orc_footprints(O.ptr(O.c(d, np.int32)), d.size // 4, O.ptr(O.c(h, np.uint32)), O.ptr(O.c(cells, np.uint32)),
                                O.ptr(params), O.ptr(O.c(case.materials, np.float32)), O.ptr(lights), O.ptr(fp), threads,
                                O.ptr(sums), O.ptr(want))
    assert rc == 0
    assert_words_equal(got, want, "event words after footprints")
    # Records: 4 event headers (3 each), then one bound (2 records) per event;
    # the reserved Light events are the last two.
    records = want.reshape(-1, 4)
    air_bound, buried_bound = records[n * 3 + 4: n * 3 + 6], records[n * 3 + 6: n * 3 + 8]
    lo, hi = air_bound[0, :3].view(np.int32), air_bound[1, :3].view(np.int32)
    assert (lo <= hi).all() and air_bound[0, 3:4].view(np.float32)[0] > 0 and air_bound[1, 3] == 4
    assert lo[1] < air[0][1]  # the shadow lands below the block
    assert (buried_bound[0, :3].view(np.int32) == EMPTY_LO).all() and (buried_bound[1, :3].view(np.int32) == EMPTY_HI).all()
    # Retention reads the filled events the same way.
    ref.apply_events(want, n)
    assert_words_equal(gpu.read_state(), ref.state, "state after footprint events")
    assert_words_equal(gpu.read_slot_meta(), ref.meta, "slot metadata after footprint events")
