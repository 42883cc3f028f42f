"""Scheduled frames: the GPU world-cache scheduler (voxel_accumulate.wgsl:
448-695) against the oracle's serial restatement. Keys, histograms,
thresholds and counts are exact; the picked set follows the thresholds
(which tied faces it takes depends on block order, as on the reference's
GPU); tracing and accumulating the GPU's picks matches the oracle doing the
same, word for word."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal, lanes_for, terrain_case

pytestmark = pytest.mark.gpu

SAMPLES = 8


def controls(ref, n, budget, focus, first, end, audit_ms, clock_ms):
    ctl = O.controls_words(n, SAMPLES, clock_ms, ref.transport, ref.batch_id)
    ctl[0] = budget
    ctl[19] = audit_ms
    ctl[20:23] = np.asarray(focus, np.int32).view(np.uint32)
    ctl[23] = budget
    ctl[24] = 0
    ctl[26], ctl[27] = first, end
    ctl[32] = 0
    return ctl


@pytest.mark.parametrize("budget_share,first_frames", [(3, 3), (10, 1)])
def test_scheduled_frames_match_oracle(gpu, budget_share, first_frames):
    case = terrain_case(bounces=2)
    case.load(gpu)
    geometry = gpu.geometry()
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                   case.pipe(lanes_for(case.transport, SAMPLES)))
    n = ref.n
    # Plain frames first, so the faces have counts, errors and ages; the
    # face set's second half has none (never traced).
    half = n // 2
    for f in range(first_frames):
        gpu.frame_shard(SAMPLES, 16 * f, 0, half)
        ref.frame_shard(SAMPLES, 16 * f, 0, half)
    keys = np.full(n, 0xFFFFFFFF, np.uint32)
    focus = (40, 30, 50)
    classes_seen, contested = set(), False
    # A face the plain frames traced is the CPU's for 4 batches (its
    # readback window), so the later scheduled frames see more classes.
    for f in range(first_frames, first_frames + 6):
        budget = n // budget_share
        clock = 16 * f + 500
        ctl = controls(ref, n, budget, focus, 0, n, 120, clock)
        before_meta = ref.meta.copy()
        gpu.frame_scheduled(SAMPLES, clock, budget, focus=focus, classify=(0, n), audit_ms=120)
        got = gpu.read_selection()
        # Keys, histograms, thresholds, tie and pick counts.
        pre_keys = keys.copy()
        lib = O.lib()
        lib.orc_classify(O.ptr(before_meta), O.ptr(pre_keys), n, O.ptr(ctl))
        sel = np.zeros(1038, np.uint32)
        meta_copy, keys_copy = before_meta.copy(), keys.copy()
        tasks = np.zeros((budget, 8), np.uint32)
        slots = np.full(budget, 0xFFFFFFFF, np.uint32)
        picks = np.zeros((budget, 4), np.uint32)
        lib.orc_select(O.ptr(ref.state), O.ptr(meta_copy), O.ptr(keys_copy), n, O.ptr(ctl), O.ptr(sel), O.ptr(tasks), O.ptr(slots),
                       O.ptr(picks))
        assert_words_equal(got["selection"], sel, "selection words")
        threshold, remainder = sel[1024:1028], sel[1028:1032]
        hist = sel[:1024].reshape(4, 256).sum(axis=1)
        classes_seen |= set(np.nonzero(hist)[0].tolist())
        contested = contested or (hist.sum() > budget and (threshold < 256).any())
        # The GPU's picks: all below the thresholds, `remainder` ties per class.
        valid = got["picks"][:, 0] != 0xFFFFFFFF
        gpu_slots = got["picks"][valid, 0]
        assert len(set(gpu_slots.tolist())) == gpu_slots.size == min(int(sel[1036]), budget)
        k = pre_keys[gpu_slots]
        cls, bucket = np.minimum(k >> 8, 3), k & 255
        assert (k != 0xFFFFFFFF).all() and (bucket <= threshold[cls]).all()
        for c in range(4):
            below = (pre_keys != 0xFFFFFFFF) & (np.minimum(pre_keys >> 8, 3) == c) & ((pre_keys & 255) < threshold[c])
            assert set(np.nonzero(below)[0].tolist()) <= set(gpu_slots.tolist())
            assert int(((cls == c) & (bucket == threshold[c])).sum()) == (remainder[c] if threshold[c] < 256 else 0)
        # Keys after the frame: classified, picked ones cleared.
        want_keys = pre_keys.copy()
        want_keys[gpu_slots] = 0xFFFFFFFF
        assert_words_equal(got["keys"], want_keys, "keys after emit")
        keys = want_keys
        # The oracle traces and accumulates the GPU's picks.
        task_rows = got["tasks"].copy()
        pick_slots = np.where(valid, got["picks"][:, 0], 0xFFFFFFFF).astype(np.uint32)
        records = np.where(valid[:, None], got["picks"], 0xFFFFFFFF).astype(np.uint32)
        # Each pick's task and record from the slot's state before the frame:
        # (voxel, face, current sequence) and (slot, revision tag, merged
        # count, incarnation).
        want_tasks = np.zeros((valid.sum(), 8), np.uint32)
        want_tasks[:, 0:3] = before_meta[gpu_slots, 0:3]
        want_tasks[:, 3] = before_meta[gpu_slots, 3] & 7
        want_tasks[:, 4] = ref.state[gpu_slots, 6]
        assert_words_equal(task_rows[valid][:, :5], want_tasks[:, :5], "pick tasks")
        ref_records = records.copy()
        ref_records[valid, 1] = before_meta[gpu_slots, 6]
        ref_records[valid, 2] = 0
        ref_records[valid, 3] = ref.state[gpu_slots, 28]
        lib.orc_mark_changed(O.ptr(ref.state), O.ptr(ref.meta), O.ptr(pick_slots), budget, O.ptr(ctl))
        params = ref.params_fn(budget, SAMPLES)
        out, _ = O.trace_faces(ref.geometry, params, ref.materials, ref.lights, ref.emitter_words, task_rows, ref.pipe, ref.state,
                               ref.index)
        lib.orc_accumulate_picks(O.ptr(ref.state), O.ptr(ref.meta), O.ptr(ref.checkpoint), O.ptr(out), O.ptr(pick_slots), budget,
                                 O.ptr(ctl), O.ptr(ref_records))
        ref.batch_id = (ref.batch_id + 1) & 0x0FFFFFFF or 1
        assert_words_equal(got["results"][valid], out[valid], "pick results")
        assert_words_equal(got["picks"][valid], ref_records[valid], "pick records")
        assert_words_equal(gpu.read_state(), ref.state, "state after the scheduled frame")
        assert_words_equal(gpu.read_slot_meta(), ref.meta, "slot metadata after the scheduled frame")
    assert len(classes_seen) >= 2 and contested, (classes_seen, contested)


def test_schedule_refuses_bad_budgets(gpu):
    case = terrain_case(bounces=2)
    case.load(gpu)
    n = case.faces.shape[0]
    with pytest.raises(vgi.VgiError, match="budget"):
        gpu.frame_scheduled(8, 0, 0)
    with pytest.raises(vgi.VgiError, match="budget"):
        gpu.frame_scheduled(8, 0, n + 1)
    with pytest.raises(vgi.VgiError, match="range"):
        gpu.frame_scheduled(8, 0, 16, classify=(0, n + 1))
