"""The oracle's restatement of the GPU world-cache scheduler (candidate,
select_* in voxel_accumulate.wgsl:448-695) on crafted slot metadata: the
class of every face, the per-class quotas and the lending of unused share."""
import numpy as np

import oracle_lib as O

URGENT, LIVE = 0x40000000, 8


def metadata(rows):
    """rows: (voxel xyz, count, urgent, noise) per slot; every slot live,
    traced long ago (age past the audit interval keeps it due)."""
    n = len(rows)
    meta = np.zeros((n, 12), np.uint32)
    for s, (v, count, urgent, noise) in enumerate(rows):
        meta[s, 0:3] = np.asarray(v, np.int32).view(np.uint32)
        meta[s, 3] = LIVE
        meta[s, 8] = np.float32(noise).view(np.uint32)
        meta[s, 9] = 0  # last merge at clock 0
        meta[s, 10] = np.float32(1.0).view(np.uint32)
        meta[s, 11] = 0x80000000 | count | (URGENT if urgent else 0)
    return meta


def controls(n, budget, focus=(0, 0, 0), clock=10_000, audit=1000):
    ctl = np.zeros(36, np.uint32)
    ctl[0] = budget
    ctl[2] = clock
    ctl[14] = n
    ctl[16] = 1
    ctl[18] = 64
    ctl[19] = audit
    ctl[20:23] = np.asarray(focus, np.int32).view(np.uint32)
    ctl[23] = budget
    ctl[25] = 100
    ctl[26], ctl[27] = 0, n
    return ctl


def select(meta, budget, **kw):
    n = meta.shape[0]
    ctl = controls(n, budget, **kw)
    state = np.zeros((n, 36), np.uint32)
    keys = np.full(n, 0xFFFFFFFF, np.uint32)
    sel = np.zeros(1038, np.uint32)
    tasks = np.zeros((budget, 8), np.uint32)
    slots = np.full(budget, 0xFFFFFFFF, np.uint32)
    picks = np.full((budget, 4), 0xFFFFFFFF, np.uint32)
    pre = np.full(n, 0xFFFFFFFF, np.uint32)
    O.lib().orc_classify(O.ptr(meta), O.ptr(pre), n, O.ptr(ctl))
    O.lib().orc_select(O.ptr(state), O.ptr(meta), O.ptr(keys), n, O.ptr(ctl), O.ptr(sel), O.ptr(tasks), O.ptr(slots), O.ptr(picks))
    return pre, sel, slots[slots != 0xFFFFFFFF]


def test_classes_follow_count_urgency_and_distance():
    rows = [((0, 0, 0), 2, False, 0.5),        # coverage: fewer than 8 samples
            ((10, 0, 0), 100, False, 0.5),     # refinement: same page as the focus
            ((500, 0, 0), 100, False, 0.5),    # sweep: far pages
            ((500, 0, 0), 100, True, 0.5)]     # urgent
    pre, _, _ = select(metadata(rows), 4)
    assert (pre >> 8).tolist() == [0, 1, 2, 3]


def test_quotas_split_the_budget_and_lend_unused_share():
    rng = np.random.default_rng(3)
    rows = []
    rows += [((int(rng.integers(0, 64)), 0, 0), 1, False, 0.5) for _ in range(100)]      # coverage
    rows += [((int(rng.integers(0, 64)), 0, 0), 100, False, float(rng.uniform(0.1, 4))) for _ in range(100)]  # refinement
    rows += [((1000 + k, 0, 0), 100, False, 0.5) for k in range(100)]                    # sweep
    meta = metadata(rows)
    pre, sel, picked = select(meta, 40)
    cls = pre[picked] >> 8
    # No urgent faces: coverage 1/4, refinement 1/2, sweep the rest.
    assert np.bincount(cls, minlength=4).tolist() == [10, 20, 10, 0]
    # Refinement picks the highest priorities (lowest buckets) first.
    ref_keys = pre[(pre >> 8) == 1] & 255
    assert (pre[picked][cls == 1] & 255).max() <= np.sort(ref_keys)[19]
    # Only 5 coverage faces: their unused share goes to refinement first.
    rows2 = rows[:5] + rows[100:]
    pre2, sel2, picked2 = select(metadata(rows2), 40)
    assert np.bincount(pre2[picked2] >> 8, minlength=4).tolist() == [5, 25, 10, 0]
    # Urgent faces take at most three quarters of the budget.
    rows3 = rows + [((2000 + k, 0, 0), 100, True, 0.5) for k in range(100)]
    pre3, _, picked3 = select(metadata(rows3), 40)
    counts = np.bincount(pre3[picked3] >> 8, minlength=4).tolist()
    assert counts[3] == 30 and sum(counts) == 40 and counts[:3] == [2, 5, 3]


def test_fresh_stable_faces_wait_for_the_audit_interval():
    rows = [((0, 0, 0), 100, False, 0.5)]
    meta = metadata(rows)
    meta[0, 5] = 8 | 4          # fresh and stable for 4 batches
    meta[0, 7] = 1              # this transport revision
    meta[0, 9] = 9_500          # merged 500 ms before the clock
    pre, _, _ = select(meta.copy(), 1, audit=1000)
    assert pre[0] == 0xFFFFFFFF
    pre, _, _ = select(meta.copy(), 1, audit=400)
    assert pre[0] != 0xFFFFFFFF
