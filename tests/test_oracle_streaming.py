"""The oracle's region streaming (orc_scene_regions, TransportScene::
with_page_contents with region-sized pages) on the CPU: after random loads,
replacements and unloads, the packed scene equals a fresh pack of the same
regions apart from the top-level extents, and the incrementally updated
top-level field is a valid fixed point of NAADF's merging rule
(src/world.rs:596-684), which is all the reference promises of it."""
import numpy as np

import oracle_lib as O
from test_oracle_pins import assert_valid_fixed_point


def test_streamed_scene_equals_a_fresh_pack_and_keeps_a_valid_field():
    rng = np.random.default_rng(8)
    pool = {}
    for z in range(5):
        for y in range(3):
            for x in range(6):
                v = np.full(4096, 256, np.uint16)
                if rng.random() < 0.35:
                    v[rng.integers(0, 4096, size=int(rng.integers(1, 40)))] = int(rng.integers(0, 8))
                pool[(x, y, z)] = v
    keys = sorted(pool, key=lambda k: (k[2], k[1], k[0]))
    resident = set(keys[::2])
    first = sorted(resident, key=lambda k: (k[2], k[1], k[0]))
    scene = O.Scene(np.array(first, np.int32), np.stack([pool[k] for k in first]), top_mode=0)
    all_coords = np.array(keys, np.int32)
    for step in range(12):
        out = [k for k in resident if rng.random() < 0.3]
        back = [k for k in keys if k not in resident and rng.random() < 0.4]
        for k in [k for k in resident if k not in out and rng.random() < 0.15]:
            v = pool[k].copy()
            v[rng.integers(0, 4096, size=8)] = 256 if rng.random() < 0.5 else 5
            pool[k] = v
            back.append(k)
        scene.regions(np.array(back, np.int32).reshape(-1, 3), np.stack([pool[k] for k in back]) if back else None,
                      removed=np.array(out, np.int32).reshape(-1, 3))
        resident = (resident - set(out)) | set(back)
        live = sorted(resident, key=lambda k: (k[2], k[1], k[0]))
        fresh = O.Scene(np.array(live, np.int32), np.stack([pool[k] for k in live]), top_mode=0)
        got = O.canonical(*scene.arrays()[:3], all_coords)
        want = O.canonical(*fresh.arrays()[:3], all_coords)
        assert (scene.arrays()[3] == fresh.arrays()[3]).all()
        got[:, 2:4] = 0
        want[:, 2:4] = 0
        assert (got == want).all(), step
        assert ((got[:, 0] == 0) == [tuple(c) not in resident for c in keys]).all()
        assert_valid_fixed_point(scene, {k: pool[k] for k in resident})
