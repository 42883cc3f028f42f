"""Pins of the CPU oracle against the reference's own known answers.

Each test restates one of the reference's tests (file:line within
crates/bevy_voxel_gi/src/) and checks the oracle with it, so the oracle is
trusted before it judges the CUDA kernels.
"""
import math
import struct

import numpy as np
import pytest

import oracle_lib as O


def lcg_blocked(n, divisor, state):
    out = []
    for _ in range(n):
        state = (state * 747_796_405 + 2_891_336_453) & 0xFFFFFFFF
        out.append(divisor != 0 and state % divisor == 0)
    return out, state


def full_sweep_reference(size, blocked):
    """naadf/construction_tests.rs:6-96, restated: Jacobi sweeps without the
    closed form for all-empty volumes."""
    sx, sy, sz = size
    n = sx * sy * sz
    src = [[0] * 6 for _ in range(n)]
    dst = [[0] * 6 for _ in range(n)]
    rounds = max(max(size) - 1, 0)

    def idx(x, y, z):
        return x + sx * (y + sy * z)

    def grow(cur, nb, d, source):
        if any(v < 0 for v in nb) or nb[0] >= sx or nb[1] >= sy or nb[2] >= sz:
            return
        if cur[d] == 255:
            return
        ni = idx(*nb)
        if blocked[ni]:
            return
        opp = d ^ 1
        for b in range(6):
            if b != opp and source[ni][b] < cur[b]:
                return
        cur[d] += 1

    for _ in range(rounds):
        for axis in range(3):
            for z in range(sz):
                for y in range(sy):
                    for x in range(sx):
                        i = idx(x, y, z)
                        if blocked[i]:
                            dst[i] = [0] * 6
                            continue
                        cur = list(src[i])
                        a = [0, 0, 0]
                        a[axis] = 1
                        grow(cur, (x - a[0], y - a[1], z - a[2]), axis * 2, src)
                        grow(cur, (x + a[0], y + a[1], z + a[2]), axis * 2 + 1, src)
                        dst[i] = cur
            src, dst = dst, src
    return np.array(src, np.uint8).reshape(-1, 6)


def test_empty_four_cubed_grid_expands_to_every_edge():
    # naadf.rs:201-208
    f = O.build_aadf((4, 4, 4), np.zeros(64, np.uint8))
    at = f[1 + 4 * (2 + 4 * 1)]
    assert tuple(at[[0, 2, 4]]) == (1, 2, 1)
    assert tuple(at[[1, 3, 5]]) == (2, 1, 2)


def test_every_generated_bound_contains_only_empty_cells():
    # naadf.rs:165-199
    size = (9, 7, 8)
    blocked, _ = lcg_blocked(9 * 7 * 8, 7, 0x12345678)
    f = O.build_aadf(size, np.array(blocked, np.uint8))
    b = np.array(blocked).reshape(8, 7, 9)
    for z in range(8):
        for y in range(7):
            for x in range(9):
                i = x + 9 * (y + 7 * z)
                if blocked[i]:
                    assert not f[i].any()
                    continue
                lo = (x - f[i][0], y - f[i][2], z - f[i][4])
                hi = (x + f[i][1], y + f[i][3], z + f[i][5])
                assert not b[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1].any()


def test_construction_matches_full_sweep_oracle():
    # naadf/construction_tests.rs:112-145 (sizes up to 17x3x11 and the 255-long axes)
    for bits in range(256):
        blocked = [(bits >> i) & 1 for i in range(8)]
        assert (O.build_aadf((2, 2, 2), np.array(blocked, np.uint8)) == full_sweep_reference((2, 2, 2), blocked)).all()
    state = 0x12345678
    for size in [(1, 1, 1), (4, 4, 4), (9, 7, 8), (17, 3, 11), (255, 1, 1), (1, 255, 1), (1, 1, 255)]:
        for divisor in [0, 1, 2, 7, 29]:
            blocked, state = lcg_blocked(int(np.prod(size)), divisor, state)
            got = O.build_aadf(size, np.array(blocked, np.uint8))
            assert (got == full_sweep_reference(size, blocked)).all(), (size, divisor)


def test_curve_limit_matches_the_selected_whole_range_curve():
    # retention.rs:346-376: H(d) = round((d / 12)^4), NO_LIMIT at the ceiling.
    for d, expected in [(0, 0), (8, 0), (16, 3), (24, 16), (32, 51), (48, 256), (64, 809), (96, 4096), (128, 12945),
                        (192, 0xFFFFFFFF), (384, 0xFFFFFFFF)]:
        assert O.lib().orc_curve_limit(d * d) == expected, d
    for d2 in range(0, 36864, 7):
        expected = round((math.sqrt(d2) / 12.0) ** 4)
        expected = 0xFFFFFFFF if expected >= 65536 else expected
        assert O.lib().orc_curve_limit(d2) == expected, d2


def scalar_box_reference(position, direction, cell, negative, positive, size):
    """gpu/traversal_tests.rs:15-39 restated: the scalar XYZ policy."""
    f32 = np.float32
    mn = [f32(f32(cell[a] - negative[a]) * f32(size)) for a in range(3)]
    mx = [f32(f32(cell[a] + positive[a] + 1) * f32(size)) for a in range(3)]
    distance = f32(1e30)
    normal = [0.0, 0.0, 0.0]
    for a in range(3):
        d = f32(direction[a])
        if abs(d) <= f32(1e-8):
            continue
        plane = mx[a] if d > 0 else mn[a]
        travel = f32(f32(plane - f32(position[a])) / d)
        if travel >= f32(-0.001) and travel < distance:
            distance = max(travel, f32(0.0))
            normal = [0.0, 0.0, 0.0]
            normal[a] = -1.0 if d > 0 else 1.0
    return normal, f32(max(f32(distance + f32(0.001)), f32(0.001)))


def test_box_steps_match_scalar_boundary_policy():
    # gpu/traversal_tests.rs:41-79: the generated case grid (subsampled in
    # direction components to keep the CPU suite short).
    comps = [-1.0, -1.01e-8, -1e-8, -0.99e-8, -0.0, 0.0, 0.99e-8, 1e-8, 1.01e-8, 1.0]
    rng = np.random.default_rng(5)
    case = np.zeros(16, np.float32)
    out = np.zeros(4, np.float32)
    u = case.view(np.uint32)
    checked = 0
    for size in [1.0, 4.0, 16.0]:
        for base in [-4096, -16, -1, 0, 1, 16, 4096]:
            cell = (base, -base, int(base / 2))
            for fraction in [-0.0005, 0.0, 0.5, 1.0, 1.0005]:
                for extent in [(0, 0, 0), (3, 2, 1)]:
                    dirs = [(x, y, z) for x in comps for y in comps for z in comps]
                    for k in rng.choice(len(dirs), 60, replace=False):
                        x, y, z = dirs[k]
                        pos = [np.float32(np.float32(c + np.float32(fraction)) * np.float32(size)) for c in cell]
                        case[0:3] = pos
                        case[3] = size
                        case[4:7] = (x, y, z)
                        u[7:10] = np.array(cell, np.int32).view(np.uint32)
                        u[10:13] = np.array(extent, np.int32).view(np.uint32)
                        u[13:16] = np.array(extent, np.int32).view(np.uint32)
                        O.lib().orc_advance_box(O.ptr(case), O.ptr(out))
                        n, d = scalar_box_reference(pos, (x, y, z), cell, extent, extent, size)
                        assert list(out[:3]) == n, (pos, (x, y, z))
                        assert abs(float(out[3]) - float(d)) <= 1e-5 * (1.0 + abs(float(d)))
                        checked += 1
    # The unequal negative crossings case (traversal_tests.rs:69-77).
    case[0:3] = (1.0009, 1.0001, 1.0002)
    case[3] = 1.0
    case[4:7] = (1.0, 1.0, 1.0)
    u[7:16] = 0
    O.lib().orc_advance_box(O.ptr(case), O.ptr(out))
    n, d = scalar_box_reference(case[0:3], (1.0, 1.0, 1.0), (0, 0, 0), (0, 0, 0), (0, 0, 0), 1.0)
    assert list(out[:3]) == n and abs(out[3] - d) <= 1e-5 * (1 + abs(d))
    assert checked > 10000


def test_face_index_matches_a_map():
    # gpu/face_index.rs:221-260 (insertions; the product builds the index once per face set)
    state = 12345
    seen = {}
    faces = []
    for step in range(6000):
        state = O.lib().orc_pcg(state ^ step)
        voxel = ((state % 23) - 11, (state >> 8) % 7, -((state >> 16) % 19))
        face = (state >> 24) % 6
        if (voxel, face) in seen:
            continue
        seen[(voxel, face)] = len(faces)
        faces.append((*voxel, face))
    table = O.face_index(np.array(faces, np.int32))
    mask = int(table[0, 0])
    assert table[0, 1] == 64
    entries = table[1:]
    assert entries.shape[0] == mask + 1
    found = {}
    for i, e in enumerate(entries):
        if e[3] == 0xFFFFFFFF:
            continue
        key = (tuple(int(v) for v in e[:3].view(np.int32)), int(e[3] >> 29))
        found[key] = int(e[3] & 0x1FFFFFFF)
    assert found == seen
    assert (entries[:, 3] != 0xFFFFFFFF).sum() * 2 <= mask + 1


def test_top_level_field_is_a_valid_fixed_point():
    # world.rs:596-684 assert_valid_fixed_point: every box empty, none can grow.
    rng = np.random.default_rng(3)
    coords, vox = [], []
    for z in range(6):
        for y in range(3):
            for x in range(7):
                if rng.random() < 0.15:
                    continue  # missing region = barrier
                v = np.full(4096, 256, np.uint16)
                if rng.random() < 0.3:
                    v[rng.integers(0, 4096)] = 3
                coords.append((x, y, z))
                vox.append(v)
    scene = O.Scene(np.array(coords), np.concatenate(vox), top_mode=0)
    assert_valid_fixed_point(scene, {tuple(c): v for c, v in zip(coords, vox)})


def assert_valid_fixed_point(scene, present):
    """world.rs:596-684 assert_valid_fixed_point on the oracle scene's
    top-level field: every box holds only loaded empty regions inside the
    bounds, and no box can grow by the merging rule. `present` maps region
    coordinates to their voxels."""
    field = scene.top_level()
    bounds = scene.arrays()[3]
    size = bounds[3:] - bounds[:3] + 1
    blocked = np.ones(tuple(size[::-1]), bool)
    for (x, y, z), v in present.items():
        blocked[z - bounds[2], y - bounds[1], x - bounds[0]] = (v != 256).any()
    f = field.reshape(size[2], size[1], size[0], 6)
    for z in range(size[2]):
        for y in range(size[1]):
            for x in range(size[0]):
                e = f[z, y, x]
                if blocked[z, y, x]:
                    assert not e.any()
                    continue
                lo = (x - e[0], y - e[2], z - e[4])
                hi = (x + e[1], y + e[3], z + e[5])
                assert min(lo) >= 0 and hi[0] < size[0] and hi[1] < size[1] and hi[2] < size[2]
                assert not blocked[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1].any()
                for d in range(6):
                    a = d // 2
                    n = [x, y, z]
                    n[a] += -1 if d % 2 == 0 else 1
                    if min(n) < 0 or n[0] >= size[0] or n[1] >= size[1] or n[2] >= size[2]:
                        continue
                    if blocked[n[2], n[1], n[0]] or e[d] == 255:
                        continue
                    ne = f[n[2], n[1], n[0]]
                    can = all(ne[b] >= e[b] for b in range(6) if b != (d ^ 1))
                    assert not can, ((x, y, z), d)


def test_own_sine_cosine_and_exp_are_accurate():
    s = np.zeros(1, np.float32)
    c = np.zeros(1, np.float32)
    for x in np.linspace(0.0, 6.2831855, 20001, dtype=np.float32):
        O.lib().orc_sincos(float(x), O.ptr(s), O.ptr(c))
        assert abs(float(s[0]) - math.sin(float(x))) <= 2.5e-7
        assert abs(float(c[0]) - math.cos(float(x))) <= 2.5e-7
    for x in np.linspace(-80.0, 80.0, 20001, dtype=np.float32):
        e = O.lib().orc_exp(float(x))
        ref = math.exp(float(x))
        assert abs(e - ref) <= 4e-7 * ref


def test_halton_dimensions_are_rotated_radical_inverses():
    # voxel_path.wgsl:187-201: dims < 12 are radical inverses of (seq & 0xffffff) + 1
    # in prime bases, rotated by a per-stream hash, wrapped to [0, 1).
    primes = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37]
    for dim in range(12):
        for seq in [0, 1, 7, 100, 12345, 0xFFFFFF, 0x1000003]:
            stream = 0xDEADBEEF ^ dim
            idx = (seq & 0xFFFFFF) + 1
            base = primes[dim]
            value, scale = 0.0, 1.0
            while idx:
                scale /= base
                value += (idx % base) * scale
                idx //= base
            rot = (O.lib().orc_pcg(stream ^ O.lib().orc_pcg(dim)) >> 9) / 8388608.0
            expect = (value + rot) % 1.0
            got = O.lib().orc_sample_1d(stream, seq, dim)
            assert 0.0 <= got < 1.0
            assert abs(got - expect) < 1e-5 or abs(abs(got - expect) - 1.0) < 1e-5


def test_hemisphere_directions_are_unit_and_upper():
    out = np.zeros(3, np.float32)
    rng = np.random.default_rng(1)
    for face in range(6):
        n = np.zeros(3, np.float32)
        n[face // 2] = -1.0 if face & 1 else 1.0
        for _ in range(200):
            u, v = rng.random(2)
            O.lib().orc_hemisphere(O.ptr(n), float(u), float(v), O.ptr(out))
            assert abs(np.linalg.norm(out) - 1.0) < 1e-5
            assert float(np.dot(out, n)) >= -1e-6


def test_measured_edit_flux_is_own_plus_brightest_neighbour_light_twice_per_voxel():
    # finish_edits (voxel_accumulate.wgsl:407-423): flux = own + brightest * 2 * voxels,
    # brightest = albedo_lum * (mean_lum + direct_lum) + emission_lum over the scan's
    # traced faces; a scan with no traced face marks the bound unknown (kind 0).
    faces = np.array([[4, 5, 6, 2], [4, 5, 6, 3], [9, 9, 9, 0]], np.int32)
    index = O.face_index(faces)
    state = np.zeros((3, 36), np.uint32)
    meta = np.zeros((3, 12), np.uint32)
    meta[:, 0:3] = faces[:, 0:3].view(np.uint32)
    meta[:, 3] = faces[:, 3].astype(np.uint32) | 8 | (np.array([7, 7, 9], np.uint32) << 16)
    sf = state.view(np.float32)
    sf[0, 0:3] = [1.0, 1.0, 1.0]   # mean
    sf[0, 16:19] = [0.5, 0.5, 0.5]  # direct
    state[0, 5] = 20                 # count
    sf[1, 0:3] = [4.0, 4.0, 4.0]
    state[1, 5] = 0                  # never traced: ignored
    sf[2, 0:3] = [9.0, 9.0, 9.0]
    state[2, 5] = 3                  # outside both scans
    light = np.zeros((256, 2), np.float32)
    light[7] = [0.5, 0.25]
    light[9] = [1.0, 1.0]
    # Two bounds: the first scans the 3^3 voxels around (4, 5, 6), which hold
    # one traced and one untraced face; the second scans empty space.
    words = np.zeros((3 + 4) * 4, np.uint32)
    words[0:12] = [0, 0, 0, 0, 8, 8, 8, 0, 0, 0, 0, 2]
    words[12:16] = [4, 5, 6, np.float32(2.0).view(np.uint32)]
    words[16:20] = [4, 5, 6, 6 | 8]
    words[20:24] = [50, 50, 50, np.float32(1.0).view(np.uint32)]
    words[24:28] = [50, 50, 50, 6]
    measures = np.array([[3, 0, 27, 2], [3, 4, 5, np.float32(2.0).view(np.uint32)], [3, 3, 3, 0],
                         [5, 27, 27, 1], [49, 49, 49, np.float32(1.0).view(np.uint32)], [3, 3, 3, 0]], np.uint32)
    out = words.copy()
    O.lib().orc_measure_edits(O.ptr(state), O.ptr(meta), O.ptr(index), O.ptr(light), O.ptr(measures), 2, O.ptr(out))
    lum = lambda v: (np.float32(0.2126) * np.float32(v) + np.float32(0.7152) * np.float32(v)) + np.float32(0.0722) * np.float32(v)
    brightest = np.float32(0.5) * (lum(1.0) + lum(0.5)) + np.float32(0.25)
    assert out[15] == (np.float32(2.0) + brightest * np.float32(2.0) * np.float32(2.0)).view(np.uint32)
    assert out[19] == 3 | 8
    assert out[23] == words[23] and out[27] == 0


def encode_retention_events(events):
    """encode_events (src/gpu/resident.rs:1320-1414) for the pin cases.
    An event is ("bounds", [(min, max, flux, kind, high)]) with the union of
    its bounds, or ("source", cap, [(centre, radius)])."""
    head, records = [], []
    first = 0
    for e in events:
        if e[0] == "source":
            _, cap, spheres = e
            head += [[0, 0, 0, 2], [0, 0, 0, 0], [cap, 0, first, len(spheres)]]
            first += len(spheres)
        else:
            bounds = e[1]
            lo = np.min([b[0] for b in bounds], axis=0)
            hi = np.max([b[1] for b in bounds], axis=0)
            head += [[*lo, 0], [*hi, 0], [0, 0, first, len(bounds)]]
            first += len(bounds)
    for e in events:
        if e[0] == "source":
            for centre, radius in e[2]:
                records += [[*np.float32(centre).view(np.uint32), np.float32(radius * radius).view(np.uint32)], [0, 0, 0, 5]]
        else:
            for lo, hi, flux, kind, high in e[1]:
                records += [[*lo, int(np.float32(flux).view(np.uint32))], [*hi, kind | high]]
    words = np.array(head + records, np.int64).astype(np.uint32).reshape(-1)
    return words, len(events)


def point(p):
    return (np.array(p), np.array(p))


def test_measured_change_follows_flux_height_and_falls_back_when_unknown():
    # retention.rs:275-319, against the oracle's resolve_retention
    # (voxel_retention.wgsl:29-96) with the influence radius 192 as reach.
    def change_at(p, kind, flux, high, receiver):
        events = encode_retention_events([("bounds", [(*point(p), flux, kind, high)])])
        return O.resolve_retention(events, receiver)[1]

    edit = change_at((0, 0, 0), 3, 10.0, 0, (10, 0, 0))
    assert abs(edit - 10.0 / (math.pi * 100.0)) < 1e-6
    # A load whose top solid voxel (5) is below the receiver replaces no sky it saw.
    load_high = 5 << 3
    assert change_at((0, 5, 0), 2, 2.0, load_high, (4, 12, 0)) == 0.0
    below = change_at((0, 5, 0), 2, 2.0, load_high, (4, 0, 0))
    assert abs(below - 2.0 * 6.0 / (math.pi * (16 + 25))) < 1e-6
    # An air-only load (top i32::MIN, saturated to 28 bits).
    air_high = ((-(1 << 27)) & 0xFFFFFFFF) << 3 & 0xFFFFFFFF
    assert change_at((0, 0, 0), 2, 2.0, air_high, (1, 1, 1)) == 0.0
    # Unloads predict nothing; unknown flux falls back to the curve.
    assert change_at((0, 0, 0), 1, 0.0, 0, (1, 1, 1)) == 0.0
    unknown = encode_retention_events([("bounds", [(*point((0, 0, 0)), 0.0, 0, 0)])])
    limit, change, _ = O.resolve_retention(unknown, (64, 0, 0))
    assert (limit, change) == (809, None)


def test_events_reach_and_sources_cap_everywhere():
    # retention.rs:321-343: an unknown change at 64 caps the origin at H(64);
    # a source change caps every face at its cap, 4 inside its spheres, and
    # wakes every face; a change beyond the influence radius does nothing.
    events = encode_retention_events([("bounds", [(*point((64, 0, 0)), 0.0, 0, 0)]),
                                      ("source", 64, [((0.0, 0.0, 300.0), 10.0)])])
    limit, _, woken = O.resolve_retention(events, (0, 0, 0))
    assert limit == 64 and woken  # min(H(64) = 809, the source cap 64)
    assert O.resolve_retention(events, (0, 0, 295))[0] == 4
    assert O.resolve_retention(events, (4000, 0, 0))[2], "source changes wake everyone"
    only_bounds = encode_retention_events([("bounds", [(*point((64, 0, 0)), 0.0, 0, 0)])])
    assert O.resolve_retention(only_bounds, (0, 0, 0))[0] == 809
    far = encode_retention_events([("bounds", [(*point((4000, 0, 0)), 0.0, 0, 0)])])
    assert O.resolve_retention(far, (0, 0, 0)) == (0xFFFFFFFF, 0.0, False)
