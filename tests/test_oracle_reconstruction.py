"""The presentation's virtual-corner reconstruction (orc_corner_value) and
the view reconstruction (orc_reconstruct) on the CPU. The corner tests
restate the reference's CPU oracle for it (src/reconstruction.rs:58-173):
constants are preserved, coplanar neighbours agree at shared corners with
any confidences, and a diagonal face across two missing edges adds
nothing."""
import itertools

import numpy as np

import oracle_lib as O
from test_oracle_far import Scene


def wc(center, u=None, v=None, diagonal=None):
    return float(O.corner_value(center, u, v, diagonal)[0])


def corner(center, u=None, v=None, diagonal=None):
    one = lambda x: None if x is None else (x, 1.0)
    return wc((center, 1.0), one(u), one(v), one(diagonal))


def test_confidence_weighting_preserves_constants_and_reduces_unmeasured_neighbours():
    assert wc((2.5, 0.03125), (2.5, 0.125)) == 2.5
    assert wc((2.5, 0.03125)) == 2.5
    a = wc((0.0, 0.03125), (8.0, 1.0))
    b = wc((8.0, 1.0), (0.0, 0.03125))
    assert a == b, "shared corners agree even with different confidence"
    assert a > 7.7, "an unmeasured face should not halve measured lighting"
    assert wc((0.0, 0.125), None, None, (100.0, 1.0)) == 0.0


def test_coplanar_neighbours_agree_at_shared_corners():
    values = [1.0, 3.0, 5.0, 7.0]
    weights = [0.03125, 0.125, 0.5, 1.0]
    for mask in range(16):
        value = lambda i: values[i] if mask & (1 << i) else None
        weighted = lambda i: (values[i], weights[i]) if mask & (1 << i) else None
        for a in range(4):
            if not mask & (1 << a):
                continue
            ca = corner(values[a], value(a ^ 1), value(a ^ 2), value(a ^ 3))
            wa = wc(weighted(a), weighted(a ^ 1), weighted(a ^ 2), weighted(a ^ 3))
            for b in (a ^ 1, a ^ 2):
                if mask & (1 << b):
                    assert corner(values[b], value(b ^ 1), value(b ^ 2), value(b ^ 3)) == ca, mask
                    wb = wc(weighted(b), weighted(b ^ 1), weighted(b ^ 2), weighted(b ^ 3))
                    assert abs(wa - wb) < 1e-6, mask


def test_diagonal_light_does_not_cross_occluded_edges():
    assert corner(0.0, None, None, 100.0) == 0.0


def test_constant_field_is_preserved_at_missing_boundaries():
    for mask in range(8):
        value = lambda bit: 2.5 if mask & bit else None
        assert corner(2.5, value(1), value(2), value(4)) == 2.5


def floor_receivers(n_side=8):
    """Unit +y faces of the floor (y = 0) on an n_side x n_side patch, one
    receiver each, tiles of 2 x 2 faces."""
    rows, tiles = [], []
    for z, x in itertools.product(range(n_side), range(n_side)):
        surface = np.float32([x + 0.5, 1.0, z + 0.5])
        rows.append([*surface.view(np.uint32), 2, x, 0, z, 0])
        tiles.append((z // 2) * (n_side // 2) + x // 2)
    return np.array(rows, np.uint32), np.array(tiles, np.uint32)


def estimates_for(means, counts, moments=None, shown=None):
    e = np.zeros((len(means), 16), np.uint32)
    f = e.view(np.float32)
    f[:, 0:3] = np.asarray(means, np.float32).reshape(-1, 3)
    f[:, 3] = counts
    f[:, 4:7] = (np.asarray(means, np.float32) ** 2).reshape(-1, 3) if moments is None else moments
    if shown is not None:
        f[:, 8:11], f[:, 11] = shown, 1.0
    return e


def run(scene, receivers, estimates, tiles, display=(0.031, 1.0, 1.0)):
    pipe = O.Pipeline(1, 0, 2048, 0, 1)
    conts = np.zeros((len(receivers), 32), np.uint32)
    return O.reconstruct(scene.geometry, scene.params, scene.materials, scene.lights, scene.emitters, pipe, receivers, estimates, conts,
                         tiles, 4, 4, display)


def test_reconstruction_keeps_a_converged_constant_field_and_fills_unsampled_faces():
    scene = Scene(slab=False)
    receivers, tiles = floor_receivers()
    means = np.tile(np.float32([0.4, 0.5, 0.6]), (64, 1))
    counts = np.full(64, 512.0, np.float32)
    counts[27] = 0.0  # one face never sampled
    est, published, stats = run(scene, receivers, estimates_for(means, counts), tiles)
    shown = est.view(np.float32)[:, 8:12]
    assert np.all(shown[:, 3] == 1.0)
    # A sampled face with zero variance keeps its mean; the unsampled one takes its neighbours'.
    np.testing.assert_allclose(shown[:, :3], means, rtol=1e-6)
    assert stats[2] == 1 and stats[3] == 64 and stats[0] == 63 * 512 and stats[1] == 512
    p = published.view(np.float32)
    np.testing.assert_allclose(p[:, 4:7], means, rtol=1e-6)
    assert np.all(published[:, 3] == 2)


def test_noisy_faces_borrow_from_coplanar_neighbours_only_within_the_bias_bound():
    scene = Scene(slab=False)
    receivers, tiles = floor_receivers()
    rng = np.random.default_rng(3)
    truth = np.float32(0.5)
    counts = np.full(64, 4.0, np.float32)
    means = truth + rng.normal(0, 0.15, (64, 3)).astype(np.float32)
    moments = means ** 2 + np.float32(0.05)
    est, _, _ = run(scene, receivers, estimates_for(means, counts, moments), tiles)
    shown = est.view(np.float32)[:, 8:11]
    # Pooling neighbours brings the faces closer to the truth than their own means.
    assert np.abs(shown - truth).mean() < 0.6 * np.abs(means - truth).mean()
    # Without spatial strength each face shows its own mean.
    est, _, _ = run(scene, receivers, estimates_for(means, counts, moments), tiles, display=(0.031, 0.0, 1.0))
    np.testing.assert_allclose(est.view(np.float32)[:, 8:11], means, rtol=1e-6)
