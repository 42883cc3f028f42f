"""The oracle's MLP cache termination (CPU): an uncached hit that takes the
network's value for the hit face ends the path exactly as a cache hit with
that value does (voxel_path.wgsl:63-87 and advance_path's cached branch)."""
import numpy as np

import oracle_lib as O
import vgi


def stone_room():
    coords, vox = vgi.stone_room()
    m = vgi.VoxelGiMaterials()
    m.set(0, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5)))
    m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(8.0, 4.0, 1.5)))
    words = m.words()
    emitters, n_emit, total = vgi.host_emitters(coords, vox, words)
    faces = vgi.exposed_faces(coords, vox)
    geometry = O.Scene(coords, vox, top_mode=0).arrays()
    return geometry, words, emitters, n_emit, total, faces


def test_predicted_termination_equals_a_full_cache_of_the_same_values():
    geometry, words, emitters, n_emit, total, faces = stone_room()
    n = faces.shape[0]
    rng = np.random.default_rng(4)
    values = rng.uniform(0.1, 2.0, size=(n, 3)).astype(np.float32)
    # Every face of the closed room is a slot whose cache holds its value
    # with 16 samples (enough to be gathered).
    state = np.zeros((n, 36), np.uint32)
    state[:, 0:3] = values.view(np.uint32)
    state[:, 5] = 16
    index = O.face_index(faces[:, :4])
    tasks = vgi.tasks_for(faces, 77)
    pipe = O.Pipeline(1, 0, 64, 0, 1)
    d, _, _, bounds = geometry
    params = O.params_words(n, 4, d.size // 4, 0, bounds, 0, (0, 0, 0), total, n_emit)
    cached, c_counts = O.trace_faces(geometry, params, words, [], emitters, tasks, pipe, state=state, index=index)
    predicted, p_counts = O.trace_faces(geometry, params, words, [], emitters, tasks, pipe, predicted=(faces[:, :4], values))
    assert c_counts["cache_hits"] > 1000 and p_counts["cache_hits"] == 0
    assert (cached == predicted).all()
    # A different prediction changes the results.
    other, _ = O.trace_faces(geometry, params, words, [], emitters, tasks, pipe, predicted=(faces[:, :4], values * 2.0))
    assert (other != predicted).any()
