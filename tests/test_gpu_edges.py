"""Edge cases of the boundary: ragged and tiny face sets, scenes without
emitters, the extreme sample counts, empty inputs, and the inputs the entry
points must refuse with an error rather than trace."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal, lanes_for, stone_room_case, terrain_case, trace_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("count", [1, 31, 33, 257])
def test_ragged_face_counts_match_oracle(gpu, count):
    case = terrain_case(bounces=2)
    case.faces = case.faces[:count].copy()
    got, want, gcnt, wcnt = trace_pair(gpu, case, 8, lanes_for(case.transport, 8), sequence=99)
    assert_words_equal(got, want, f"{count} faces")
    assert gcnt == wcnt


def test_scene_without_emitters_matches_oracle(gpu):
    case = terrain_case(bounces=2, emitters=0)
    assert case.n_emit == 0
    got, want, gcnt, wcnt = trace_pair(gpu, case, 8, lanes_for(case.transport, 8), sequence=3)
    assert_words_equal(got, want, "no emitters")
    assert gcnt == wcnt


@pytest.mark.parametrize("samples", [1, 32])
def test_extreme_sample_counts_match_oracle(gpu, samples):
    case = stone_room_case()
    got, want, gcnt, wcnt = trace_pair(gpu, case, samples, lanes_for(case.transport, samples), sequence=5)
    assert_words_equal(got, want, f"{samples} samples")
    assert gcnt == wcnt


def test_empty_inputs_do_nothing(gpu):
    case = terrain_case(bounces=2)
    case.load(gpu)
    assert gpu.trace_tasks(np.zeros((0, 8), np.uint32), 8).shape == (0, 24)
    gpu.edit_voxels(np.zeros((0, 4), np.int32))
    assert gpu.read_cache(0, 0).shape == (0, 4)
    gpu.mlp_set_weights(np.zeros(vgi.GpuTracer.MLP_WEIGHTS, np.float32))
    assert gpu.mlp_forward(np.zeros((0, 96), np.float32)).shape == (0, 3)


def test_invalid_inputs_are_refused(gpu):
    case = terrain_case(bounces=2)
    case.load(gpu)
    n = case.faces.shape[0]
    bad_face = case.faces[:4].copy()
    bad_face[0, 3] = 6
    with pytest.raises(vgi.VgiError):
        gpu.set_faces(bad_face)
    bad_material = case.faces[:4].copy()
    bad_material[0, 4] = 256
    with pytest.raises(vgi.VgiError):
        gpu.set_faces(bad_material)
    case.load(gpu)
    with pytest.raises(vgi.VgiError, match="samples"):
        gpu.frame(0)
    with pytest.raises(vgi.VgiError, match="samples"):
        gpu.trace_tasks(vgi.tasks_for(case.faces[:8]), 0)
    with pytest.raises(vgi.VgiError, match="one task per slot"):
        gpu.trace_batch(vgi.tasks_for(case.faces[:8]), 8)
    with pytest.raises(vgi.VgiError, match="shard"):
        gpu.frame_shard(8, 0, n - 4, 8)
    with pytest.raises(vgi.VgiError):
        gpu.frame_shard(8, 0, 0, 0)
    with pytest.raises(vgi.VgiError):
        gpu.read_cache(n - 1, 2)
    with pytest.raises(vgi.VgiError, match="19456"):
        gpu.mlp_set_weights(np.zeros(100, np.float32))
    fresh = vgi.GpuTracer(0)
    try:
        with pytest.raises(vgi.VgiError, match="not set"):
            fresh.set_mlp_cache(True)
        with pytest.raises(vgi.VgiError, match="geometry"):
            fresh.frame(8)
    finally:
        fresh.close()
    with pytest.raises(vgi.VgiError):
        vgi.GpuBatch([])
    # Nothing above changed the context: a frame still matches the oracle.
    case.load(gpu)
    geometry = gpu.geometry()
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                   case.pipe(lanes_for(case.transport, 8)))
    gpu.frame(8)
    ref.frame(8)
    assert_words_equal(gpu.read_results(), ref.results, "frame after refused calls")


def test_repeated_voxel_edits_keep_the_last_value(gpu):
    """Edits apply in order (VoxelGiInput::edit_voxel): a voxel edited twice
    in one list keeps its last value, as the oracle's in-order edits do."""
    case = terrain_case()
    case.load(gpu, with_faces=False)
    ref = O.Scene(case.coords, case.vox, top_mode=0)
    rng = np.random.default_rng(8)
    block = [(x, y, z) for x in range(30, 38) for y in range(20, 36) for z in range(40, 48)]
    edits = [(x, y, z, 256) for x, y, z in block] + [(x, y, z, int(rng.integers(0, 8))) for x, y, z in block]
    edits += [(x, y, z, 256) for x, y, z in block[::3]]
    # Shuffled, so a voxel's edits are far apart in the list; both sides apply the list in order.
    edits = np.array(edits, np.int32)[rng.permutation(len(edits))]
    gpu.edit_voxels(edits)
    ref.edit(edits)
    d, h, cl, _ = gpu.geometry()
    rd, rh, rcl, _ = ref.arrays()
    assert_words_equal(O.canonical(d, h, cl, case.coords), O.canonical(rd, rh, rcl, case.coords), "geometry after repeated edits")
