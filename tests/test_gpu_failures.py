"""Failure semantics of the GPU path, with every failure made on the host or
by a wait limit, never by faulting the device:

- a device allocation or a host-to-device copy that fails
  (vgi_inject_failure) makes the call return VGI_ERR_CUDA with the reason in
  vgi_last_error. The context stays usable: a failed vgi_set_faces leaves no
  faces and a failed upload no geometry, so frames are refused with
  VGI_ERR_STATE instead of reading released buffers, and after the next
  successful setters the frames equal the oracle's word for word;
- a context whose set-up meets a failed allocation is not created: the call
  returns VGI_UNAVAILABLE, as for a device that cannot run the path (the
  reference idles after a failed pipeline build, src/tests.rs:38-80);
- a tensor-core wait of the MLP kernels that runs out (wait limit 0) gives
  VGI_ERR_CUDA; with the default limit the next calls return exactly what
  they returned before, so the kernels that gave up freed their TMEM and
  left nothing in flight.
"""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_parity import assert_words_equal, lanes_for, stone_room_case

pytestmark = pytest.mark.gpu


def oracle_frames(g, case, frames, samples):
    geometry = g.geometry()
    ref = O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                   case.pipe(lanes_for(case.transport, samples)))
    for f in range(frames):
        g.frame(samples, clock_ms=16 * f)
        ref.frame(samples, clock_ms=16 * f)
    assert_words_equal(g.read_results(), ref.results, "frame results")
    assert_words_equal(g.read_state(), ref.state, "resident state")


def test_failed_face_allocation_leaves_no_faces_then_recovers():
    case = stone_room_case()
    with vgi.GpuTracer(0) as g:
        case.load(g, with_faces=False)
        vgi.inject_failure(vgi.INJECT_ALLOC, 1)
        with pytest.raises(vgi.VgiError) as err:
            g.set_faces(case.faces)
        assert err.value.status == vgi.ERR_CUDA and "memory" in str(err.value)
        with pytest.raises(vgi.VgiError) as err:
            g.frame(4, clock_ms=0)
        assert err.value.status == vgi.ERR_STATE
        g.set_faces(case.faces)
        oracle_frames(g, case, 3, 4)


def test_failed_upload_leaves_no_geometry_then_recovers():
    case = stone_room_case()
    with vgi.GpuTracer(0) as g:
        case.load(g)
        g.frame(4, clock_ms=0)
        vgi.inject_failure(vgi.INJECT_UPLOAD, 1)
        with pytest.raises(vgi.VgiError) as err:
            g.upload_regions(case.coords, case.vox)
        assert err.value.status == vgi.ERR_CUDA
        with pytest.raises(vgi.VgiError) as err:
            g.frame(4, clock_ms=16)
        assert err.value.status == vgi.ERR_STATE and "geometry" in str(err.value)
        case.load(g)
        oracle_frames(g, case, 3, 4)


def test_refused_upload_keeps_the_previous_geometry():
    case = stone_room_case()
    with vgi.GpuTracer(0) as g:
        case.load(g)
        bad = case.vox.copy()
        bad[17] = 300
        with pytest.raises(vgi.VgiError) as err:
            g.upload_regions(case.coords, bad)
        assert err.value.status == vgi.ERR_INVALID
        # Refused before any device work: the context keeps its scene.
        oracle_frames(g, case, 2, 4)


def test_context_setup_failure_idles_like_a_missing_device():
    vgi.inject_failure(vgi.INJECT_ALLOC, 1)
    try:
        with pytest.raises(vgi.TransportUnavailable):
            vgi.GpuTracer(0)
    finally:
        vgi.inject_failure(vgi.INJECT_ALLOC, 0)
    with vgi.GpuTracer(0) as g:
        g.upload_regions(*vgi.stone_room())


def random_weights(seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.normal(0.0, 1.0 / np.sqrt(i), size=(i, o)).astype(np.float32).reshape(-1)
                           for i, o in vgi.GpuTracer.MLP_LAYERS])


def test_mlp_waits_that_run_out_report_and_leave_the_context_working(gpu):
    rng = np.random.default_rng(5)
    n = 4099
    features = np.zeros((n, 96), np.float32)
    features[:, :81] = rng.uniform(-1.0, 1.0, size=(n, 81))
    targets = rng.uniform(0.1, 2.0, size=(n, 3)).astype(np.float32)
    gpu.mlp_set_weights(random_weights(9))
    out0 = gpu.mlp_forward(features)
    grads0, loss0 = gpu.mlp_gradients(features, targets)
    try:
        gpu.mlp_set_wait_limit(0)
        for call in (lambda: gpu.mlp_forward(features), lambda: gpu.mlp_gradients(features, targets)):
            with pytest.raises(vgi.VgiError) as err:
                call()
            assert err.value.status == vgi.ERR_CUDA and "ran out" in str(err.value)
    finally:
        gpu.mlp_set_wait_limit(None)
    out1 = gpu.mlp_forward(features)
    grads1, loss1 = gpu.mlp_gradients(features, targets)
    assert (out1.view(np.uint32) == out0.view(np.uint32)).all()
    assert (grads1.view(np.uint32) == grads0.view(np.uint32)).all() and loss1 == loss0
