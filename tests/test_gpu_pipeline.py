"""Pipelined batches (vgi_submit_batch / vgi_complete_batch): the same
frames as vgi_trace_batch, with the host copies on their own streams and two
batches in flight, give the same results word for word."""
import numpy as np
import pytest
import torch

import vgi
from test_gpu_parity import assert_words_equal, terrain_case

pytestmark = pytest.mark.gpu


def pinned(shape):
    return torch.empty(shape, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)


@pytest.mark.parametrize("graph", [False, True])
def test_pipelined_batches_equal_synchronous_batches(gpu, graph):
    case = terrain_case(bounces=2)
    n = case.faces.shape[0]
    frames = 6
    case.load(gpu)
    tasks = vgi.tasks_for(case.faces)
    want = [gpu.trace_batch(tasks, 8, clock_ms=16 * f).copy() for f in range(frames)]
    case.load(gpu)
    gpu.set_graph(graph)
    try:
        host_tasks = pinned((n, 8))
        host_tasks[:] = tasks
        outs = [pinned((n, 24)) for _ in range(frames)]
        tickets = []
        for f in range(frames):
            tickets.append(gpu.submit_batch(host_tasks, 8, 16 * f, outs[f]))
            if f >= 1:
                gpu.complete_batch(tickets[f - 1])
        gpu.complete_batch(tickets[-1])
        for f in range(frames):
            assert_words_equal(outs[f], want[f], f"pipelined batch {f}")
        with pytest.raises(vgi.VgiError):
            gpu.complete_batch(tickets[-1] + 1)
    finally:
        gpu.set_graph(False)
