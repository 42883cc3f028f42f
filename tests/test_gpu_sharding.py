"""Face-sharded frames on the GPU: vgi_frame_shard over slot ranges plus the
exchange of gather records equals whole frames, word for word. Two contexts
on one GPU stand for two ranks (they exchange through the host, so no
kernel waits on another), and a one-rank NCCL group runs the device-side
exchange of vgi.sharding."""
import datetime
import os
import socket

import numpy as np
import pytest

import vgi
from test_gpu_parity import assert_words_equal, terrain_case
from vgi.sharding import shard_range

pytestmark = pytest.mark.gpu

FRAMES, SAMPLES = 5, 8


def whole_frames(gpu, case):
    case.load(gpu)
    for f in range(FRAMES):
        gpu.frame(SAMPLES, clock_ms=16 * f)
    n = case.faces.shape[0]
    return gpu.read_results(), gpu.read_state(), gpu.read_cache(0, n)


def test_two_context_shards_equal_whole_frames(gpu):
    case = terrain_case(bounces=2)
    results, state, cache = whole_frames(gpu, case)
    n = case.faces.shape[0]
    ranks = [vgi.GpuTracer(0) for _ in range(2)]
    try:
        for t in ranks:
            case.load(t)
        ranges = [shard_range(n, 2, r) for r in range(2)]
        hits = 0
        for f in range(FRAMES):
            for t, (first, count, _) in zip(ranks, ranges):
                t.frame_shard(SAMPLES, 16 * f, first, count)
            records = [t.read_cache(first, count) for t, (first, count, _) in zip(ranks, ranges)]
            for r, t in enumerate(ranks):
                other = 1 - r
                t.write_cache(ranges[other][0], ranges[other][1], records[other])
        for t, (first, count, _) in zip(ranks, ranges):
            assert_words_equal(t.read_results()[first:first + count], results[first:first + count], "shard results")
            assert_words_equal(t.read_state()[first:first + count], state[first:first + count], "shard state")
            assert_words_equal(t.read_cache(0, n), cache, "gather records after the exchange")
    finally:
        for t in ranks:
            t.close()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_exchange_of_a_one_rank_group(gpu):
    import torch
    import torch.distributed as dist

    from vgi.sharding import FaceShards

    case = terrain_case(bounces=2)
    results, state, cache = whole_frames(gpu, case)
    case.load(gpu)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shards = FaceShards(gpu, case.faces.shape[0])
        assert shards.on_device and shards.count == case.faces.shape[0]
        for f in range(FRAMES):
            shards.frame(SAMPLES, 16 * f)
        assert_words_equal(gpu.read_results(), results, "one-rank shard results")
        assert_words_equal(gpu.read_state(), state, "one-rank shard state")
    finally:
        dist.destroy_process_group()


def test_mlp_data_parallel_step_of_a_one_rank_group(gpu):
    """MlpDataParallel through NCCL (device gradient, all-reduce on the
    tracer's stream): a one-rank group's step is mlp_train's step, within the
    gradient sums' atomic noise."""
    import torch
    import torch.distributed as dist

    from test_gpu_mlp import batch, random_weights
    from vgi.sharding import MlpDataParallel

    master = random_weights(5)
    features, targets = batch(3000, 8)
    gpu.mlp_set_weights(master)
    gpu.mlp_train(features, targets, 1e-2)
    want = gpu.mlp_get_weights()
    gpu.mlp_set_weights(master)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dp = MlpDataParallel(gpu)
        assert dp.on_device
        loss = dp.step(features, targets, lr=1e-2)
        assert np.isfinite(loss) and loss > 0.0
        diff = np.abs(gpu.mlp_get_weights() - want)
        assert np.mean(diff < 1e-4) > 0.999, diff.max()
    finally:
        dist.destroy_process_group()
