"""Face-sharded frames (vgi.sharding) on two gloo ranks over CPU, with the
oracle as each rank's tracer: every rank traces, prepares and accumulates
its own slot range and one all-gather per frame shares the gather records,
so every slot's results and state equal an unsharded frame's."""
import datetime
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle_lib as O
from test_gpu_parity import lanes_for, terrain_case
from vgi.sharding import shard_range

FRAMES, SAMPLES = 4, 8


def make_frames():
    case = terrain_case(bounces=2)
    geometry = O.Scene(case.coords, case.vox, top_mode=0).arrays()
    return O.Frames(geometry, case.params_fn(geometry), case.materials, case.lights, case.emitters, case.faces, case.transport,
                    case.pipe(lanes_for(case.transport, SAMPLES)), threads=2)


def _worker(rank, world, port, queue):
    import torch.distributed as dist

    from vgi.sharding import FaceShards

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        frames = make_frames()
        tracer = O.OracleShardTracer(frames)
        shards = FaceShards(tracer, frames.n)
        for f in range(FRAMES):
            shards.frame(SAMPLES, 16 * f)
        first, count, _ = shards.ranges[rank]
        queue.put((rank, first, count, frames.results[first:first + count].copy(), frames.state[first:first + count].copy(),
                   tracer.cache_hits))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges_cover_the_faces_once():
    for n in (1, 7, 4699):
        for world in (1, 2, 3, 8):
            seen = np.zeros(n, np.int32)
            for r in range(world):
                first, count, size = shard_range(n, world, r)
                assert 0 <= count <= size
                seen[first:first + count] += 1
            assert (seen == 1).all()


def test_two_gloo_ranks_equal_unsharded_frames():
    whole = make_frames()
    for f in range(FRAMES):
        whole.frame(SAMPLES, 16 * f)
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = [queue.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    hits = 0
    for rank, first, count, results, state, cache_hits in got:
        assert (results == whole.results[first:first + count]).all(), rank
        assert (state == whole.state[first:first + count]).all(), rank
        hits += cache_hits
    assert hits > 0  # the later frames gathered records the other rank wrote


def test_shards_without_the_exchange_differ():
    """The exchange is what makes the shards equal: two ranks that never
    share records trace from stale snapshots."""
    whole = make_frames()
    for f in range(FRAMES):
        whole.frame(SAMPLES, 16 * f)
    ranks = [make_frames() for _ in range(2)]
    for f in range(FRAMES):
        for r, frames in enumerate(ranks):
            first, count, _ = shard_range(frames.n, 2, r)
            frames.frame_shard(SAMPLES, 16 * f, first, count)
    first, count, _ = shard_range(whole.n, 2, 0)
    assert (ranks[0].results[first:first + count] != whole.results[first:first + count]).any()
