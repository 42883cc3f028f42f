"""Face-sharded frames across torch.distributed ranks.

Faces are independent given the frame's geometry and the world cache's
snapshot. Every rank's tracer therefore holds the whole scene and every face
(the face index and a gather record per slot) but traces, prepares and
accumulates only its own contiguous slot range. After each frame one
all-gather gives every rank the other ranks' new gather records, so the next
frame gathers from the snapshot a single GPU would have, and every slot's
results and state are those of an unsharded frame.

The tracer is anything with

    frame_shard(samples, clock_ms, first, n)
    read_cache(first, n) -> (n, W) array      write_cache(first, n, array)

and, for device exchange (NCCL), ``read_cache_device(first, n, ptr)``,
``write_cache_device(first, n, ptr)`` and ``stream``: GpuTracer provides
all of them with W = 4 (mean rgb, count word). With the NCCL backend the
records go through CUDA tensors on the tracer's stream; with gloo through
host arrays.
"""
from __future__ import annotations

import numpy as np


def shard_range(n_faces: int, world: int, rank: int):
    """(first, count, padded size) of a rank's slots: equal contiguous ranges
    of ceil(n / world), the last one shorter."""
    size = (n_faces + world - 1) // world
    first = min(n_faces, rank * size)
    count = min(n_faces, first + size) - first
    return first, count, size


class FaceShards:
    def __init__(self, tracer, n_faces: int, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.tracer = tracer
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.n_faces = n_faces
        self.ranges = [shard_range(n_faces, self.world, r) for r in range(self.world)]
        self.first, self.count, self.size = self.ranges[self.rank]
        self.on_device = dist.get_backend(group) == "nccl"

    def frame(self, samples: int, clock_ms: int = 0) -> None:
        """One frame of this rank's slots, then the record exchange (every
        rank calls it, in the same order)."""
        if self.count:
            self.tracer.frame_shard(samples, clock_ms, self.first, self.count)
        self.exchange()

    def exchange(self) -> None:
        if self.on_device:
            self._exchange_device()
        else:
            self._exchange_host()

    def _exchange_host(self) -> None:
        import torch

        mine = self.tracer.read_cache(self.first, self.count) if self.count else None
        width = mine.shape[1] if mine is not None else self._width()
        dtype = mine.dtype if mine is not None else np.uint32
        padded = np.zeros((self.size, width), dtype)
        if self.count:
            padded[: self.count] = mine
        # int32 views: the records are raw words.
        send = torch.from_numpy(padded.view(np.int32))
        parts = [torch.empty_like(send) for _ in range(self.world)]
        self.dist.all_gather(parts, send, group=self.group)
        for r, (first, count, _) in enumerate(self.ranges):
            if r != self.rank and count:
                self.tracer.write_cache(first, count, parts[r].numpy()[:count].view(dtype))

    def _width(self) -> int:
        return getattr(self.tracer, "record_words", 4)

    def _exchange_device(self) -> None:
        import torch

        device = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.ExternalStream(self.tracer.stream, device=device)
        with torch.cuda.stream(stream):
            send = torch.zeros((self.size, 4), dtype=torch.int32, device=device)
            if self.count:
                self.tracer.read_cache_device(self.first, self.count, send.data_ptr())
            full = torch.empty((self.world * self.size, 4), dtype=torch.int32, device=device)
            self.dist.all_gather_into_tensor(full, send, group=self.group)
            for r, (first, count, size) in enumerate(self.ranges):
                if r != self.rank and count:
                    self.tracer.write_cache_device(first, count, full[r * size].data_ptr())
            # The tensors are released only after the copies have read them.
            stream.synchronize()
