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
        if getattr(self, "_send", None) is None:
            # Kept for the life of the shards, so no frame waits on the host
            # for the copies out of them: every use is ordered on the
            # tracer's stream (the collective waits for it and it waits for
            # the collective).
            self._send = torch.zeros((self.size, 4), dtype=torch.int32, device=device)
            self._full = torch.empty((self.world * self.size, 4), dtype=torch.int32, device=device)
        with torch.cuda.stream(stream):
            if self.count:
                self.tracer.read_cache_device(self.first, self.count, self._send.data_ptr())
            self.dist.all_gather_into_tensor(self._full, self._send, group=self.group)
            for r, (first, count, size) in enumerate(self.ranges):
                if r != self.rank and count:
                    self.tracer.write_cache_device(first, count, self._full[r * size].data_ptr())


class MlpDataParallel:
    """Data-parallel training of the MLP radiance cache: every rank computes
    the gradient of the loss over its own rows (``mlp_gradients``), one
    all-reduce averages the 19,456 gradients and the losses, and every rank
    takes the same Adam step from the average (``mlp_apply_gradients``), so
    the ranks' weights stay identical. With the NCCL backend the gradient
    goes through a CUDA tensor; with gloo through a host tensor. Every rank
    calls ``step`` in the same order with equally many rows."""

    def __init__(self, tracer, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.tracer = tracer
        self.group = group
        self.world = dist.get_world_size(group)
        self.on_device = dist.get_backend(group) == "nccl"

    def step(self, features, targets, lr: float = 1e-2) -> float:
        """One data-parallel Adam step over this rank's rows; returns the mean
        loss over all ranks' rows (before the step)."""
        import torch

        grads, loss = self.tracer.mlp_gradients(features, targets)
        buf = torch.from_numpy(np.concatenate([np.asarray(grads, np.float32).reshape(-1), np.float32([loss])]))
        if not self.on_device:
            self.dist.all_reduce(buf, group=self.group)
            buf /= self.world
            mean_loss = float(buf[-1])
            self.tracer.mlp_apply_gradients(buf[:-1].numpy(), mean_loss, lr)
            return mean_loss
        # On the tracer's stream, so the step reads the reduced gradient.
        device = torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.stream(torch.cuda.ExternalStream(self.tracer.stream, device=device)):
            buf = buf.to(device)
            self.dist.all_reduce(buf, group=self.group)
            buf /= self.world
            mean_loss = float(buf[-1])
            self.tracer.mlp_apply_gradients(buf[:-1], mean_loss, lr)
        return mean_loss
