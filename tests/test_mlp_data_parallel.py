"""Data-parallel MLP training (vgi.sharding.MlpDataParallel) on two gloo
ranks over CPU. Each rank's tracer is a stand-in with the GpuTracer's
training surface (mlp_gradients, mlp_apply_gradients) over a small linear
model with the Adam step of the library's adam_kernel restated in numpy.
Every rank takes its own half of each batch; after the steps both ranks hold
the same weights, and those equal one process training on whole batches
(the gradient of a mean over the whole batch is the mean of the halves')."""
import datetime
import os
import socket

import numpy as np
import torch.multiprocessing as mp

STEPS, ROWS, DIM = 6, 64, 16


class LinearStandIn:
    """mlp_gradients / mlp_apply_gradients over y = x W (mean squared error),
    Adam with beta 0.9 / 0.99, eps 1e-8 and bias correction, as adam_kernel."""

    MLP_WEIGHTS = DIM * 3

    def __init__(self):
        self.w = np.random.default_rng(1).normal(size=(DIM, 3)).astype(np.float64)
        self.m = np.zeros_like(self.w)
        self.v = np.zeros_like(self.w)
        self.steps = 0

    def mlp_gradients(self, x, y):
        d = x @ self.w - y
        return (2.0 * x.T @ d / x.shape[0]).reshape(-1), float(np.mean(np.sum(d * d, axis=1)))

    def mlp_apply_gradients(self, grads, loss, lr):
        g = np.asarray(grads, np.float64).reshape(DIM, 3)
        self.steps += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.99 * self.v + 0.01 * g * g
        mh = self.m / (1.0 - 0.9 ** self.steps)
        vh = self.v / (1.0 - 0.99 ** self.steps)
        self.w = self.w - lr * mh / (np.sqrt(vh) + 1e-8)


def batches():
    rng = np.random.default_rng(5)
    truth = rng.normal(size=(DIM, 3))
    for _ in range(STEPS):
        x = rng.normal(size=(ROWS, DIM))
        yield x, x @ truth


def _worker(rank, world, port, queue):
    import torch.distributed as dist

    from vgi.sharding import MlpDataParallel

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        tracer = LinearStandIn()
        dp = MlpDataParallel(tracer)
        losses = []
        half = ROWS // world
        for x, y in batches():
            losses.append(dp.step(x[rank * half:(rank + 1) * half], y[rank * half:(rank + 1) * half], lr=0.05))
        queue.put((rank, tracer.w.copy(), losses))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_data_parallel_steps_keep_ranks_identical_and_match_whole_batches():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r, (w, l)) for r, w, l in (queue.get(timeout=180) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # The all-reduce is in float32: both ranks apply the same bytes.
    assert np.array_equal(got[0][0], got[1][0])
    single = LinearStandIn()
    for x, y in batches():
        g, _ = single.mlp_gradients(x, y)
        single.mlp_apply_gradients(g, 0.0, 0.05)
    assert np.allclose(got[0][0], single.w, rtol=1e-4, atol=1e-5)
    assert got[0][1][-1] < got[0][1][0]
