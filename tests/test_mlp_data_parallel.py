"""Data-parallel training of the surrogate (akantu_b200.surrogate.
data_parallel_train) on CPU: a least-squares model stands in for the
network (same three calls: compute_gradients, gradient_tensor,
apply_gradients), trained by one process on whole minibatches and by two
and four gloo ranks on their shares; the averaged gradients give the same
parameters (to rounding of the sum order) and every rank holds the same
replica bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


class LeastSquares:
    """y = x W; loss = mean((x W - t)^2) over samples and outputs; plain
    gradient descent in apply_gradients."""

    def __init__(self, nin, nout):
        self.W = torch.zeros((nin, nout), dtype=torch.float64)
        self.g = torch.zeros(nin * nout, dtype=torch.float64)

    def compute_gradients(self, x, t):
        r = x @ self.W - t
        self.g.copy_((2.0 / r.numel()) * (x.T @ r).reshape(-1))
        return float((r * r).mean())

    def gradient_tensor(self):
        return self.g

    def apply_gradients(self, lr):
        self.W -= lr * self.g.reshape(self.W.shape)


def _data():
    rng = np.random.default_rng(3)
    x = torch.as_tensor(rng.normal(size=(512, 10)))
    t = x @ torch.as_tensor(rng.normal(size=(10, 9))) + 0.01 * torch.as_tensor(rng.normal(size=(512, 9)))
    return x, t


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    from datetime import timedelta
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from akantu_b200.surrogate import data_parallel_train
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        x, t = _data()
        m = LeastSquares(10, 9)
        losses = data_parallel_train(m, x, t, epochs=3, batch=64, lr=0.05, lr_final=0.005, seed=5)
        out[rank] = dict(W=m.W.numpy().copy(), losses=losses)
    finally:
        dist.destroy_process_group()


def _run(world):
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        return dict(out)


@pytest.mark.timeout(300)
def test_ranks_average_to_the_whole_minibatch():
    one = _run(1)[0]
    for world in (2, 4):
        res = _run(world)
        for r in range(world):
            assert np.array_equal(res[r]["W"], res[0]["W"])  # replicas stay equal
        W, W1 = res[0]["W"], one["W"]
        assert np.abs(W - W1).max() <= 1e-12 * np.abs(W1).max()
        assert np.allclose(res[0]["losses"], one["losses"], rtol=1e-12)
    assert one["losses"][-1] < one["losses"][0]
