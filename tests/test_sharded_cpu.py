"""virtualct_b200.sharded on CPU with the gloo backend, world size 2: the
collectives (the (max, -min) all-reduce, the all-gather of uneven row
pieces, the sum of disjoint image bands) put together exactly what one rank
computes alone.  The per-rank device calls are played by a stand-in context
whose rows, statistics, normalisation and bands are simple functions of
their inputs (the kernels themselves are checked on the GPU in
tests/test_gpu_sharded.py)."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest


class FakeCtx:
    """The five Context calls ShardedSlice makes, on CPU tensors."""

    def __init__(self, views=9, width=5, bands=7):
        self.geometry = SimpleNamespace(views=views, width=width)
        self.bands = bands

    def set_stream(self, s):
        pass

    def forward_views_dev(self, v0, v1, out, maxmin):
        import torch

        rows = torch.arange(v0, v1, dtype=torch.float32)[:, None]
        cols = torch.arange(self.geometry.width, dtype=torch.float32)[None]
        out[v0:v1] = 1.0 + torch.sin(rows * 0.7 + cols * 1.3) ** 2 * (rows + 1)
        maxmin[0] = out[v0:v1].max() if v1 > v0 else 0.0
        maxmin[1] = out[v0:v1].min() if v1 > v0 else 3.0e38

    def normalize_noise_rows_dev(self, sino, r0, r1, maxmin, sigma, seed):
        sino[r0:r1] = sino[r0:r1] / maxmin[0] + 1e-3 * maxmin[1] + sigma * seed

    def fbp_band_count(self):
        return self.bands

    def fbp_band_dev(self, sino, b0, b1, img, filter=1, in_mode=False):
        for b in range(b0, b1):
            img[b] = sino.sum() * (b + 1) + sino[b % sino.shape[0]].sum() * filter


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from virtualct_b200.sharded import ShardedSlice

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ctx = FakeCtx()
        sh = ShardedSlice(ctx, dist)
        sino = torch.full((9, 5), -7.0)
        sh.mbfpa(0.5, 3, sino)
        img = torch.full((7, 4), -7.0)
        sh.fbp(sino, img, filter=2)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.concatenate([sino.numpy().ravel(), img.numpy().ravel()]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one(tmp_path):
    import torch
    import torch.multiprocessing as mp

    from virtualct_b200.sharded import ShardedSlice

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    one = ShardedSlice(FakeCtx())
    sino = torch.zeros((9, 5))
    one.mbfpa(0.5, 3, sino)
    img = torch.zeros((7, 4))
    one.fbp(sino, img, filter=2)
    ref = np.concatenate([sino.numpy().ravel(), img.numpy().ravel()])
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"r{r}.npy"), ref)


@pytest.mark.parametrize("n,parts", [(9, 2), (800, 8), (3, 5), (0, 2)])
def test_split_covers_once(n, parts):
    from virtualct_b200.sharded import split

    pieces = [split(n, parts, i) for i in range(parts)]
    assert pieces[0][0] == 0 and pieces[-1][1] == n
    assert all(a[1] == b[0] for a, b in zip(pieces, pieces[1:]))
    assert max(b - a for a, b in pieces) - min(b - a for a, b in pieces) <= 1
