"""The multi-rank path of bench.py on CPU with the gloo backend, world size
2 (the GPU runs use NCCL, one process per GPU, the same calls): elapsed
times are reduced to their maximum on every rank, every rank projects its
own slice (phantom seed = rank), and the reference arm runs on rank 0 only."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                           timeout=datetime.timedelta(seconds=60))
    try:
        t_max = bench.reduce_max(1.5 + rank, dist, "cpu")
        dist.barrier()
        maps, _, _ = bench.replica_inputs(rank)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([t_max, float(maps.astype(np.int64).sum())]))

        class A:
            steps, warmup = 1, 0

        if rank != 0:
            assert bench.run_reference(A(), rank) is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = np.load(tmp_path / "r0.npy"), np.load(tmp_path / "r1.npy")
    assert r0[0] == r1[0] == 2.5          # the max over ranks, on both ranks
    assert r0[1] != r1[1]                 # different slices per rank


def test_single_process_reduce_is_identity():
    import bench

    assert bench.reduce_max(3.25, None, "cpu") == 3.25
