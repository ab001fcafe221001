"""The multi-rank path of bench.py on CPU (gloo, world size 2).

`bench.py --gpus N` runs one replica per GPU: every rank compresses its own frame
(weak scaling, no data-path collective) and the job's time is the maximum over ranks.
Here two gloo ranks check that reduction, and that the ranks' frames differ.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.distributed as tdist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    got = bench.max_over_ranks([1.0 + rank, 5.0 - rank, 0.5 * rank])
    out[rank] = got
    tdist.barrier()
    tdist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        for r in range(world):
            assert out[r] == [2.0, 5.0, 0.5]


def test_ranks_compress_different_frames():
    sys.path.insert(0, str(ROOT))
    import bench

    a = bench._frame("column", 0)
    b = bench._frame("column", 1)
    assert a[0].shape == b[0].shape and a[2:4] == b[2:4]
    assert not np.array_equal(a[0], b[0])
