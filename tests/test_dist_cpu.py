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


def _stub_rank_work(args, rank, world):
    """Stands in for bench.run_ours on CPU: a rank-dependent 'step time', reduced over
    the process group exactly as run_ours reduces its CUDA-event timings."""
    import bench

    t = bench.max_over_ranks([0.010 * (rank + 1)])[0]
    return {"metric": "stub", "value": world * 1.0 / t, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "rank_frame": bench._frame("column", rank)[0][:2].tolist()}


def _bench_env():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    env.pop("RANK", None)
    env.pop("LOCAL_RANK", None)
    env["CHAIN_BENCH_RANK_FN"] = "test_dist_cpu:_stub_rank_work"
    env["PYTHONPATH"] = os.pathsep.join([str(ROOT / "tests"), str(ROOT), env.get("PYTHONPATH", "")])
    return env


def test_bench_gpus2_spawns_two_ranks():
    """bench.py --gpus 2 without torchrun starts two ranks itself (gloo here, no GPU);
    rank 0 prints one line whose n_gpus is 2 and whose time is the slower rank's."""
    import json
    import subprocess

    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--steps", "3", "--warmup", "3"],
                       env=_bench_env(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["n_gpus"] == 2
    assert abs(line["ms_per_step"] - 20.0) < 1e-9      # max over ranks of 10 and 20 ms
    assert abs(line["value"] - 2 / 0.020) < 1e-6


def test_bench_rejects_gpus_world_size_mismatch():
    import subprocess

    env = _bench_env()
    env.update(WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--steps", "3"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "WORLD_SIZE" in r.stderr
