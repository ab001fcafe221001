"""Chain compressor benchmark (one JSON line on rank 0).

Workload (default): the large single frame -- 16,777,216 float32 particles in
[0,100]^3, 80% from 64 Gaussian blobs and 20% uniform, random order, eb = 1e-3 x range,
p = 4, threshold = 2 (seeded synthetic data; the reference names no public dataset).
A step = one compress of the frame followed by one decompress of its container.

  value  : compress throughput, GB/s of uncompressed input, device-resident input
           (HBM -> container in HBM), max over ranks
  e2e    : the same through the C ABI with pinned HOST buffers (H2D of the points
           and D2H of the container inside the timed region)
  decompress : the same two numbers for the decoder (container -> float64 points)

Multi-GPU: frames are independent, so N ranks compress N independent frames
(replicas, weak scaling, no collective on the data path).

--impl reference runs the reference CPU Chain (lcps_cpp / lcps_cpu_decompress built
from the reference sources into oracle/_ref) on a bounded sample of the same workload
with one process per host core.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "oracle"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "compress GB/s (uncompressed bytes/s) at eb=1e-3*range"
UNIT = "GB/s"


def _peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def _frame(config: str, rank: int):
    from chaincompressor_b200 import workloads as W

    if config == "blobs":
        pts = W.blobs(W.BLOBS_N, seed=1 + rank)
        return pts, W.eb_for(pts, 1e-3), 4, 2, "blobs-16M-f32"
    if config == "column":
        pts = W.column(seed=rank)
        return pts, W.eb_for(pts, 1e-3), 4, 2, "column-80703-f32"
    if config == "trajectory":
        pts = W.trajectory(0, seed=2 + rank)
        return pts, W.eb_for(pts, 1e-3), 4, 2, "trajectory-4M-f64"
    raise SystemExit(f"unknown config {config}")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        self.path = None
        try:
            import tempfile
            self.path = tempfile.mktemp(suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows)}


def run_ours(args, rank: int, world: int):
    import torch

    from chaincompressor_b200 import _native as N

    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    pts, eb, p, t, wl = _frame(args.config, rank)
    n, d = pts.shape
    esz = pts.dtype.itemsize
    soa_host = torch.from_numpy(np.ascontiguousarray(pts.T)).pin_memory()
    soa_dev = soa_host.to(f"cuda:{dev}")
    codec = N.Codec(dev)
    dist = world > 1
    if dist:
        import torch.distributed as tdist

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    dtype_code = N.CHAIN_F32 if esz == 4 else N.CHAIN_F64
    # warm-up (also sizes the arenas)
    for _ in range(args.warmup):
        codec.compress_ptr(soa_dev.data_ptr(), dtype_code, N.CHAIN_SOA, n, d, eb, p, t)
    clen = codec.compress_ptr(soa_dev.data_ptr(), dtype_code, N.CHAIN_SOA, n, d, eb, p, t)
    cont_dev = torch.empty(clen, dtype=torch.uint8, device=f"cuda:{dev}")
    codec.result_copy_to(cont_dev.data_ptr(), clen)
    cont_host = torch.empty(clen, dtype=torch.uint8).pin_memory()
    cont_host.copy_(cont_dev.cpu())
    out_dev = torch.empty((n, d), dtype=torch.float64, device=f"cuda:{dev}")
    out_host = torch.empty((n, d), dtype=torch.float64).pin_memory()
    for _ in range(args.warmup):
        codec.decompress_ptr(cont_dev.data_ptr(), clen, out_dev.data_ptr(), out_dev.numel() * 8)

    def timed(fn):
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fn()
        barrier()
        return (time.perf_counter() - t0) / args.steps

    # The library call is synchronous (it ends with a stream synchronize), so host
    # time around it brackets the device work; it is cross-checked with CUDA events
    # recorded on the library stream below.
    clocks = Clocks(dev)
    t_c = timed(lambda: codec.compress_ptr(soa_dev.data_ptr(), dtype_code, N.CHAIN_SOA, n, d, eb, p, t))
    t_d = timed(lambda: codec.decompress_ptr(cont_dev.data_ptr(), clen, out_dev.data_ptr(), out_dev.numel() * 8))

    def e2e_c():
        codec.compress_ptr(soa_host.data_ptr(), dtype_code, N.CHAIN_SOA, n, d, eb, p, t)
        codec.result_copy_to(cont_host.data_ptr(), clen)

    def e2e_d():
        codec.decompress_ptr(cont_host.data_ptr(), clen, out_host.data_ptr(), out_host.numel() * 8)

    t_ce = timed(e2e_c)
    t_de = timed(e2e_d)
    clk = clocks.stop()
    if dist:
        tt = torch.tensor([t_c, t_d, t_ce, t_de], dtype=torch.float64, device=f"cuda:{dev}")
        tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
        t_c, t_d, t_ce, t_de = tt.tolist()
    # correctness of the measured run
    dec = out_host.numpy()
    err = float(np.abs(dec - pts.astype(np.float64)).max())
    raw = n * d * esz
    gbs = lambda sec: world * raw / sec / 1e9  # noqa: E731
    peaks, src = _peaks()
    line = {
        "metric": METRIC, "value": round(gbs(t_c), 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round((t_c + t_d) * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64-quantize/u32-codes", "data": "synthetic",
        "config": {"workload": wl, "n": n, "dims": d, "eb": eb, "eb_frac_of_range": 1e-3, "p": p, "threshold": t,
                   "l2_flush": "inputs larger than L2 (input %d MB)" % (raw // 2**20),
                   "parallelism": f"replicas{world}"},
        "e2e": {"value": round(gbs(t_ce), 3), "unit": UNIT, "h2d_bytes_per_step": raw, "d2h_bytes_per_step": clen},
        "decompress": {"value": round(gbs(t_d), 3), "unit": UNIT,
                       "e2e": {"value": round(gbs(t_de), 3), "unit": UNIT, "h2d_bytes_per_step": clen,
                               "d2h_bytes_per_step": n * d * 8}},
        "compressed_bytes": clen, "ratio": round(raw / clen, 4), "max_abs_err_over_eb": err / eb,
        "ms": {"compress": t_c * 1e3, "decompress": t_d * 1e3, "compress_e2e": t_ce * 1e3,
               "decompress_e2e": t_de * 1e3},
        "peak_source": src,
    }
    if clk:
        line["clocks"] = clk
    codec.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="blobs", choices=["blobs", "column", "trajectory"])
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps({"impl": "reference", "unavailable": "not implemented yet"}))
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_ours(args, rank, world)
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
