"""Chain compressor benchmark (one JSON line on rank 0).

Workload (default): the large single frame -- 16,777,216 float32 particles in
[0,100]^3, 80% from 64 Gaussian blobs and 20% uniform, random particle order,
eb = 1e-3 x range, p = 4, threshold = 2.  Seeded synthetic data (the reference names no
public dataset).  A step = one compress of the frame; the decompress of its container
is timed the same way and reported beside it.

  value : compress throughput in GB/s of uncompressed input, input already in HBM,
          container left in HBM; device time from CUDA events on the library's stream,
          max over ranks
  e2e   : the same through the C ABI with pinned HOST buffers: H2D of the points and
          D2H of the container inside the timed region
  decompress : the same two numbers for the decoder (container -> float64 points)
  roofline   : the dominant kernel of the compress step (radix_scatter_kernel, one
          launch per sort pass) against the measured HBM copy bandwidth;
          roofline_rans_encode for the encoder's entropy kernel; decompress.roofline
          for rans_decode_kernel; path_roofline: (input + container bytes) / step time

On one GPU the line also carries `batch` (the uneven 256-frame collection through
chain_batch_compress against one call per frame, as --config batch) and `serve` (the
request server's capacity and p50/p99 at 0.5/0.8/0.95 of it, as --config serve).

Multi-GPU: frames are independent, so N ranks compress N independent frames
(replicas, weak scaling, no collective on the data path; only the timing max-reduce).

--impl reference: the reference's own CPU Chain (cpp/chain/lcps_cpp.cpp, built from
the reference sources into oracle/_ref) on a bounded sample of the same workload (its
first 2^20 particles), one process per host core up to 64, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "oracle"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "compress GB/s (uncompressed bytes/s) at eb=1e-3*range"
UNIT = "GB/s"
SAMPLE_N = 1 << 20


def _peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def _frame(config: str, rank: int, n: int = 0):
    """(points, eb, p, threshold, workload name); n > 0 overrides the blobs frame's size
    (smaller profiling cases of the same distribution)."""
    from chaincompressor_b200 import workloads as W

    if config == "blobs":
        size = n or W.BLOBS_N
        pts = W.blobs(size, seed=1 + rank)
        name = "blobs-16M-f32" if size == W.BLOBS_N else f"blobs-{size}-f32"
        return pts, W.eb_for(pts, 1e-3), 4, 2, name + " (64 Gaussian blobs + 20% uniform, random order)"
    if config == "column":
        pts = W.column(seed=rank)
        return pts, W.eb_for(pts, 1e-3), 4, 2, "column-80703-f32 (dam-break-like lattice, random order)"
    if config == "trajectory":
        pts = W.trajectory(0, seed=2 + rank)
        return pts, W.eb_for(pts, 1e-3), 4, 2, "trajectory-4M-f64 (jittered lattice, periodic box)"
    raise SystemExit(f"unknown config {config}")


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 + ",".join("clocks_event_reasons." + f for f in self.FIELDS),
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
        reasons = sorted({self.FIELDS[k] for r in rows for k, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": rows[0][1], "reasons": reasons,
                "samples": len(rows)}


def max_over_ranks(values, device="cpu"):
    """Element-wise maximum of per-rank timings over the process group (the job's time
    is its slowest rank's).  Every rank calls it once, in the same place."""
    import torch
    import torch.distributed as tdist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return t.tolist()


def _profile_traffic(kernel: str):
    """dram read+write bytes per launch of `kernel` from the committed ncu summary."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(rf"^{kernel} traffic_bytes_per_launch: (\d+)", f.read_text(), re.M)
        if m:
            return int(m.group(1)), f.name
    return None, None


def _cpu_baseline(pts, eb, p, t):
    """Reference CPU compress (oracle/_ref) of the first 2^20 particles, one core."""
    import oracle

    if not oracle.ref_available():
        return None
    sample = np.ascontiguousarray(pts[:SAMPLE_N])
    oracle.ref_compress(sample[:4096], eb, p, t)
    reps, t0 = 0, time.perf_counter()
    while True:
        oracle.ref_compress(sample, eb, p, t)
        reps += 1
        el = time.perf_counter() - t0
        if el > 10.0 or reps >= 4:
            break
    return {"value": round(reps * sample.nbytes / el / 1e9, 6), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"first {len(sample)} particles of the same frame, {reps} compress call(s), "
                      f"{el:.1f} s; reference lcps_cpp.lcps_compress2 is single-threaded"}


def run_ours(args, rank: int, world: int):
    import torch

    from chaincompressor_b200 import _native as N

    ndev = max(1, torch.cuda.device_count())
    dev = int(os.environ.get("LOCAL_RANK", rank)) % ndev
    torch.cuda.set_device(dev)
    pts, eb, p, t, wl = _frame(args.config, rank, args.n)
    n, d = pts.shape
    esz = pts.dtype.itemsize
    raw = n * d * esz
    soa_host = torch.from_numpy(np.ascontiguousarray(pts.T)).pin_memory()
    soa_dev = soa_host.to(f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)
    codec = N.Codec(dev, stream=stream.cuda_stream)
    dist = world > 1
    if dist:
        import torch.distributed as tdist

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    dtype_code = N.CHAIN_F32 if esz == 4 else N.CHAIN_F64
    comp = lambda ptr: codec.compress_ptr(ptr, dtype_code, N.CHAIN_SOA, n, d, eb, p, t)  # noqa: E731
    for _ in range(args.warmup):
        comp(soa_dev.data_ptr())
    clen = comp(soa_dev.data_ptr())
    cont_dev = torch.empty(clen, dtype=torch.uint8, device=f"cuda:{dev}")
    codec.result_copy_to(cont_dev.data_ptr(), clen)
    cont_host = torch.empty(clen, dtype=torch.uint8).pin_memory()
    cont_host.copy_(cont_dev.cpu())
    out_dev = torch.empty((n, d), dtype=torch.float64, device=f"cuda:{dev}")
    out_host = torch.empty((n, d), dtype=torch.float64).pin_memory()
    decomp = lambda src, dst: codec.decompress_ptr(src, clen, dst, n * d * 8)  # noqa: E731
    for _ in range(args.warmup):
        decomp(cont_dev.data_ptr(), out_dev.data_ptr())
    # the host-buffer calls stage through the same arenas; warm them too
    for _ in range(args.warmup):
        comp(soa_host.data_ptr())
        codec.result_copy_to(cont_host.data_ptr(), clen)
        decomp(cont_host.data_ptr(), out_host.data_ptr())

    counts = {}   # stage marks per step (a stage named more than once is summed)

    def timed(fn, stages=False):
        """Device time per step from CUDA events on the library stream (the library
        calls are synchronous, so the events bracket all of their device work)."""
        codec.set_stage_timing(stages)
        acc, occ = {}, {}
        barrier()
        l0 = N.launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            fn()
            if stages:
                for name, ms in codec.stage_times():
                    acc[name] = acc.get(name, 0.0) + ms
                    occ[name] = occ.get(name, 0) + 1
        ev1.record(stream)
        barrier()
        launches = N.launch_count() - l0
        codec.set_stage_timing(False)
        counts.update({k: v // args.steps for k, v in occ.items()})
        return ev0.elapsed_time(ev1) / 1e3 / args.steps, launches, {k: v / args.steps for k, v in acc.items()}

    clocks = Clocks(dev)
    # headline timings without stage events; the per-stage breakdown (and the per-kernel
    # durations of the roofline) come from a second pass of the same steps with them
    t_c, launches_c, _ = timed(lambda: comp(soa_dev.data_ptr()))
    t_d, launches_d, _ = timed(lambda: decomp(cont_dev.data_ptr(), out_dev.data_ptr()))
    _, _, stages_c = timed(lambda: comp(soa_dev.data_ptr()), stages=True)
    _, _, stages_d = timed(lambda: decomp(cont_dev.data_ptr(), out_dev.data_ptr()), stages=True)

    def e2e_c():
        comp(soa_host.data_ptr())
        codec.result_copy_to(cont_host.data_ptr(), clen)

    t_ce, _, _ = timed(e2e_c)
    t_de, _, _ = timed(lambda: decomp(cont_host.data_ptr(), out_host.data_ptr()))
    clk = clocks.stop()
    if dist:
        t_c, t_d, t_ce, t_de = max_over_ranks([t_c, t_d, t_ce, t_de], f"cuda:{dev}")
    dec = out_host.numpy()
    err = float(np.abs(dec - pts.astype(np.float64)).max())

    # roofline of the dominant kernels: algorithmic bytes per launch / event-timed duration
    from chaincompressor_b200 import lcg2

    info = lcg2.inspect(bytes(cont_host.numpy()))
    rans_syms = sum(c["section"]["symbols"] for c in info["components"].values() if "section" in c)
    rans_bytes = sum(c["section"]["payload"] + c["section"]["state_bytes"] + 4 * c["section"]["chunks"]
                     for c in info["components"].values() if "section" in c)
    # bytes of the symbols the encoder reads: the library stores each stream no wider than
    # its values (rel: one byte when p <= 256; choice2: one; keep / diff: the narrowest of
    # 1, 2, 4 bytes holding kb + 1 bits, kb = bits of the largest block coordinate, which
    # the container's wrap maximum equals); tags and idrel are four bytes
    kb = int(info["wrap"][1]).bit_length()
    kd = 1 if kb + 1 <= 8 else (2 if kb + 1 <= 16 else 4)
    width = {"IDR0": 4, "DIF0": kd, "KEP0": kd, "CH20": 1, "REL0": 1 if info["p"] <= 256 else 4}
    rans_sym_bytes = sum(c["section"]["symbols"] * (4 if c["enc"] == "tagged" else width[name])
                         for name, c in info["components"].items() if "section" in c)
    peaks, src = _peaks()
    peak = float(peaks["hbm_gbs"])

    def roof(kernel, stage_ms, alg_bytes, launches=1):
        if not stage_ms:
            return None
        stage_ms = stage_ms / launches
        ach = alg_bytes / (stage_ms / 1e3) / 1e9
        traffic, prof = _profile_traffic(kernel)
        return {"kernel": kernel, "bound": "hbm", "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                "avg_launch_ms": round(stage_ms, 4), "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic_source": prof}

    # radix scatter: pass 0 reads keys (indices are implicit) and writes keys + indices;
    # later passes read and write both
    scatter_roof = None
    for kw in (4, 8):
        name = f"sort_scatter_k{kw * 8}"
        passes = counts.get(name, 0)
        if passes:
            alg = (n * (kw + kw + 4) + (passes - 1) * n * 2 * (kw + 4)) // passes
            scatter_roof = roof("radix_scatter_kernel", stages_c.get(name), alg, passes)
            if scatter_roof:
                scatter_roof["launches_per_step"] = passes

    gbs = lambda sec: world * raw / sec / 1e9  # noqa: E731
    line = {
        "metric": METRIC, "value": round(gbs(t_c), 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_c * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 quantize, u32 codes, u8 rANS", "data": "synthetic (seeded)",
        "config": {"workload": wl, "n": n, "dims": d, "input_dtype": str(pts.dtype), "eb": eb,
                   "eb_frac_of_range": 1e-3, "p": p, "threshold": t,
                   "l2_flush": f"inputs larger than L2 ({raw >> 20} MB input per frame)",
                   "parallelism": f"replicas x{world} (independent frames)"},
        "e2e": {"value": round(gbs(t_ce), 3), "unit": UNIT, "h2d_bytes_per_step": raw, "d2h_bytes_per_step": clen},
        "gpu_launches": launches_c, "gpu_launches_per_step": launches_c // max(1, args.steps),
        "roofline": scatter_roof,
        "roofline_rans_encode": roof("rans_encode_kernel", stages_c.get("rans_encode"), rans_sym_bytes + rans_bytes),
        "decompress": {"value": round(gbs(t_d), 3), "unit": UNIT, "ms_per_step": round(t_d * 1e3, 4),
                       "gpu_launches": launches_d,
                       "e2e": {"value": round(gbs(t_de), 3), "unit": UNIT, "h2d_bytes_per_step": clen,
                               "d2h_bytes_per_step": n * d * 8},
                       "roofline": roof("rans_decode_kernel", stages_d.get("rans_decode"),
                                        4 * rans_syms + rans_bytes)},
        "path_roofline": {"compress_frac": round((raw + clen) / t_c / 1e9 / peak, 4),
                          "decompress_frac": round((clen + n * d * 8) / t_d / 1e9 / peak, 4),
                          "note": "algorithmic bytes = input + container (compress), container + "
                                  "float64 output (decompress), per step / device time"},
        "compressed_bytes": clen, "ratio": round(raw / clen, 4), "max_abs_err_over_eb": err / eb,
        "exact_corrections": info["corrections"]["count"],
        "stages_ms": {"compress": {k: round(v, 4) for k, v in stages_c.items()},
                      "decompress": {k: round(v, 4) for k, v in stages_d.items()}},
        "ms": {"compress": t_c * 1e3, "decompress": t_d * 1e3, "compress_e2e": t_ce * 1e3,
               "decompress_e2e": t_de * 1e3},
    }
    if clk:
        line["clocks"] = clk
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _cpu_baseline(pts, eb, p, t)
    codec.close()
    return line


def run_batch_bench(args):
    """The uneven collection (256 frames, N log-uniform in [1e4, 2e6], column / blobs /
    uniform content, eb in {1e-2, 1e-3, 1e-4} x range, float32), device-resident: one
    frame per chain_compress call on one context, against chain_batch_compress with
    `--workers` contexts.  Frames run on several streams, so the time of a pass is the
    host wall clock between device synchronisations around the whole collection."""
    import torch

    from chaincompressor_b200 import _native as N
    from chaincompressor_b200 import workloads as W

    torch.cuda.set_device(0)
    specs = W.uneven_specs(256, seed=3)
    frames = []
    for n, kind, frac, seed in specs:
        pts = W.make_frame(n, kind, seed)
        eb = W.eb_for(pts, frac)
        frames.append((torch.from_numpy(np.ascontiguousarray(pts.T)).cuda(), n, eb))
    raw = sum(n * 3 * 4 for _, n, _ in frames)
    caps = [N.compress_bound(n, 3) for _, n, _ in frames]
    outbuf = torch.empty(sum(caps), dtype=torch.uint8, device="cuda")
    offs = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    codec = N.Codec(0)

    def seq_compress():
        lens = []
        for (x, n, eb), off, cap in zip(frames, offs, caps):
            ln = codec.compress_ptr(x.data_ptr(), N.CHAIN_F32, N.CHAIN_SOA, n, 3, eb, 4, 2)
            codec.result_copy_to(outbuf.data_ptr() + int(off), cap)
            lens.append(ln)
        return lens

    items = [N.BatchItem(input=x.data_ptr(), dtype=N.CHAIN_F32, layout=N.CHAIN_SOA, n=n, dims=3, eb=eb, p=4,
                         threshold=2, output=outbuf.data_ptr() + int(off), output_capacity=cap)
             for (x, n, eb), off, cap in zip(frames, offs, caps)]
    batch = N.Batch(0, workers=args.workers or 8)

    def bat_compress():
        arr = batch.compress_items(items)
        return [arr[i].output_bytes for i in range(len(items))]

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        l0 = N.launch_count()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / args.steps, out, (N.launch_count() - l0) // args.steps

    t_seq, lens_seq, l_seq = timed(seq_compress)
    t_bat, lens_bat, l_bat = timed(bat_compress)
    assert lens_seq == lens_bat
    # the autotuner on a sample of the collection (every eighth frame), then the tuned batch
    tune = batch.tune_items(items[::8])
    t_tun, lens_tun, l_tun = timed(bat_compress)
    # decompression of the (tuned batch's) containers, now in outbuf, into float64 AoS
    # device buffers
    outs = torch.empty(sum(n * 3 for _, n, _ in frames), dtype=torch.float64, device="cuda")
    ooffs = np.concatenate([[0], np.cumsum([n * 3 for _, n, _ in frames])[:-1]]).astype(np.int64)

    def seq_decompress():
        for (x, n, eb), off, ln, oo in zip(frames, offs, lens_tun, ooffs):
            codec.decompress_ptr(outbuf.data_ptr() + int(off), ln, outs.data_ptr() + 8 * int(oo), n * 3 * 8)
        return None

    ditems = [N.BatchItem(input=outbuf.data_ptr() + int(off), input_bytes=ln, dtype=N.CHAIN_F64, layout=N.CHAIN_AOS,
                          output=outs.data_ptr() + 8 * int(oo), output_capacity=n * 3 * 8)
              for (x, n, eb), off, ln, oo in zip(frames, offs, lens_tun, ooffs)]

    def bat_decompress():
        batch.decompress_items(ditems)
        return None

    td_seq, _, ld_seq = timed(seq_decompress)
    td_bat, _, ld_bat = timed(bat_decompress)
    batch.close()
    codec.close()
    gbs = lambda s: raw / s / 1e9  # noqa: E731
    return {
        "metric": "batch compress GB/s (uncompressed bytes/s) over 256 uneven frames", "value": round(gbs(t_tun), 3),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_tun * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 quantize, u32 codes, u8 rANS", "data": "synthetic (seeded)",
        "config": {"workload": "uneven-256 (N log-uniform 1e4..2e6; column/blobs/uniform; eb 1e-2/1e-3/1e-4 x range;"
                               " f32)", "frames": len(frames), "points": sum(n for _, n, _ in frames),
                   "workers": args.workers or 8, "timing": "host wall clock per pass, device synchronised on both sides",
                   "l2_flush": "inputs larger than L2 (whole collection > 1 GB)"},
        "sequential": {"value": round(gbs(t_seq), 3), "ms_per_step": round(t_seq * 1e3, 3), "gpu_launches": l_seq},
        "speedup_vs_sequential": round(t_seq / t_tun, 3), "gpu_launches": l_tun,
        "untuned": {"value": round(gbs(t_bat), 3), "ms_per_step": round(t_bat * 1e3, 3),
                    "speedup_vs_sequential": round(t_seq / t_bat, 3), "workers": args.workers or 8, "rans_max_steps": 1024,
                    "compressed_bytes": int(sum(lens_bat))},
        "tuned": {"rans_max_steps": tune["rans_max_steps"], "workers": tune["workers"],
                  "sample_frames": len(items[::8]), "sample_ms": round(tune["best_ms"], 3),
                  "sample_default_ms": round(tune["default_ms"], 3),
                  "bytes_vs_default": round(sum(lens_tun) / sum(lens_bat), 5)},
        "decompress": {"value": round(gbs(td_bat), 3), "ms_per_step": round(td_bat * 1e3, 3),
                       "sequential": round(gbs(td_seq), 3), "speedup_vs_sequential": round(td_seq / td_bat, 3),
                       "gpu_launches": ld_bat},
        "compressed_bytes": int(sum(lens_tun)),
    }


def run_serve_bench(args):
    """Serving loop: `--requests` requests (50% compress, 50% decompress of containers
    made beforehand) over a seeded pool of 48 frames (N log-uniform in [1e3, 8e6];
    column / blobs / uniform content; eb in {1e-2, 1e-3, 1e-4} x range; 70% float32,
    30% float64; device-resident) through chain_server with `--workers` contexts and a
    40 GB admission budget.  First the capacity (all requests queued at once), then
    Poisson arrivals at 0.5, 0.8 and 0.95 of it; latency = queueing + service time as
    stamped by the server.  Every request writes its own output region: regions are cut
    in submission order from a device ring large enough that a region is reused only
    long after its previous user finished, and each run checks from the server's time
    stamps that no two requests whose regions overlap were ever in service at once."""
    import threading

    import torch

    from chaincompressor_b200 import _native as N
    from chaincompressor_b200 import workloads as W

    torch.cuda.set_device(0)
    rng = np.random.default_rng(4)
    pool = []
    codec = N.Codec(0)
    for k in range(48):
        n = int(np.floor(np.exp(rng.uniform(np.log(1e3), np.log(8e6)))))
        kind = ("column", "blobs", "uniform")[int(rng.integers(0, 3))]
        frac = float((1e-2, 1e-3, 1e-4)[int(rng.integers(0, 3))])
        dt = np.float32 if rng.random() < 0.7 else np.float64
        pts = W.make_frame(n, kind, int(rng.integers(0, 2**31 - 1)), dt)
        eb = W.eb_for(pts, frac)
        x = torch.from_numpy(np.ascontiguousarray(pts.T)).cuda()
        code = N.CHAIN_F32 if dt == np.float32 else N.CHAIN_F64
        ln = codec.compress_ptr(x.data_ptr(), code, N.CHAIN_SOA, n, 3, eb, 4, 2)
        cont = torch.empty(ln, dtype=torch.uint8, device="cuda")
        codec.result_copy_to(cont.data_ptr(), ln)
        cap = N.compress_bound(n, 3)
        pool.append(dict(x=x, n=n, eb=eb, code=code, cont=cont, ln=ln, cap=cap, raw=n * 3 * pts.dtype.itemsize))
    codec.close()
    torch.cuda.synchronize()
    R = args.requests
    picks = rng.integers(0, len(pool), size=R)
    ops = rng.integers(0, 2, size=R)
    # output regions: consecutive, 256-byte aligned slices of one device ring
    ring_bytes = 6 << 30
    ring = torch.empty(ring_bytes, dtype=torch.uint8, device="cuda")
    region = np.zeros((R, 2), np.int64)   # [offset, bytes]
    lap = np.zeros(R, np.int64)            # how often the ring had wrapped before the request
    off, laps = 0, 0
    for i, (f, op) in enumerate(zip(picks, ops)):
        P = pool[int(f)]
        need = (P["ln"] if op == 0 else P["n"] * 24) + 255 & ~255
        if off + need > ring_bytes:
            off, laps = 0, laps + 1
        region[i] = (off, need)
        lap[i] = laps
        off += need
    items = []
    for i, (f, op) in enumerate(zip(picks, ops)):
        P = pool[int(f)]
        out_ptr = ring.data_ptr() + int(region[i, 0])
        if op == 0:
            items.append(N.BatchItem(input=P["x"].data_ptr(), dtype=P["code"], layout=N.CHAIN_SOA, n=P["n"], dims=3,
                                     eb=P["eb"], p=4, threshold=2, output=out_ptr, output_capacity=P["ln"]))
        else:
            items.append(N.BatchItem(input=P["cont"].data_ptr(), input_bytes=P["ln"], dtype=N.CHAIN_F64,
                                     layout=N.CHAIN_AOS, output=out_ptr, output_capacity=P["n"] * 24))
    # requests whose regions overlap, as (earlier, later) pairs: a region overlaps only
    # regions of the previous lap of the ring (no region exceeds the ring)
    overlaps = []
    starts, ends = region[:, 0], region[:, 0] + region[:, 1]
    by_lap = {int(k): np.nonzero(lap == k)[0] for k in np.unique(lap)}
    for j in np.nonzero(lap > 0)[0]:
        prev = by_lap[int(lap[j]) - 1]
        hit = prev[(starts[prev] < ends[j]) & (starts[j] < ends[prev])]
        overlaps.extend((int(i), int(j)) for i in hit)
    raw_total = sum(pool[int(f)]["raw"] for f in picks)
    srv = N.Server(0, workers=args.workers or 4, memory_budget_bytes=40 << 30)

    def run(arrivals):
        """Submit item i at t0 + arrivals[i] (seconds); returns (latencies ms, wall s)."""
        tickets = [None] * R
        lat = np.zeros(R)
        qs = np.zeros(R)
        sub = np.zeros(R)
        failed = [0]

        def waiter():
            for i in range(R):
                while tickets[i] is None:
                    time.sleep(2e-5)
                st, q, s, _ = srv.wait(tickets[i], check=False)
                lat[i] = q + s
                qs[i] = q
                failed[0] += st != 0

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        for i in range(R):
            target = t0 + arrivals[i]
            while True:
                d = target - time.perf_counter()
                if d <= 0:
                    break
                time.sleep(min(d, 5e-4) if d > 1e-3 else 0)
            sub[i] = time.perf_counter()
            tickets[i] = srv.submit(int(ops[i]), items[i])
        th.join()
        torch.cuda.synchronize()
        if failed[0]:
            raise RuntimeError(f"{failed[0]} of {R} requests failed")
        # no two requests with overlapping output regions were in service together
        # (start = submit + queueing, end = start + service; 50 us of stamp slack)
        for i, j in overlaps:
            end_i = sub[i] + lat[i] / 1e3
            start_j = sub[j] + qs[j] / 1e3
            if start_j < end_i + 5e-5:
                raise RuntimeError(f"requests {i} and {j} shared output memory while both ran")
        run.queue = qs
        return lat, time.perf_counter() - t0

    run(np.zeros(R))   # warm-up: the resident arenas reach their sizes
    # isolated latency of every (pool frame, operation): the request served alone on the
    # idle server, median of five
    iso_tab = np.zeros((len(pool), 2))
    first = {}
    for i, (f, op) in enumerate(zip(picks, ops)):
        first.setdefault((int(f), int(op)), i)
    for (f, op), i in first.items():
        ts = []
        for _ in range(5):
            st, q, s, _ = srv.wait(srv.submit(op, items[i]), check=True)
            ts.append(q + s)
        iso_tab[f, op] = float(np.median(ts))
    iso = iso_tab[picks, ops]
    big = iso >= np.percentile(iso, 90)   # the slowest tenth of the mix when served alone
    lat0, wall0 = run(np.zeros(R))
    capacity = R / wall0
    loads = []
    for f in (0.5, 0.8, 0.95):
        lam = f * capacity
        arr = np.cumsum(np.random.default_rng(5).exponential(1.0 / lam, size=R))
        lat, wall = run(arr)
        p99 = float(np.percentile(lat, 99))
        loads.append({"load": f, "offered_rps": round(lam, 1), "achieved_rps": round(R / wall, 1),
                      "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(p99, 3),
                      "mean_ms": round(float(lat.mean()), 3),
                      "p99_over_isolated_p99": round(p99 / float(np.percentile(iso, 99)), 3),
                      "slowdown_p50": round(float(np.percentile(lat / iso, 50)), 3),
                      "slowdown_p99": round(float(np.percentile(lat / iso, 99)), 3),
                      "queue_p99_ms": round(float(np.percentile(run.queue, 99)), 3),
                      "service_p99_ms": round(float(np.percentile(lat - run.queue, 99)), 3),
                      "p99_large_ms": round(float(np.percentile(lat[big], 99)), 3),
                      "p99_small_ms": round(float(np.percentile(lat[~big], 99)), 3)})
    srv.close()
    return {
        "metric": "serving capacity (requests/s), mixed compress/decompress", "value": round(capacity, 1),
        "unit": "requests/s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": round(wall0 * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 quantize, u32 codes, u8 rANS", "data": "synthetic (seeded)",
        "config": {"workload": "serving mix: 48-frame pool, N log-uniform 1e3..8e6, 70% f32 / 30% f64, "
                               "50% compress / 50% decompress", "requests": R, "workers": args.workers or 4,
                   "memory_budget_gb": 40, "timing": "server-stamped queueing + service time per request; "
                                                     "capacity = requests / wall time with all queued at once"},
        "capacity_gbs": round(raw_total / wall0 / 1e9, 3),
        "saturated": {"p50_ms": round(float(np.percentile(lat0, 50)), 3),
                      "p99_ms": round(float(np.percentile(lat0, 99)), 3)},
        "isolated": {"p50_ms": round(float(np.percentile(iso, 50)), 3), "p99_ms": round(float(np.percentile(iso, 99)), 3),
                     "note": "each request's latency served alone on the idle server (median of 5), over the "
                             "same request mix; slowdown = served latency / isolated latency per request"},
        "loads": loads,
    }


_REF_JOB = None


def _ref_init(job):
    global _REF_JOB
    _REF_JOB = job


def _ref_worker(_):
    import oracle

    pts, eb, p, t = _REF_JOB
    t0 = time.perf_counter()
    oracle.ref_compress(pts, eb, p, t)
    return time.perf_counter() - t0


def run_reference(args):
    import multiprocessing as mp

    import oracle

    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "reference CPU modules (oracle/_ref) were not built"}
    pts, eb, p, t, wl = _frame(args.config, 0)
    sample = np.ascontiguousarray(pts[:SAMPLE_N])
    cores = max(1, min(os.cpu_count() or 1, 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_init, initargs=((sample, eb, p, t),)) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_worker, range(cores))
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            pool.map(_ref_worker, range(cores))
            times.append(time.perf_counter() - t0)
    step = float(np.mean(times))
    value = cores * sample.nbytes / step / 1e9
    n, d = pts.shape
    sample_desc = (f"each step: {cores} processes each compress the first {len(sample)} particles "
                   f"({sample.nbytes >> 20} MB) of the frame with lcps_cpp.lcps_compress2")
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": wl, "n": n, "dims": d, "eb": eb, "eb_frac_of_range": 1e-3, "p": p, "threshold": t},
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample_desc},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_once(args):
    """Compress + decompress the workload twice (the first pair warms the arenas)."""
    import torch

    from chaincompressor_b200 import _native as N

    pts, eb, p, t, wl = _frame(args.config, 0, args.n)
    n, d = pts.shape
    soa = torch.from_numpy(np.ascontiguousarray(pts.T)).cuda()
    codec = N.Codec(0)
    dt = N.CHAIN_F32 if pts.dtype == np.float32 else N.CHAIN_F64
    out = torch.empty((n, d), dtype=torch.float64, device="cuda")
    for _ in range(2):
        clen = codec.compress_ptr(soa.data_ptr(), dt, N.CHAIN_SOA, n, d, eb, p, t)
        cont = torch.empty(clen, dtype=torch.uint8, device="cuda")
        codec.result_copy_to(cont.data_ptr(), clen)
        codec.decompress_ptr(cont.data_ptr(), clen, out.data_ptr(), out.numel() * 8)
    torch.cuda.synchronize()
    err = float((out.cpu().numpy() - pts).__abs__().max()) / eb
    print(json.dumps({"workload": wl, "compressed_bytes": clen, "max_abs_err_over_eb": err}))
    codec.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="blobs", choices=["blobs", "column", "trajectory", "batch", "serve"])
    ap.add_argument("--requests", type=int, default=20000, help="requests of the serving run (--config serve)")
    ap.add_argument("--workers", type=int, default=0,
                    help="contexts of the batch path (default 8) or of the request server (default 4)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-system-forms", action="store_true",
                    help="skip the batched and served runs that the default line reports beside the frame")
    ap.add_argument("--n", type=int, default=0,
                    help="particles of the blobs frame (default 16,777,216); smaller sizes are profiling cases")
    ap.add_argument("--once", action="store_true",
                    help="one warm-up and one measured compress + decompress, no timing (for ncu launch lists)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.gpus < 1:
        raise SystemExit("--gpus must be >= 1")
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # not started by torchrun: start the N local ranks ourselves
        return spawn_local_ranks(args.gpus, sys.argv[1:])
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one rank per GPU", file=sys.stderr)
        return 2
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return 0
    if args.once:
        run_once(args)
        return 0
    if args.config in ("batch", "serve") and world > 1:
        print(f"bench.py: --config {args.config} runs on one GPU", file=sys.stderr)
        return 2
    if args.config == "batch":
        print(json.dumps(run_batch_bench(args)))
        return 0
    if args.config == "serve":
        print(json.dumps(run_serve_bench(args)))
        return 0
    import torch

    gpu = torch.cuda.is_available()
    if world > 1:
        import datetime

        import torch.distributed as tdist

        if gpu:
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)) % torch.cuda.device_count())
        tdist.init_process_group("nccl" if gpu else "gloo", timeout=datetime.timedelta(seconds=120))
    line = _rank_work()(args, rank, world)
    if world > 1:
        import torch.distributed as tdist

        tdist.destroy_process_group()
    if rank == 0 and world == 1 and args.config == "blobs" and not args.n and not args.no_system_forms \
            and "CHAIN_BENCH_RANK_FN" not in os.environ:
        line.update(_system_forms(args))
    if rank == 0:
        print(json.dumps(line))
    return 0


def _system_forms(args):
    """The batched and the served forms of the path (the same runs as --config batch and
    --config serve), summarised beside the single-frame line."""
    import copy

    b_args = copy.copy(args)
    b_args.steps, b_args.warmup = 5, 3
    b = run_batch_bench(b_args)
    s_args = copy.copy(args)
    s = run_serve_bench(s_args)
    return {
        "batch": {k: b[k] for k in ("metric", "value", "unit", "ms_per_step", "speedup_vs_sequential", "sequential",
                                    "untuned", "tuned", "decompress", "compressed_bytes", "config")},
        "serve": {k: s[k] for k in ("metric", "value", "unit", "capacity_gbs", "isolated", "loads", "config")},
    }


def _rank_work():
    """The per-rank step function: run_ours, or -- for tests of the launch path on
    machines without a GPU -- the callable named by CHAIN_BENCH_RANK_FN
    ("module:function", same signature)."""
    spec = os.environ.get("CHAIN_BENCH_RANK_FN")
    if not spec:
        return run_ours
    import importlib

    mod, fn = spec.split(":")
    return getattr(importlib.import_module(mod), fn)


def spawn_local_ranks(nproc: int, argv) -> int:
    """Starts `nproc` ranks of this script on this node through torch.distributed.run
    (rendezvous on 127.0.0.1, a free port) and returns its exit status; rank 0 prints
    the JSON line.  Used when bench.py --gpus N (N > 1) is started without torchrun."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *argv]
    return subprocess.run(cmd).returncode


if __name__ == "__main__":
    sys.exit(main())
