"""Generates tests/golden/dambreak/frame0654.npz from the reference's bundled DamBreak frame and
the REFERENCE CPU Chain.

Run where the reference checkout and its modules are built (oracle/_ref, compiled from
the reference sources by oracle/Makefile):

    python tests/golden/make_dambreak.py

The frame is data/DamBreak/0654_*.vtp of the reference (80,703 float32 particles), read
as the reference's reader.py:24-61 reads it (the 'Points' DataArray, whitespace
separated, float32).  The cases are the experiment tables of reader.py:
  * CPU table (testCPU, reader.py:300-302):  qb 11..14 -> (p, threshold) =
    (256, 4), (4, 25), (16, 22), (16, 25)
  * GPU table (testGPU, reader.py:343-344):  qb 11..14 -> (p, threshold) =
    (2, 2), (4, 2), (16, 16), (16, 2)
with eb = equivalent_eb(range, qb - 1) = max per-axis extent / (2^qb - 2)
(reader.py:269-272, 309).

Stored per case: the parameters, the size of the reference encoder's LCP2 bitstream,
the SHA-256 of each of the five integer streams and of the exact corrections as the
reference's own component decoder reads them back out of that bitstream
(lcps_cpp.cpp:1715-1825; canonical form: int64 little-endian, C order, shape (D, records)),
and the SHA-256 of the reference serial decoder's float64 (N, D) output.  The points are
stored once.  tests/test_gpu_dambreak.py holds the GPU path to these digests; the
digests keep the fixture small (the streams themselves would be megabytes).
"""
import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]

import oracle  # noqa: E402

STREAMS = ("idrel", "diff", "keep", "choice2", "rel")
CPU_TABLE = {11: (256, 4), 12: (4, 25), 13: (16, 22), 14: (16, 25)}
GPU_TABLE = {11: (2, 2), 12: (4, 2), 13: (16, 16), 14: (16, 2)}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype="<i8")).tobytes()).hexdigest()


def digest_f64(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype="<f8")).tobytes()).hexdigest()


def read_frame() -> np.ndarray:
    import xml.etree.ElementTree as ET

    files = sorted((oracle.reference_dir() / "data" / "DamBreak").glob("0654*.vtp"))
    if len(files) != 1:
        raise SystemExit("reference DamBreak frame 0654 not found")
    root = ET.parse(files[0]).getroot()
    for da in root.iter("DataArray"):
        if da.attrib.get("Name") == "Points":
            return np.array(da.text.split(), dtype=np.float32).reshape(-1, 3)
    raise SystemExit("no Points DataArray")


def main():
    if not oracle.ref_available():
        raise SystemExit("build the reference modules first: make -C oracle ref")
    pts = read_frame()
    rng_ = float(np.max(pts.max(0).astype(np.float64) - pts.min(0)))
    rows = []
    for table, tab in (("cpu", CPU_TABLE), ("gpu", GPU_TABLE)):
        for qb, (p, t) in tab.items():
            eb = rng_ / (2 ** qb - 2)
            data = oracle.ref_compress(pts, eb, p, t)
            rs = oracle.ref_streams(data)
            dec = oracle.ref_decompress(data)
            assert np.abs(dec - pts.astype(np.float64)).max() <= eb
            row = {"table": table, "qb": qb, "p": p, "threshold": t, "eb": eb, "lcp2_bytes": len(data),
                   "exact_index": digest(rs["exact_index"].astype(np.int64)),
                   "exact_count": int(len(rs["exact_index"])), "decoded": digest_f64(dec)}
            for k in STREAMS:
                a = np.asarray(rs[k], np.int64)
                row[k] = digest(a)
                row[k + "_shape"] = list(a.shape)
            rows.append(row)
            print(table, qb, p, t, len(data), "bytes")
    import json

    (HERE / "dambreak").mkdir(exist_ok=True)
    np.savez_compressed(HERE / "dambreak" / "frame0654.npz", points=pts, cases=np.array(json.dumps(rows)))
    print("wrote", HERE / "dambreak" / "frame0654.npz", (HERE / "dambreak" / "frame0654.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    main()
