"""Generates the golden fixtures in this directory from the REFERENCE CPU Chain.

Run where the reference modules are built (oracle/_ref: lcps_cpp, lcps_cpu_decompress,
lcps_ref_streams, compiled from the reference sources by oracle/Makefile):

    python tests/golden/make_golden.py

For each seeded case it stores the input points and parameters, the five integer
streams and exact corrections read back out of the reference encoder's LCP2 bitstream
(by the reference's own component decoder), the LCP2 byte size and component codecs,
and the reference serial decoder's float64 output.  tests/test_oracle.py checks the
oracle restatement against these files; they need no reference build to be checked.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]

import oracle  # noqa: E402
from chaincompressor_b200 import workloads as W  # noqa: E402


def cases():
    rng = np.random.default_rng(2024)
    col = W.column(3000, seed=31)
    yield "column3k", col, W.eb_for(col, 1e-3), 4, 2, {}
    yield "column3k_qb11", col, float(np.max(col.max(0).astype(np.float64) - col.min(0))) / (2 ** 11 - 2), 256, 4, {}
    clip = W.blobs(4000, seed=32, clip=True)
    yield "blobs_clipped4k", clip, W.eb_for(clip, 1e-3), 4, 2, {}
    tr = W.trajectory(1, n=3000, seed=33)
    yield "traj3k_f64_p1", tr, W.eb_for(tr, 1e-4), 1, 2, {}
    yield "uniform2k_p64_t25", W.uniform(2000, 34), 0.001 * 100, 64, 25, {}
    yield "dims1_gauss", rng.normal(0, 3, size=(2500, 1)), 1e-3, 8, 1, {}
    yield "dims2_f32", rng.normal(0, 3, size=(2500, 2)).astype(np.float32), 1e-3, 4, 2, {}
    yield "dims4", rng.uniform(-5, 5, size=(1500, 4)), 1e-2, 4, 2, {}
    yield "neg_threshold", W.column(2000, seed=35), 0.002, 2, -5, {}
    yield "no_l1", W.column(2000, seed=36), 0.002, 4, 2, {"l1": False}
    yield "no_l2", W.column(2000, seed=37), 0.002, 4, 2, {"l2": False}
    yield "no_bl", W.column(2000, seed=38), 0.002, 16, 2, {"bl": False}
    yield "single_point", np.array([[1.5, -2.0, 3.25]]), 0.01, 4, 2, {}
    yield "negative_zero", np.array([[0.0, -0.0], [-0.0, 0.0], [1.0, 2.0], [0.5, -0.0]]), 0.05, 2, 0, {}


def main():
    if not oracle.ref_available():
        raise SystemExit("reference modules not built: make -C oracle ref")
    for name, pts, eb, p, t, kw in cases():
        data = oracle.ref_compress(pts, eb, p, t, **kw)
        rs = oracle.ref_streams(data)
        dec = oracle.ref_decompress(data)
        out = {"points": pts, "eb": eb, "p": p, "threshold": t, "bl": kw.get("bl", True),
               "l1": kw.get("l1", True), "l2": kw.get("l2", True), "lcp2_bytes": len(data),
               "magics": np.array(rs["magics"]), "mins": np.array(rs["mins"]), "wrap_min": rs["wrap_min"],
               "wrap_max": rs["wrap_max"], "exact_index": rs["exact_index"], "exact_value": rs["exact_value"],
               "decoded": dec, "p_eff": rs["p"]}
        for k in ("idrel", "diff", "keep", "choice2", "rel"):
            out[k] = np.asarray(rs[k])
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, len(pts), len(data), rs["magics"])


if __name__ == "__main__":
    main()
