"""Writes tests/golden/lcg2/<case>.lcg2: the GPU encoder's container for the input of
every golden fixture in this directory (same points and parameters).

Run on a machine with a CUDA GPU and the built library:

    python tests/golden/make_lcg2.py [output directory, default tests/golden/lcg2]

tests/test_transcode.py (CPU) transcodes these containers to LCP2 and checks that the
reference decoder returns each fixture's stored reference output.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT)]

from chaincompressor_b200 import _native as N  # noqa: E402


def main():
    out_dir = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "lcg2"
    out_dir.mkdir(exist_ok=True)
    codec = N.Codec(0)
    for f in sorted(HERE.glob("*.npz")):
        z = np.load(f)
        pts = z["points"]
        data = codec.compress(np.ascontiguousarray(pts.T), float(z["eb"]), int(z["p"]), int(z["threshold"]),
                              layout=N.CHAIN_SOA, bl=bool(z["bl"]), l1=bool(z["l1"]), l2=bool(z["l2"]))
        (out_dir / (f.stem + ".lcg2")).write_bytes(data)
        print(f.stem, len(data))
    codec.close()


if __name__ == "__main__":
    main()
