"""The reference's only real data -- its bundled DamBreak frame (80,703 float32
particles) -- through the GPU path, against the reference CPU Chain's own output.

tests/golden/dambreak/frame0654.npz (made by tests/golden/make_dambreak.py where the reference is
built) holds the frame and, for the experiment tables of the reference's reader.py
(CPU table :300-302 and GPU table :343-344, qb 11..14, eb = range / (2^qb - 2)), the
SHA-256 of the five integer streams and exact corrections that the reference encoder
wrote, and of the reference serial decoder's float64 output.  The GPU encoder's streams
and the GPU decoder's output must hash the same (bit-exact), and every point must lie
within eb.  (Sizes are not compared here: this frame is stored in spatial order, and
the reference's Zstd-22 candidates exploit the resulting repeats, which the project's
order-0 entropy stage does not; the measured sizes are reported with the design notes.)
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from chaincompressor_b200 import _native as N

pytestmark = pytest.mark.gpu

_G = np.load(Path(__file__).parent / "golden" / "dambreak" / "frame0654.npz")
POINTS = _G["points"]
CASES = json.loads(str(_G["cases"]))
STREAMS = ("idrel", "diff", "keep", "choice2", "rel")


def _digest(a, dt="<i8"):
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=dt)).tobytes()).hexdigest()


@pytest.mark.parametrize("case", CASES, ids=[f"{c['table']}_qb{c['qb']}" for c in CASES])
def test_dambreak_matches_reference(codec, case):
    n, d = POINTS.shape
    eb = case["eb"]
    data = codec.compress(np.ascontiguousarray(POINTS.T), eb, case["p"], case["threshold"], layout=N.CHAIN_SOA)
    got = codec.debug_streams(n, d)
    for k in STREAMS:
        assert list(got[k].shape) == case[k + "_shape"], k
        assert _digest(got[k]) == case[k], k
    dec = codec.decompress(data)
    assert _digest(dec, "<f8") == case["decoded"]
    assert float(np.abs(dec - POINTS.astype(np.float64)).max()) <= eb
