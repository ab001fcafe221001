"""Parity at full workload sizes.

The bench frame (16,777,216 float32 particles, 64 blobs + 20% uniform), the
4,194,304-particle float64 trajectory frames (frame 0 at eb = 1e-2, 1e-3 and 1e-4 x
range; frame 63, after 63 wrapped Gaussian steps have mixed the lattice, at 1e-3), and
a 4,194,304-particle clipped blob frame (points piled onto the box faces: the
exact-correction stress case) are compressed on the GPU; the five integer streams must
equal the oracle's bit for bit, the decoded float64 points must equal the oracle
decoder's bit for bit, and every point must lie within eb of its input.
"""
import numpy as np
import pytest

import oracle
from chaincompressor_b200 import _native as N
from chaincompressor_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _frames():
    pts = W.blobs(W.BLOBS_N, seed=1)
    yield "blobs16m", pts, W.eb_for(pts, 1e-3), 4, 2
    tr = W.trajectory(0, seed=2)
    yield "traj4m_f64_e4", tr, W.eb_for(tr, 1e-4), 4, 2
    yield "traj4m_f64_e3_p1", tr, W.eb_for(tr, 1e-3), 1, 2
    yield "traj4m_f64_e2", tr, W.eb_for(tr, 1e-2), 4, 2
    tr63 = W.trajectory(63, seed=2)
    yield "traj4m_f64_frame63_e3", tr63, W.eb_for(tr63, 1e-3), 4, 2
    cl = W.blobs(1 << 22, seed=5, clip=True)
    yield "blobs4m_clipped", cl, W.eb_for(cl, 1e-3), 4, 2


@pytest.mark.parametrize("frame", list(_frames()), ids=lambda f: f[0])
def test_full_size_bit_exact(codec, frame):
    name, pts, eb, p, t = frame
    n, d = pts.shape
    data = codec.compress(np.ascontiguousarray(pts.T), eb, p, t, layout=N.CHAIN_SOA)
    got = codec.debug_streams(n, d)
    want = oracle.streams(pts, eb, p, t)
    for k in ("idrel", "diff", "keep", "choice2", "rel"):
        assert got[k].shape == want[k].shape, (name, k)
        assert np.array_equal(got[k], want[k]), (name, k)
    dec = codec.decompress(data)
    ref = oracle.decode(want)
    assert np.array_equal(dec.view(np.uint64), ref.view(np.uint64)), name
    assert float(np.abs(dec - pts.astype(np.float64)).max()) <= eb
    if name == "blobs4m_clipped":
        assert want["exact_index"].size > 1000   # the stress case does exercise corrections
