"""Batched path (chain_batch_*) against one-frame calls.

Frames of a batch run on several contexts from several host threads at once; every
frame's container must be byte-identical to a one-frame chain_compress of the same
frame, and every decoded frame identical to chain_decompress.  A failing frame reports
its own status without disturbing the others.
"""
import numpy as np
import pytest

from chaincompressor_b200 import _native as N
from chaincompressor_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _frames():
    """A small uneven batch: three content kinds, sizes 1e3..2e5, three error bounds,
    float32 and float64, SoA (D, N) arrays."""
    out = []
    for k, (n, kind, frac, seed) in enumerate(W.uneven_specs(count=14, seed=21, lo=1e3, hi=2e5)):
        pts = W.make_frame(n, kind, seed, np.float64 if k % 3 == 0 else np.float32)
        out.append((np.ascontiguousarray(pts.T), W.eb_for(pts, frac), 4, 2))
    return out


@pytest.fixture(scope="module")
def frames():
    return _frames()


def test_batch_compress_matches_single_calls(codec, frames):
    want = [codec.compress(pts, eb, p, t, layout=N.CHAIN_SOA) for pts, eb, p, t in frames]
    batch = N.Batch(0, workers=4)
    for _ in range(2):   # the second round reuses the warm worker contexts
        got = batch.compress(frames, layout=N.CHAIN_SOA)
        assert [len(g) for g in got] == [len(w) for w in want]
        for g, w in zip(got, want):
            assert g == w
    batch.close()


def test_batch_decompress_matches_single_calls(codec, frames):
    containers = [codec.compress(pts, eb, p, t, layout=N.CHAIN_SOA) for pts, eb, p, t in frames]
    batch = N.Batch(0, workers=3)
    for dtype, layout in ((np.float64, N.CHAIN_AOS), (np.float32, N.CHAIN_SOA)):
        got = batch.decompress(containers, dtype=dtype, layout=layout)
        for g, c in zip(got, containers):
            w = codec.decompress(c, dtype=dtype, layout=layout)
            assert g.shape == w.shape
            assert np.array_equal(g.view(np.uint8), w.view(np.uint8))
    batch.close()


def test_batch_reports_failing_frame(codec, frames):
    bad = list(frames[:5])
    pts = bad[2][0].copy()
    pts[0, 7] = np.nan
    bad[2] = (pts,) + bad[2][1:]
    batch = N.Batch(0, workers=2)
    with pytest.raises(N.ChainError) as ei:
        batch.compress(bad, layout=N.CHAIN_SOA)
    assert ei.value.status == N.CHAIN_ERR_NONFINITE_INPUT
    assert "frame 2" in str(ei.value)
    # the item array carries every frame's own status; the good frames' bytes are right
    items, outs = [], []
    for p_, eb, p, t in bad:
        cap = N.compress_bound(p_.shape[1], p_.shape[0])
        out = np.empty(cap, np.uint8)
        outs.append((p_, out))
        items.append(N.BatchItem(input=p_.ctypes.data, dtype=N.CHAIN_F32 if p_.dtype == np.float32 else N.CHAIN_F64,
                                 layout=N.CHAIN_SOA, n=p_.shape[1], dims=p_.shape[0], eb=eb, p=p, threshold=t,
                                 output=out.ctypes.data, output_capacity=cap))
    arr = (N.BatchItem * len(items))(*items)
    st = batch.L.chain_batch_compress(batch.h, arr, len(items), None)
    assert st == N.CHAIN_ERR_NONFINITE_INPUT
    assert [arr[i].status for i in range(5)] == [0, 0, N.CHAIN_ERR_NONFINITE_INPUT, 0, 0]
    for i in (0, 1, 3, 4):
        want = codec.compress(bad[i][0], *bad[i][1:], layout=N.CHAIN_SOA)
        assert outs[i][1][: arr[i].output_bytes].tobytes() == want
    batch.close()


def test_batch_small_output_buffer(codec, frames):
    pts, eb, p, t = frames[0]
    out = np.empty(16, np.uint8)
    item = N.BatchItem(input=pts.ctypes.data, dtype=N.CHAIN_F32 if pts.dtype == np.float32 else N.CHAIN_F64,
                       layout=N.CHAIN_SOA, n=pts.shape[1], dims=pts.shape[0], eb=eb, p=p, threshold=t,
                       output=out.ctypes.data, output_capacity=out.nbytes)
    batch = N.Batch(0, workers=1)
    arr = (N.BatchItem * 1)(item)
    st = batch.L.chain_batch_compress(batch.h, arr, 1, None)
    assert st == N.CHAIN_ERR_BUFFER_TOO_SMALL
    assert arr[0].output_bytes == len(codec.compress(pts, eb, p, t, layout=N.CHAIN_SOA))
    batch.close()


def test_many_small_frames_many_workers(codec):
    """Contexts used from several threads at once, on frames whose entropy tables (and so
    the shared memory of their rANS launches) differ widely."""
    frames = []
    rng = np.random.default_rng(23)
    for k in range(64):
        n = int(rng.integers(1000, 50_000))
        pts = W.make_frame(n, ("column", "blobs", "uniform")[k % 3], int(rng.integers(0, 2**31 - 1)))
        frames.append((np.ascontiguousarray(pts.T), W.eb_for(pts, float(10.0 ** -rng.integers(2, 6))), 4, 2))
    want = [codec.compress(pts, eb, p, t, layout=N.CHAIN_SOA) for pts, eb, p, t in frames]
    batch = N.Batch(0, workers=8)
    for _ in range(3):
        got = batch.compress(frames, layout=N.CHAIN_SOA)
        assert got == want
        dec = batch.decompress(got)
        for g, c in zip(dec, got):
            assert np.array_equal(g.view(np.uint64), codec.decompress(c).view(np.uint64))
    batch.close()


def test_tuned_batch_matches_single_calls_with_the_tuned_depth(codec, frames):
    """chain_batch_tune picks a lane depth and worker count from a sample; later batch
    calls without options use them, and each container is then byte-identical to a
    one-frame call with that lane depth."""
    batch = N.Batch(0, workers=4)
    r = batch.tune(frames[:6])
    assert r["rans_max_steps"] in (256, 512, 1024)
    assert 1 <= r["workers"] <= 4
    assert r["best_bytes"] <= 1.003 * r["default_bytes"]
    assert r["best_ms"] <= r["default_ms"]
    got = batch.compress(frames, layout=N.CHAIN_SOA)
    for (pts, eb, p, t), g in zip(frames, got):
        assert g == codec.compress(pts, eb, p, t, layout=N.CHAIN_SOA, rans_max_steps=r["rans_max_steps"])
    for g, d in zip(got, batch.decompress(got)):
        assert np.array_equal(d.view(np.uint64), codec.decompress(g).view(np.uint64))
    batch.close()
