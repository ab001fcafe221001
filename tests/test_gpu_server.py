"""Request server (chain_server_*): mixed concurrent requests against requests run alone.

Requests of a mix run on several resident contexts at once, admitted under a memory
budget; each result must equal the same request served alone by a one-frame call
(containers byte for byte, decoded values bit for bit).
"""
import numpy as np
import pytest

from chaincompressor_b200 import _native as N
from chaincompressor_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _requests(codec):
    """Seeded mix: compress requests (float32 and float64, three content kinds) and
    decompress requests of containers made alone beforehand."""
    rng = np.random.default_rng(41)
    reqs = []
    for k, (n, kind, frac, seed) in enumerate(W.uneven_specs(count=24, seed=42, lo=1e3, hi=3e5)):
        pts = W.make_frame(n, kind, seed, np.float64 if k % 3 == 1 else np.float32)
        soa = np.ascontiguousarray(pts.T)
        eb = W.eb_for(pts, frac)
        if rng.random() < 0.5:
            want = codec.compress(soa, eb, 4, 2, layout=N.CHAIN_SOA)
            out = np.zeros(N.compress_bound(n, 3), np.uint8)
            item = N.BatchItem(input=soa.ctypes.data, dtype=N.CHAIN_F32 if soa.dtype == np.float32 else N.CHAIN_F64,
                               layout=N.CHAIN_SOA, n=n, dims=3, eb=eb, p=4, threshold=2, output=out.ctypes.data,
                               output_capacity=out.nbytes)
            reqs.append((N.Server.COMPRESS, item, (soa, out), want))
        else:
            data = codec.compress(soa, eb, 4, 2, layout=N.CHAIN_SOA)
            want = codec.decompress(data)
            src = np.frombuffer(data, np.uint8).copy()
            out = np.zeros((n, 3), np.float64)
            item = N.BatchItem(input=src.ctypes.data, input_bytes=src.nbytes, dtype=N.CHAIN_F64, layout=N.CHAIN_AOS,
                               output=out.ctypes.data, output_capacity=out.nbytes)
            reqs.append((N.Server.DECOMPRESS, item, (src, out), want))
    return reqs


def _check(op, item, bufs, want):
    out = bufs[1]
    if op == N.Server.COMPRESS:
        assert out[: item.output_bytes].tobytes() == want
    else:
        assert np.array_equal(out.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("budget", [40 << 30, 64 << 20])
def test_mix_equals_alone(codec, budget):
    reqs = _requests(codec)
    srv = N.Server(0, workers=4, memory_budget_bytes=budget)   # 64 MiB: admission gates most requests
    tickets = [srv.submit(op, item) for op, item, _, _ in reqs]
    for t, (op, item, bufs, want) in zip(tickets, reqs):
        st, q_ms, s_ms, _ = srv.wait(t)
        assert st == N.CHAIN_OK and q_ms >= 0 and s_ms > 0
        _check(op, item, bufs, want)
    srv.close()


def test_failing_request_does_not_disturb_others(codec):
    reqs = _requests(codec)[:8]
    bad = np.frombuffer(b"LCG2" + bytes(200), np.uint8).copy()
    out = np.zeros(64, np.float64)
    bad_item = N.BatchItem(input=bad.ctypes.data, input_bytes=bad.nbytes, dtype=N.CHAIN_F64, layout=N.CHAIN_AOS,
                           output=out.ctypes.data, output_capacity=out.nbytes)
    srv = N.Server(0, workers=3)
    tickets = [srv.submit(op, item) for op, item, _, _ in reqs[:4]]
    tb = srv.submit(N.Server.DECOMPRESS, bad_item)
    tickets += [srv.submit(op, item) for op, item, _, _ in reqs[4:]]
    st, _, _, _ = srv.wait(tb, check=False)
    assert st == N.CHAIN_ERR_CORRUPT_STREAM
    for t, (op, item, bufs, want) in zip(tickets, reqs):
        srv.wait(t)
        _check(op, item, bufs, want)
    srv.close()


def test_destroy_finishes_queued_requests(codec):
    """chain_server_destroy right after the submits, with most requests still queued on
    the single worker: every request still runs to completion, with the same result as
    alone (the items carry status and output)."""
    reqs = _requests(codec)[:12]
    srv = N.Server(0, workers=1, memory_budget_bytes=40 << 30)
    for op, item, _, _ in reqs:
        srv.submit(op, item)
    srv.close()
    for op, item, bufs, want in reqs:
        assert item.status == N.CHAIN_OK
        _check(op, item, bufs, want)


def test_destroy_releases_a_blocked_waiter(codec):
    """A thread blocked in chain_server_wait when destroy begins is released with its
    request's status, and destroy returns only after it has left the call."""
    import ctypes
    import threading
    import time

    reqs = _requests(codec)[:4]
    srv = N.Server(0, workers=1, memory_budget_bytes=40 << 30)
    tickets = [srv.submit(op, item) for op, item, _, _ in reqs]
    h = srv.h
    got = []

    def waiter():
        got.append(srv.L.chain_server_wait(h, ctypes.c_uint64(tickets[-1]), None, None))

    th = threading.Thread(target=waiter)
    th.start()
    time.sleep(0.5)            # the waiter is inside chain_server_wait by now
    srv.h = None
    srv.L.chain_server_destroy(h)
    th.join(timeout=120)
    assert not th.is_alive()
    assert got == [N.CHAIN_OK]
    op, item, bufs, want = reqs[-1]
    _check(op, item, bufs, want)
