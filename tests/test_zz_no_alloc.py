"""chain_decompress_noalloc against chain_decompress, bit for bit.

The no-allocation entry point decodes with a fixed device array as its only working
memory; its output must equal chain_decompress's on the same container (the decoder
tests hold decoded values to bit equality), on consecutive calls that share that array.
The file name makes pytest collect it last, so it also runs after every other test in
one process; it needs nothing from them and passes alone as well.
"""
import ctypes

import numpy as np
import pytest

from chaincompressor_b200 import _native as N
from chaincompressor_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    return torch


@pytest.fixture(scope="module")
def frames(torch_cuda):
    """Two different frames compressed by chain_compress: (container bytes, n, dims)."""
    codec = N.Codec(0)
    out = []
    for pts, frac, p, t in ((W.blobs(200_000, seed=11), 1e-3, 4, 2),
                            (W.trajectory(0, n=60_000, seed=12), 1e-4, 2, 2)):
        eb = W.eb_for(pts, frac)
        data = codec.compress(np.ascontiguousarray(pts.T), eb, p, t, layout=N.CHAIN_SOA)
        out.append((data, pts.shape[0], pts.shape[1]))
    codec.close()
    return out


def _noalloc(src_ptr, length, out_ptr, capacity, dtype, layout, stream=0):
    """One call through the C ABI; returns (status, n, dims).  Every call, failing ones
    included, must leave the library's count of its own cudaMalloc / cudaMallocHost
    calls unchanged: the entry point's defining property."""
    L = N.load()
    n, d = ctypes.c_uint64(), ctypes.c_uint32()
    before = N.alloc_count()
    st = L.chain_decompress_noalloc(ctypes.c_void_p(src_ptr), length, dtype, layout, ctypes.c_void_p(out_ptr),
                                    capacity, ctypes.byref(n), ctypes.byref(d), ctypes.c_void_p(stream))
    assert N.alloc_count() == before, "chain_decompress_noalloc allocated memory"
    return st, n.value, d.value


def test_allocation_counter_sees_context_allocations(torch_cuda, frames):
    """The counter the no-allocation checks rely on does move when the library
    allocates (a fresh context's arenas and state on its first decode)."""
    data, n, d = frames[0]
    before = N.alloc_count()
    _existing(data, n, d, np.float64, N.CHAIN_AOS)
    assert N.alloc_count() > before


def _existing(data, n, d, dtype, layout):
    codec = N.Codec(0)
    want = codec.decompress(data, dtype=dtype, layout=layout)
    codec.close()
    return want


def test_two_calls_in_a_row_match_chain_decompress(torch_cuda, frames):
    torch = torch_cuda
    stream = torch.cuda.current_stream().cuda_stream
    # call 1: host container -> device float64 AoS output
    data, n, d = frames[0]
    want = _existing(data, n, d, np.float64, N.CHAIN_AOS)
    src = ctypes.create_string_buffer(data, len(data))
    dout = torch.full((n, d), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st, n1, d1 = _noalloc(ctypes.addressof(src), len(data), dout.data_ptr(), dout.numel() * 8, N.CHAIN_F64,
                          N.CHAIN_AOS, stream)
    assert st == N.CHAIN_OK, N.load().chain_last_error_message()
    assert (n1, d1) == (n, d)
    got = dout.cpu().numpy()
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    # call 2, straight after: device container (a different frame) -> host float32 SoA
    data, n, d = frames[1]
    want = _existing(data, n, d, np.float32, N.CHAIN_SOA)
    dsrc = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    hout = np.full((d, n), np.nan, np.float32)
    torch.cuda.synchronize()
    st, n2, d2 = _noalloc(dsrc.data_ptr(), len(data), hout.ctypes.data, hout.nbytes, N.CHAIN_F32, N.CHAIN_SOA, stream)
    assert st == N.CHAIN_OK, N.load().chain_last_error_message()
    assert (n2, d2) == (n, d)
    assert np.array_equal(hout.view(np.uint32), want.view(np.uint32))


def test_repeated_calls_are_identical(torch_cuda, frames):
    """The array keeps the previous call's contents; results must not depend on them."""
    data, n, d = frames[0]
    want = _existing(data, n, d, np.float64, N.CHAIN_SOA)
    src = ctypes.create_string_buffer(data, len(data))
    for _ in range(2):
        out = np.full((d, n), np.nan)
        st, _, _ = _noalloc(ctypes.addressof(src), len(data), out.ctypes.data, out.nbytes, N.CHAIN_F64, N.CHAIN_SOA)
        assert st == N.CHAIN_OK, N.load().chain_last_error_message()
        assert np.array_equal(out.view(np.uint64), want.view(np.uint64))


def test_rejects_frames_beyond_the_scratch(torch_cuda, frames):
    pts = W.blobs(2_000_000, seed=13)
    codec = N.Codec(0)
    data = codec.compress(np.ascontiguousarray(pts.T), W.eb_for(pts, 1e-3), 4, 2, layout=N.CHAIN_SOA)
    codec.close()
    src = ctypes.create_string_buffer(data, len(data))
    out = np.empty(pts.shape, np.float64)
    st, _, _ = _noalloc(ctypes.addressof(src), len(data), out.ctypes.data, out.nbytes, N.CHAIN_F64, N.CHAIN_AOS)
    assert st == N.CHAIN_ERR_UNSUPPORTED
    assert "too large for chain_decompress_noalloc" in N.load().chain_last_error_message().decode()
    # the entry point still works after a rejection
    data, n, d = frames[1]
    want = _existing(data, n, d, np.float64, N.CHAIN_AOS)
    src = ctypes.create_string_buffer(data, len(data))
    out = np.empty((n, d), np.float64)
    st, _, _ = _noalloc(ctypes.addressof(src), len(data), out.ctypes.data, out.nbytes, N.CHAIN_F64, N.CHAIN_AOS)
    assert st == N.CHAIN_OK, N.load().chain_last_error_message()
    assert np.array_equal(out.view(np.uint64), want.view(np.uint64))


def test_argument_errors(torch_cuda, frames):
    data, n, d = frames[0]
    src = ctypes.create_string_buffer(data, len(data))
    small = np.empty(8, np.float64)
    st, _, _ = _noalloc(ctypes.addressof(src), len(data), small.ctypes.data, small.nbytes, N.CHAIN_F64, N.CHAIN_AOS)
    assert st == N.CHAIN_ERR_BUFFER_TOO_SMALL
    st, _, _ = _noalloc(0, len(data), small.ctypes.data, small.nbytes, N.CHAIN_F64, N.CHAIN_AOS)
    assert st == N.CHAIN_ERR_INVALID_ARGUMENT
    bad = bytearray(data)
    bad[:4] = b"XXXX"
    bsrc = ctypes.create_string_buffer(bytes(bad), len(bad))
    out = np.empty((n, d), np.float64)
    st, _, _ = _noalloc(ctypes.addressof(bsrc), len(bad), out.ctypes.data, out.nbytes, N.CHAIN_F64, N.CHAIN_AOS)
    assert st == N.CHAIN_ERR_CORRUPT_STREAM
