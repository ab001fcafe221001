"""GPU parity: the CUDA path (through the C ABI) against the oracle, bit for bit.

For every case: the five integer streams the GPU encoder produced equal the oracle's
(the restatement of cpp/chain/lcps_cpp.cpp:2017-2250), the GPU decoder's float64
output equals the oracle decoder's bit for bit, max |err| <= eb, and the container is
within 1% of the reference CPU Chain's LCP2 size when the reference modules are built.
"""
import numpy as np
import pytest

import oracle
from cases import GPU_CASES, case
from chaincompressor_b200 import _native as N

pytestmark = pytest.mark.gpu


def _soa(pts):
    return np.ascontiguousarray(pts.T)


@pytest.mark.parametrize("name", GPU_CASES)
def test_streams_and_decode_bit_exact(codec, name):
    pts, eb, p, t, kw = case(name)
    n, d = pts.shape
    data = codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA, **kw)
    got = codec.debug_streams(n, d)
    want = oracle.streams(pts, eb, p, t, **kw)
    for k in ("idrel", "diff", "keep", "choice2", "rel"):
        assert got[k].shape == want[k].shape, (k, got[k].shape, want[k].shape)
        assert np.array_equal(got[k], want[k]), k
    dec = codec.decompress(data)
    ref_dec = oracle.decode(want)
    assert np.array_equal(dec.view(np.uint64), ref_dec.view(np.uint64))
    err = np.abs(dec - pts.astype(np.float64)).max()
    assert err <= eb
    # SoA float32 output is the float64 result rounded
    dec32 = codec.decompress(data, dtype=np.float32, layout=N.CHAIN_SOA)
    assert np.array_equal(dec32, ref_dec.T.astype(np.float32))


@pytest.mark.parametrize("name", ["column", "blobs200k", "traj_f64_e4_p1", "blobs_clipped", "uniform_p64_t25"])
def test_size_within_one_percent_of_reference(codec, name):
    if not oracle.ref_available():
        pytest.skip("reference CPU modules not built")
    pts, eb, p, t, kw = case(name)
    ours = codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA, **kw)
    ref = oracle.ref_compress(pts, eb, p, t, **kw)
    assert len(ours) <= 1.01 * len(ref), (len(ours), len(ref))


def test_aos_and_host_device_inputs_agree(codec):
    import torch
    pts, eb, p, t, _ = case("blobs200k")
    a = codec.compress(pts, eb, p, t, layout=N.CHAIN_AOS)
    b = codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA)
    dev = torch.from_numpy(_soa(pts)).cuda()
    c = codec.compress(dev, eb, p, t, layout=N.CHAIN_SOA)
    assert a == b == c


def test_deterministic(codec):
    pts, eb, p, t, _ = case("column")
    outs = {codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA) for _ in range(3)}
    assert len(outs) == 1


def test_errors(codec):
    pts, eb, p, t, _ = case("column")
    with pytest.raises(N.ChainError) as e:
        codec.compress(_soa(pts), -1.0, p, t, layout=N.CHAIN_SOA)
    assert e.value.status == N.CHAIN_ERR_INVALID_ARGUMENT
    with pytest.raises(N.ChainError) as e:
        codec.compress(_soa(pts), eb, 0, t, layout=N.CHAIN_SOA)
    assert e.value.status == N.CHAIN_ERR_INVALID_ARGUMENT
    bad = pts.copy()
    bad[17, 1] = np.nan
    with pytest.raises(N.ChainError) as e:
        codec.compress(_soa(bad), eb, p, t, layout=N.CHAIN_SOA)
    assert e.value.status == N.CHAIN_ERR_NONFINITE_INPUT
    # quantized values of 2^32 and more are beyond this build (below 2^32 they are coded)
    with pytest.raises(N.ChainError) as e:
        codec.compress(_soa(pts), float(np.max(pts.max(0) - pts.min(0))) * 1e-11, p, t, layout=N.CHAIN_SOA)
    assert e.value.status == N.CHAIN_ERR_UNSUPPORTED
    # the context stays usable after errors
    data = codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA)
    assert codec.decompress(data).shape == pts.shape


def test_corrupt_containers_are_rejected(codec):
    pts, eb, p, t, _ = case("column")
    data = bytearray(codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA))
    rng = np.random.default_rng(0)
    rejected = 0
    for trial in range(40):
        bad = bytearray(data)
        if trial % 4 == 0:
            bad = bad[: rng.integers(1, len(bad))]
        else:
            for _ in range(int(rng.integers(1, 6))):
                k = int(rng.integers(0, len(bad)))
                bad[k] ^= int(rng.integers(1, 256))
        try:
            out = codec.decompress(bytes(bad))
        except N.ChainError as e:
            assert e.status in (N.CHAIN_ERR_CORRUPT_STREAM, N.CHAIN_ERR_UNSUPPORTED, N.CHAIN_ERR_OUT_OF_MEMORY)
            rejected += 1
            continue
        assert out.shape[1] == pts.shape[1]
    assert rejected >= 20
    # still healthy
    assert np.array_equal(codec.decompress(bytes(data)), codec.decompress(bytes(data)))


def test_pybind_surface_matches_reference_api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from chaincompressor_b200 import chain_caller
    pts, eb, p, t, _ = case("column")
    data = chain_caller.chain_gpu(_soa(pts), eb, p, t, 0)
    assert isinstance(data, bytes) and data[:4] == b"LCG2"
    out = chain_caller.gpu_decompress(data)
    assert out.shape == pts.shape and out.dtype == np.float64
    assert np.abs(out - pts).max() <= eb
    soa = chain_caller.lcps_gpu_decompress_ans.lcps_decompress_gpu(data, output_soa=True)
    assert np.array_equal(soa, out.T)
    with pytest.raises(ValueError):
        chain_caller.chain_gpu(_soa(pts), 0.0, p, t, 0)


GOLDEN = sorted((__import__("pathlib").Path(__file__).parent / "golden").glob("*.npz"))


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_gpu_matches_reference_golden(codec, path):
    """GPU streams and decoded float64 coordinates equal the reference CPU Chain's
    (fixtures made from the reference modules by tests/golden/make_golden.py)."""
    g = np.load(path)
    pts = g["points"]
    kw = {"bl": bool(g["bl"]), "l1": bool(g["l1"]), "l2": bool(g["l2"])}
    n, d = pts.shape
    data = codec.compress(_soa(pts), float(g["eb"]), int(g["p"]), int(g["threshold"]), layout=N.CHAIN_SOA, **kw)
    got = codec.debug_streams(n, d)
    for k in ("idrel", "diff", "keep", "choice2", "rel"):
        assert np.array_equal(got[k], g[k]), k
    dec = codec.decompress(data)
    assert np.array_equal(dec.view(np.uint64), g["decoded"].view(np.uint64))


@pytest.mark.parametrize("name", ["column", "blobs200k", "traj_f64_e4_p1", "blobs_clipped", "uniform_p64_t25"])
def test_device_container_decodes_like_host_container(codec, name):
    """A container already in device memory is parsed on the device (the host copy is
    parsed on the host); both must give the same points, for device and host outputs."""
    import torch
    pts, eb, p, t, kw = case(name)
    data = codec.compress(_soa(pts), eb, p, t, layout=N.CHAIN_SOA, **kw)
    want = codec.decompress(data)
    n, d = want.shape
    dsrc = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    dout = torch.empty((n, d), dtype=torch.float64, device="cuda")
    assert codec.decompress_ptr(dsrc.data_ptr(), len(data), dout.data_ptr(), dout.numel() * 8) == (n, d)
    assert np.array_equal(dout.cpu().numpy().view(np.uint64), want.view(np.uint64))
    hout = np.empty((n, d), np.float64)
    codec.decompress_ptr(dsrc.data_ptr(), len(data), hout.ctypes.data, hout.nbytes)
    assert np.array_equal(hout.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_encoder_reproduces_committed_lcg2_fixture(codec, path):
    """The container of every golden input equals, byte for byte, the LCG2 fixture that
    tests/golden/make_lcg2.py committed (the CPU transcoder tests decode those files).
    This pins the whole encoder output (statistics, tables, chunking, layout) against
    silent changes; a deliberate format change regenerates the fixtures."""
    g = np.load(path)
    fixture = path.parent / "lcg2" / (path.stem + ".lcg2")
    kw = {"bl": bool(g["bl"]), "l1": bool(g["l1"]), "l2": bool(g["l2"])}
    data = codec.compress(_soa(g["points"]), float(g["eb"]), int(g["p"]), int(g["threshold"]), layout=N.CHAIN_SOA,
                          **kw)
    assert data == fixture.read_bytes()
