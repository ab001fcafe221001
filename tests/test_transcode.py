"""LCG2 -> LCP2 transcoding on the CPU (chain_transcode_lcp2 needs no GPU).

tests/golden/lcg2/*.lcg2 are GPU containers of the golden fixtures' inputs (made by
tests/golden/make_lcg2.py).  Each is transcoded here and decoded by the reference's own
serial decoder, which must return the fixture's stored reference output bit for bit:
the GPU encoder, the container and the transcoder together reproduce the reference.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from chaincompressor_b200 import _native as N

GOLD = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in (GOLD / "lcg2").glob("*.lcg2"))
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU modules not built (oracle/_ref)")


def test_fixtures_present():
    assert len(CASES) >= 10


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_reference_decodes_transcoded_fixture(name):
    z = np.load(GOLD / f"{name}.npz")
    lcp2 = N.transcode_lcp2((GOLD / "lcg2" / f"{name}.lcg2").read_bytes())
    got = np.ascontiguousarray(oracle.ref_decompress(lcp2))
    assert np.array_equal(got.view(np.uint64), z["decoded"].view(np.uint64))
    # the header carries the fixture's quantization parameters
    hdr = np.frombuffer(lcp2[:48], np.uint8)
    assert lcp2[:4] == b"LCP2"
    assert int(hdr[4:8].view(np.uint32)[0]) == z["points"].shape[1]
    assert int(hdr[8:16].view(np.uint64)[0]) == z["points"].shape[0]
    assert int(hdr[16:24].view(np.int64)[0]) == int(z["p_eff"])


@pytest.mark.parametrize("name", CASES[:3])
def test_transcode_errors(name):
    data = (GOLD / "lcg2" / f"{name}.lcg2").read_bytes()
    with pytest.raises(N.ChainError) as ei:
        N.transcode_lcp2(data[:-1])
    assert ei.value.status == N.CHAIN_ERR_CORRUPT_STREAM
    with pytest.raises(N.ChainError):
        N.transcode_lcp2(b"LCG1" + data[4:])
