"""LCG2 -> LCP2 transcoding, decoded by the reference's own CPU decoder.

For every parity case the GPU container is transcoded on the host; the reference serial
decoder (built from the reference sources into oracle/_ref) must return, bit for bit,
the points the GPU decoder returns for the original container.
"""
import numpy as np
import pytest

import oracle
from cases import GPU_CASES, case
from chaincompressor_b200 import _native as N

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU modules not built (oracle/_ref)")


@needs_ref
@pytest.mark.parametrize("name", GPU_CASES)
def test_reference_decoder_reads_transcoded_container(codec, name):
    pts, eb, p, t, kw = case(name)
    data = codec.compress(np.ascontiguousarray(pts.T), eb, p, t, layout=N.CHAIN_SOA, **kw)
    lcp2 = N.transcode_lcp2(data)
    assert lcp2[:4] == b"LCP2"
    got = oracle.ref_decompress(lcp2)
    want = codec.decompress(data)
    assert got.shape == want.shape
    assert np.array_equal(np.ascontiguousarray(got).view(np.uint64), want.view(np.uint64))


def test_transcode_rejects_bad_input(codec):
    pts, eb, p, t, kw = case("column")
    data = bytearray(codec.compress(np.ascontiguousarray(pts.T), eb, p, t, layout=N.CHAIN_SOA))
    data[-3] ^= 0xFF
    with pytest.raises(N.ChainError) as ei:
        N.transcode_lcp2(bytes(data))
    assert ei.value.status == N.CHAIN_ERR_CORRUPT_STREAM
