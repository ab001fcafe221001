"""The oracle restatement against the reference CPU Chain (CPU only).

* golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
  reference modules): integer streams, exact corrections, wrap range, minima and the
  reference decoder's float64 output must match the restatement exactly;
* live, where the reference modules are built (oracle/_ref): more seeded cases.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = sorted((Path(__file__).parent / "golden").glob("*.npz"))
STREAMS = ("idrel", "diff", "keep", "choice2", "rel")


def test_golden_fixtures_exist():
    assert len(GOLDEN) >= 10


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_golden(path):
    g = np.load(path)
    kw = {"bl": bool(g["bl"]), "l1": bool(g["l1"]), "l2": bool(g["l2"])}
    s = oracle.streams(g["points"], float(g["eb"]), int(g["p"]), int(g["threshold"]), **kw)
    for k in STREAMS:
        assert s[k].shape == g[k].shape, k
        assert np.array_equal(s[k], g[k]), k
    assert s["wrap_min"] == int(g["wrap_min"]) and s["wrap_max"] == int(g["wrap_max"])
    assert s["p"] == int(g["p_eff"])
    assert np.array_equal(s["mins"].view(np.uint64), g["mins"].view(np.uint64))  # sign of zero included
    assert np.array_equal(s["exact_index"], g["exact_index"])
    assert np.array_equal(s["exact_value"].view(np.uint64), g["exact_value"].view(np.uint64))
    dec = oracle.decode(s)
    assert np.array_equal(dec.view(np.uint64), g["decoded"].view(np.uint64))
    pts = np.asarray(g["points"], np.float64)
    assert np.abs(dec - pts).max() <= float(g["eb"])


def test_decoder_rejects_corrupt_streams():
    g = np.load(GOLDEN[0])
    s = oracle.streams(g["points"], float(g["eb"]), int(g["p"]), int(g["threshold"]))
    bad = dict(s)
    bad["idrel"] = s["idrel"].copy()
    bad["idrel"][0, -1] = 5          # jumps past the end
    with pytest.raises(oracle.OracleError):
        oracle.decode_q(bad)
    bad = dict(s)
    bad["choice2"] = s["choice2"].copy()
    bad["choice2"][0, 0] = 1         # first record cannot be a difference
    with pytest.raises(oracle.OracleError):
        oracle.decode_q(bad)
    bad = dict(s)
    bad["rel"] = s["rel"].copy()
    bad["rel"][0, 0] = s["p"]        # offset must be < p
    with pytest.raises(oracle.OracleError):
        oracle.decode_q(bad)


def test_oracle_input_validation():
    pts = np.zeros((4, 3))
    with pytest.raises(oracle.OracleError):
        oracle.streams(pts, 0.0, 4, 2)
    bad = pts.copy()
    bad[1, 2] = np.inf
    with pytest.raises(oracle.OracleError):
        oracle.streams(bad, 0.1, 4, 2)


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference modules not built (make -C oracle ref)")


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_live(seed):
    from chaincompressor_b200 import workloads as W

    rng = np.random.default_rng(100 + seed)
    kind = ["column", "blobs", "uniform"][seed % 3]
    n = int(rng.integers(500, 20000))
    pts = W.make_frame(n, kind, int(rng.integers(0, 1 << 30)), np.float32 if seed % 2 else np.float64)
    eb = W.eb_for(pts, [1e-2, 1e-3, 1e-4][seed % 3])
    p = int(2 ** rng.integers(0, 7))
    t = int(rng.integers(-3, 8))
    data = oracle.ref_compress(pts, eb, p, t)
    rs = oracle.ref_streams(data)
    s = oracle.streams(pts, eb, p, t)
    for k in STREAMS:
        assert np.array_equal(np.asarray(rs[k]), s[k]), k
    assert np.array_equal(rs["exact_index"], s["exact_index"])
    dec = oracle.ref_decompress(data)
    assert np.array_equal(dec.view(np.uint64), oracle.decode(s).view(np.uint64))


@needs_ref
def test_dambreak_frame_if_present():
    """The reference's bundled DamBreak frame (only where the reference checkout exists)."""
    import xml.etree.ElementTree as ET

    files = sorted((oracle.reference_dir() / "data" / "DamBreak").glob("0654*.vtp"))
    if not files:
        pytest.skip("reference data not present")
    root = ET.parse(files[0]).getroot()
    arr = next(np.array(da.text.split(), np.float32) for da in root.iter("DataArray")
               if da.attrib.get("Name") == "Points").reshape(-1, 3)
    rng_ = float(np.max(arr.max(0).astype(np.float64) - arr.min(0)))
    eb = rng_ / (2 ** 11 - 2)   # reader.py equivalent_eb(maximum, qb - 1) for qb = 12
    data = oracle.ref_compress(arr, eb, 4, 25)
    rs = oracle.ref_streams(data)
    s = oracle.streams(arr, eb, 4, 25)
    for k in STREAMS:
        assert np.array_equal(np.asarray(rs[k]), s[k]), k


def _dambreak():
    import json

    g = np.load(Path(__file__).parent / "golden" / "dambreak" / "frame0654.npz")
    return g["points"], json.loads(str(g["cases"]))


_DB_POINTS, _DB_CASES = _dambreak()


@pytest.mark.parametrize("case", _DB_CASES, ids=[f"{c['table']}_qb{c['qb']}" for c in _DB_CASES])
def test_oracle_matches_dambreak_fixture(case):
    """The reference's DamBreak frame at the reader.py (p, threshold) tables: the
    restatement's streams, corrections and decoded output hash to what the reference
    encoder and decoder produced (tests/golden/make_dambreak.py)."""
    import hashlib

    def digest(a, dt="<i8"):
        return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=dt)).tobytes()).hexdigest()

    s = oracle.streams(_DB_POINTS, case["eb"], case["p"], case["threshold"])
    for k in STREAMS:
        assert list(s[k].shape) == case[k + "_shape"], k
        assert digest(s[k]) == case[k], k
    assert digest(s["exact_index"].astype(np.int64)) == case["exact_index"]
    assert digest(oracle.decode(s), "<f8") == case["decoded"]
