"""C ABI of libchain_b200 (CPU only: loading and exports, no device work)."""
import re
from pathlib import Path

import pytest

from chaincompressor_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "chain_b200.h").read_text()
    return sorted(set(re.findall(r"CHAIN_API\s+[\w\s\*]+?\b(chain_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "chain_compress" in syms and "chain_decompress" in syms
    assert set(syms) == set(N.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    for sym in declared_symbols():
        assert hasattr(lib, sym), sym


def test_pybind_modules_import():
    import importlib
    import sys

    pkg = str(ROOT / "chaincompressor_b200")
    if pkg not in sys.path:
        sys.path.insert(0, pkg)
    m1 = importlib.import_module("lcps_gpu_cpp")
    m2 = importlib.import_module("lcps_gpu_decompress_ans")
    assert hasattr(m1, "lcps_compress2_gpu") and hasattr(m2, "lcps_decompress_gpu")


def test_bound_is_monotone():
    assert N.compress_bound(1000, 3) < N.compress_bound(2000, 3)
    assert N.compress_bound(1 << 20, 3) > (1 << 20) * 3 * 4


def test_peek_rejects_garbage():
    with pytest.raises(N.ChainError) as e:
        N.peek(b"not a container at all")
    assert e.value.status == N.CHAIN_ERR_CORRUPT_STREAM


def test_context_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(N.ChainError) as e:
        N.Codec(0)
    assert e.value.status == N.CHAIN_ERR_DEVICE
