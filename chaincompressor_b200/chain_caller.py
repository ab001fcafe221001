"""The reference's Python API for the GPU path (chain_caller.py:33-40), B200-native.

    chain_gpu(coords, eb, p, threshold, diff)   coords: (D, N) SoA, float32 or float64
    gpu_decompress(compressed_data)             -> (N, D) float64

Both route through the pybind11 modules ``lcps_gpu_cpp`` and
``lcps_gpu_decompress_ans`` of this package, which call libchain_b200's C ABI.
There is no CPU fallback: importing this module on a machine without the built
extension raises ImportError.
"""
from __future__ import annotations

import sys
from pathlib import Path

_PKG = Path(__file__).resolve().parent
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))

import lcps_gpu_cpp  # noqa: E402  (in-tree pybind11 module)
import lcps_gpu_decompress_ans  # noqa: E402


def chain_gpu(coords, eb, p, threshold, diff=0, timer=False):
    """GPU compress of (D, N) coordinates (chain_caller.py:38-40)."""
    return lcps_gpu_cpp.lcps_compress2_gpu(coords, eb, p, threshold, diff)


def gpu_decompress(compressed_data, timer=False):
    """GPU decompress into (N, D) float64 coordinates (chain_caller.py:33-35)."""
    return lcps_gpu_decompress_ans.lcps_decompress_gpu(compressed_data)
