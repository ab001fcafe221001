"""chaincompressor_b200: B200-native (sm_100a) Chain compressor hot path.

Order-preserving, error-bounded lossy compression of particle coordinates with the
integer semantics of the reference CPU Chain encoder, on hand-written CUDA kernels.

* ``chaincompressor_b200.chain_caller`` -- the reference's Python API for the GPU
  path (chain_gpu / gpu_decompress) over the pybind11 modules.
* ``chaincompressor_b200._native.Codec`` -- ctypes binding of the C ABI
  (include/chain_b200.h) with host or device buffers.
* ``chaincompressor_b200.workloads`` -- seeded synthetic frames.
"""
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
__all__ = ["PKG_DIR"]
