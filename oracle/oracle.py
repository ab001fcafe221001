"""Python face of the Chain oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg import this
module; the product path never does.  It offers:

* ``streams(points, eb, p, threshold, ...)`` -- the project's C restatement
  (chain_oracle.c) of the reference CPU encoder's integer pipeline
  (cpp/chain/lcps_cpp.cpp:2017-2250): quantization, exact corrections, level-1
  chaining and the level-2 keep/difference split.
* ``decode(streams)`` -- the restated inverse (lcps_cpp.cpp:1890-1993).
* ``ref()`` -- the reference's own CPU modules compiled from its sources into
  oracle/_ref (lcps_cpp, lcps_cpu_decompress, lcps_ref_streams), when present.
"""
from __future__ import annotations

import contextlib
import ctypes
import importlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
_LIB = None


def reference_dir() -> Path:
    """The reference checkout the recipe in oracle/Makefile compiles from:
    $CHAIN_REFERENCE_DIR when set, else the Makefile's default (``make print-ref``)."""
    env = os.environ.get("CHAIN_REFERENCE_DIR")
    if env:
        return Path(env)
    r = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref"], capture_output=True, text=True)
    return Path(r.stdout.strip())


def build_own() -> Path:
    so = HERE / "libchain_oracle.so"
    src = [HERE / "chain_oracle.c", HERE / "chain_oracle.h"]
    if not so.exists() or any(s.stat().st_mtime > so.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE), "own"], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = build_own()
        L = ctypes.CDLL(str(so))
        P = ctypes.c_void_p
        u64, u32, i64, dbl, i32 = (ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int64,
                                   ctypes.c_double, ctypes.c_int)
        L.co_quantize.argtypes = [P, u64, u32, dbl, i64, P, P, P, P, P, P, P]
        L.co_level1.argtypes = [P, u64, u32, i64, i32, i64, P, P, P]
        L.co_level2.argtypes = [P, u64, u64, u32, i32, P, P, P, P, P, u64, P]
        L.co_decode_q.argtypes = [u64, u32, i64, i64, i64, P, P, u64, P, u64, P, u64, P, P]
        L.co_reconstruct.argtypes = [u64, u32, P, P, dbl, P, P, u64, P]
        for f in ("co_quantize", "co_level1", "co_level2", "co_decode_q", "co_reconstruct"):
            getattr(L, f).restype = ctypes.c_int
        _LIB = L
    return _LIB


class OracleError(RuntimeError):
    pass


class _Wrap(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in
                ("min_value", "max_value", "max_difference", "min_correction", "max_correction")]


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def streams(points, eb: float, p: int, threshold: int, bl: bool = True, l1: bool = True,
            l2: bool = True) -> dict:
    """Integer streams of the reference CPU encoder for (N, D) points."""
    pts = np.ascontiguousarray(np.asarray(points), dtype=np.float64)
    if pts.ndim != 2:
        raise ValueError("points must be (N, D)")
    n, dims = pts.shape
    p_eff = int(p) if bl else 1
    L = lib()
    mins = np.empty(dims, np.float64)
    bid = np.empty((dims, n), np.int64)
    rel = np.empty((dims, n), np.int64)
    cidx = np.empty(n * dims, np.uint64)
    cval = np.empty(n * dims, np.float64)
    ncorr = ctypes.c_uint64()
    maxb = ctypes.c_int64()
    st = L.co_quantize(_p(pts), n, dims, float(eb), p_eff, _p(mins), _p(bid), _p(rel), _p(cidx),
                       _p(cval), ctypes.byref(ncorr), ctypes.byref(maxb))
    if st:
        raise OracleError(f"co_quantize status {st}")
    idrel = np.empty(n, np.int64)
    blocks = np.empty((dims, n), np.int64)
    nb = ctypes.c_uint64()
    st = L.co_level1(_p(bid), n, dims, int(threshold), int(bool(l1)), maxb.value, _p(idrel),
                     _p(blocks), ctypes.byref(nb))
    if st:
        raise OracleError(f"co_level1 status {st}")
    B = nb.value
    choice2 = np.empty(B, np.int64)
    keep = np.empty((dims, max(B, 1)), np.int64)
    diff = np.empty((dims, max(B, 1)), np.int64)
    nk, nd = ctypes.c_uint64(), ctypes.c_uint64()
    w = _Wrap()
    st = L.co_level2(_p(blocks), B, n, dims, int(bool(l2)), _p(choice2), _p(keep), ctypes.byref(nk),
                     _p(diff), ctypes.byref(nd), max(B, 1), ctypes.byref(w))
    if st:
        raise OracleError(f"co_level2 status {st}")
    k, dd = nk.value, nd.value
    return {
        "n": n, "dims": dims, "p": p_eff, "eb": float(eb), "mins": mins,
        "idrel": idrel.reshape(1, n), "diff": np.ascontiguousarray(diff[:, :dd]),
        "keep": np.ascontiguousarray(keep[:, :k]), "choice2": choice2.reshape(1, B),
        "rel": rel, "bid": bid, "wrap_min": w.min_value, "wrap_max": w.max_value,
        "exact_index": cidx[: ncorr.value].copy(), "exact_value": cval[: ncorr.value].copy(),
        "max_bid": maxb.value,
    }


def decode_q(s: dict) -> np.ndarray:
    """Quantized integers (D, N) from the five streams (lcps_cpp.cpp:1890-1961)."""
    n, dims = int(s["n"]), int(s["dims"])
    idrel = np.ascontiguousarray(s["idrel"], np.int64).reshape(-1)
    diff = np.ascontiguousarray(s["diff"], np.int64)
    keep = np.ascontiguousarray(s["keep"], np.int64)
    choice2 = np.ascontiguousarray(s["choice2"], np.int64).reshape(-1)
    rel = np.ascontiguousarray(s["rel"], np.int64)
    q = np.empty((dims, n), np.int64)
    st = lib().co_decode_q(n, dims, int(s["p"]), int(s["wrap_min"]), int(s["wrap_max"]), _p(idrel),
                           _p(diff), diff.shape[1] if diff.ndim == 2 else 0, _p(keep),
                           keep.shape[1] if keep.ndim == 2 else 0, _p(choice2), choice2.size,
                           _p(rel), _p(q))
    if st:
        raise OracleError(f"co_decode_q status {st}")
    return q


def decode(s: dict) -> np.ndarray:
    """Float64 (N, D) coordinates from the five streams plus corrections."""
    q = decode_q(s)
    n, dims = int(s["n"]), int(s["dims"])
    mins = np.ascontiguousarray(s["mins"], np.float64)
    cidx = np.ascontiguousarray(s["exact_index"], np.uint64)
    cval = np.ascontiguousarray(s["exact_value"], np.float64)
    out = np.empty((n, dims), np.float64)
    st = lib().co_reconstruct(n, dims, _p(q), _p(mins), float(s["eb"]), _p(cidx), _p(cval),
                              cidx.size, _p(out))
    if st:
        raise OracleError(f"co_reconstruct status {st}")
    return out


def quantized(points, eb: float) -> np.ndarray:
    """q = floor((x - min) / (2 eb)) per value, (D, N) int64 (lcps_cpp.cpp:2091-2096)."""
    s = streams(points, eb, 1, 0, bl=False, l1=False, l2=False)
    return s["bid"]


# ---------------------------------------------------------------- reference modules
def ref_available() -> bool:
    return all((REF_DIR / f"{m}.so").exists() for m in
               ("lcps_cpp", "lcps_cpu_decompress", "lcps_ref_streams"))


def ref(module: str):
    """Import one of the reference CPU modules built into oracle/_ref."""
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    return importlib.import_module(module)


@contextlib.contextmanager
def quiet_stdout():
    """The reference CPU modules print stage times and codec names on every call."""
    sys.stdout.flush()
    saved = os.dup(1)
    with open(os.devnull, "wb") as devnull:
        os.dup2(devnull.fileno(), 1)
    try:
        yield
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def ref_compress(points, eb, p, threshold, bl=True, l1=True, l2=True, ec=True):
    """Reference CPU encoder (chain_caller.chain): returns the LCP2 bytes."""
    m = ref("lcps_cpp")
    with quiet_stdout():
        out = m.lcps_compress2(np.asarray(points), float(eb), int(p), int(threshold), 0,
                               bl, l1, l2, ec)
    return out[0]


def ref_decompress(data: bytes) -> np.ndarray:
    """Reference serial CPU decoder (chain_caller.chain_decompress)."""
    m = ref("lcps_cpu_decompress")
    with quiet_stdout():
        return m.lcps_decompress_serial(data)


def ref_streams(data: bytes) -> dict:
    return ref("lcps_ref_streams").decode_streams(data)
