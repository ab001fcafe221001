"""ctypes binding of the C ABI in include/chain_b200.h (libchain_b200.so).

This is the reference-facing boundary the tests and bench.py drive: plain pointers
and sizes, host or device buffers.  The library is loaded from this package
directory; a missing or stale build raises instead of falling back to anything.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libchain_b200.so"

CHAIN_OK = 0
CHAIN_ERR_INVALID_ARGUMENT = 1
CHAIN_ERR_NONFINITE_INPUT = 2
CHAIN_ERR_QUANT_OVERFLOW = 3
CHAIN_ERR_CORRUPT_STREAM = 4
CHAIN_ERR_DEVICE = 5
CHAIN_ERR_OUT_OF_MEMORY = 6
CHAIN_ERR_UNSUPPORTED = 7
CHAIN_ERR_BUFFER_TOO_SMALL = 8
CHAIN_F32, CHAIN_F64 = 4, 8
CHAIN_SOA, CHAIN_AOS = 0, 1

# Every entry point declared in include/chain_b200.h.
EXPORTS = ("chain_ctx_create", "chain_ctx_destroy", "chain_last_error_message", "chain_compress_bound",
           "chain_compress", "chain_result_copy", "chain_result_device_ptr", "chain_peek", "chain_decompress",
           "chain_debug_streams", "chain_set_stage_timing", "chain_stage_times", "chain_launch_count",
           "chain_alloc_count", "chain_decompress_noalloc", "chain_batch_create", "chain_batch_destroy", "chain_batch_compress",
           "chain_batch_decompress", "chain_batch_tune", "chain_server_create", "chain_server_destroy", "chain_server_submit",
           "chain_server_wait", "chain_transcode_lcp2")


class ChainError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class ChainOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("bl", ctypes.c_int32), ("l1", ctypes.c_int32),
                ("l2", ctypes.c_int32), ("rans_bytes_per_lane", ctypes.c_uint32),
                ("rans_max_steps", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 10)]


class TuneResult(ctypes.Structure):
    _fields_ = [("rans_max_steps", ctypes.c_uint32), ("workers", ctypes.c_uint32), ("best_ms", ctypes.c_double),
                ("default_ms", ctypes.c_double), ("best_bytes", ctypes.c_uint64), ("default_bytes", ctypes.c_uint64)]


class BatchItem(ctypes.Structure):
    _fields_ = [("input", ctypes.c_void_p), ("input_bytes", ctypes.c_size_t), ("dtype", ctypes.c_int),
                ("layout", ctypes.c_int), ("n", ctypes.c_uint64), ("dims", ctypes.c_uint32), ("eb", ctypes.c_double),
                ("p", ctypes.c_int64), ("threshold", ctypes.c_int64), ("output", ctypes.c_void_p),
                ("output_capacity", ctypes.c_size_t), ("output_bytes", ctypes.c_size_t), ("status", ctypes.c_int)]


_LIB = None


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m chaincompressor_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        P, u64, u32, i64, dbl, i32, sz = (ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int64,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_size_t)
        L.chain_ctx_create.argtypes = [i32, P, ctypes.POINTER(P)]
        L.chain_ctx_destroy.argtypes = [P]
        L.chain_ctx_destroy.restype = None
        L.chain_last_error_message.restype = ctypes.c_char_p
        L.chain_compress_bound.argtypes = [u64, u32]
        L.chain_compress_bound.restype = sz
        L.chain_compress.argtypes = [P, P, i32, i32, u64, u32, dbl, i64, i64, ctypes.POINTER(ChainOpts),
                                     ctypes.POINTER(sz)]
        L.chain_result_copy.argtypes = [P, P, sz]
        L.chain_result_device_ptr.argtypes = [P]
        L.chain_result_device_ptr.restype = P
        L.chain_peek.argtypes = [P, sz, ctypes.POINTER(u64), ctypes.POINTER(u32), ctypes.POINTER(i32)]
        L.chain_decompress.argtypes = [P, P, sz, i32, i32, P, sz, ctypes.POINTER(u64), ctypes.POINTER(u32)]
        L.chain_debug_streams.argtypes = [P, P, P, ctypes.POINTER(u64), P, ctypes.POINTER(u64), P,
                                          ctypes.POINTER(u64), P]
        L.chain_decompress_noalloc.argtypes = [P, sz, i32, i32, P, sz, ctypes.POINTER(u64), ctypes.POINTER(u32), P]
        L.chain_batch_create.argtypes = [i32, i32, ctypes.POINTER(P)]
        L.chain_batch_destroy.argtypes = [P]
        L.chain_batch_destroy.restype = None
        L.chain_batch_compress.argtypes = [P, ctypes.POINTER(BatchItem), sz, ctypes.POINTER(ChainOpts)]
        L.chain_batch_decompress.argtypes = [P, ctypes.POINTER(BatchItem), sz]
        L.chain_batch_tune.argtypes = [P, ctypes.POINTER(BatchItem), sz, ctypes.POINTER(TuneResult)]
        L.chain_server_create.argtypes = [i32, i32, sz, ctypes.POINTER(ChainOpts), ctypes.POINTER(P)]
        L.chain_server_destroy.argtypes = [P]
        L.chain_server_destroy.restype = None
        L.chain_server_submit.argtypes = [P, i32, ctypes.POINTER(BatchItem), ctypes.POINTER(u64)]
        L.chain_server_wait.argtypes = [P, u64, ctypes.POINTER(dbl), ctypes.POINTER(dbl)]
        L.chain_transcode_lcp2.argtypes = [P, sz, P, sz, ctypes.POINTER(sz)]
        for f in ("chain_ctx_create", "chain_compress", "chain_result_copy", "chain_peek", "chain_decompress",
                  "chain_debug_streams", "chain_set_stage_timing", "chain_stage_times", "chain_decompress_noalloc",
                  "chain_batch_create", "chain_batch_compress", "chain_batch_decompress", "chain_batch_tune",
                  "chain_server_create",
                  "chain_server_submit", "chain_server_wait", "chain_transcode_lcp2"):
            getattr(L, f).restype = ctypes.c_int
        L.chain_launch_count.restype = ctypes.c_uint64
        L.chain_alloc_count.restype = ctypes.c_uint64
        _LIB = L
    return _LIB


def _check(st: int):
    if st != CHAIN_OK:
        raise ChainError(st, load().chain_last_error_message().decode())


def _ptr(x) -> int:
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):  # torch tensor (host or device)
        return x.data_ptr()
    if isinstance(x, (bytes, bytearray)):
        return ctypes.cast(ctypes.c_char_p(bytes(x)), ctypes.c_void_p).value
    return int(x)


class Codec:
    """One library context (device arena + stream) on one CUDA device."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.L = load()
        h = ctypes.c_void_p()
        _check(self.L.chain_ctx_create(device, ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.chain_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- compress
    def compress_ptr(self, ptr: int, dtype: int, layout: int, n: int, dims: int, eb: float, p: int,
                     threshold: int, bl=True, l1=True, l2=True, rans_bytes_per_lane: int = 0,
                     rans_max_steps: int = 0) -> int:
        o = ChainOpts()
        o.struct_size = ctypes.sizeof(ChainOpts)
        o.bl, o.l1, o.l2 = int(bl), int(l1), int(l2)
        o.rans_bytes_per_lane = rans_bytes_per_lane
        o.rans_max_steps = rans_max_steps
        out_len = ctypes.c_size_t()
        _check(self.L.chain_compress(self.h, ctypes.c_void_p(ptr), dtype, layout, n, dims, float(eb), int(p),
                                     int(threshold), ctypes.byref(o), ctypes.byref(out_len)))
        return out_len.value

    def compress(self, points, eb: float, p: int, threshold: int, layout: int = CHAIN_AOS, **kw) -> bytes:
        """points: numpy (N, D) [AOS] or (D, N) [SOA] float32/float64, or a torch tensor."""
        dt = str(points.dtype).replace("torch.", "")
        if dt not in ("float32", "float64"):
            raise ValueError("points must be float32 or float64")
        if isinstance(points, np.ndarray):
            points = np.ascontiguousarray(points)
        shape = tuple(points.shape)
        n, dims = (shape[0], shape[1]) if layout == CHAIN_AOS else (shape[1], shape[0])
        ln = self.compress_ptr(_ptr(points), CHAIN_F32 if dt == "float32" else CHAIN_F64, layout, n, dims, eb, p,
                               threshold, **kw)
        out = bytearray(ln)
        buf = (ctypes.c_char * ln).from_buffer(out)
        _check(self.L.chain_result_copy(self.h, ctypes.addressof(buf), ln))
        return bytes(out)

    def result_copy_to(self, dst_ptr: int, capacity: int):
        _check(self.L.chain_result_copy(self.h, ctypes.c_void_p(dst_ptr), capacity))

    def result_device_ptr(self) -> int:
        return self.L.chain_result_device_ptr(self.h) or 0

    def debug_streams(self, n: int, dims: int) -> dict:
        nd_, nk_, nb_ = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(self.L.chain_debug_streams(self.h, None, None, ctypes.byref(nd_), None, ctypes.byref(nk_), None,
                                          ctypes.byref(nb_), None))
        idrel = np.empty(n, np.int64)
        diff = np.empty(max(1, nd_.value * dims), np.int64)
        keep = np.empty(max(1, nk_.value * dims), np.int64)
        choice2 = np.empty(max(1, nb_.value), np.int64)
        rel = np.empty(n * dims, np.int64)
        _check(self.L.chain_debug_streams(self.h, idrel.ctypes.data, diff.ctypes.data, ctypes.byref(nd_),
                                          keep.ctypes.data, ctypes.byref(nk_), choice2.ctypes.data,
                                          ctypes.byref(nb_), rel.ctypes.data))
        return {
            "idrel": idrel.reshape(1, n),
            "diff": diff[: nd_.value * dims].reshape(nd_.value, dims).T.copy(),
            "keep": keep[: nk_.value * dims].reshape(nk_.value, dims).T.copy(),
            "choice2": choice2[: nb_.value].reshape(1, nb_.value),
            "rel": rel.reshape(n, dims).T.copy(),
        }

    def set_stage_timing(self, enabled: bool):
        _check(self.L.chain_set_stage_timing(self.h, int(bool(enabled))))

    def stage_times(self) -> list:
        """[(stage, ms)] of the last call (stage timing must be enabled)."""
        names = (ctypes.c_char_p * 64)()
        ms = (ctypes.c_float * 64)()
        k = self.L.chain_stage_times(self.h, names, ms, 64)
        return [(names[i].decode(), float(ms[i])) for i in range(k)]

    # ------------------------------------------------------------ decompress
    def decompress_ptr(self, src_ptr: int, length: int, out_ptr: int, capacity: int, dtype: int = CHAIN_F64,
                       layout: int = CHAIN_AOS):
        n, d = ctypes.c_uint64(), ctypes.c_uint32()
        _check(self.L.chain_decompress(self.h, ctypes.c_void_p(src_ptr), length, dtype, layout,
                                       ctypes.c_void_p(out_ptr), capacity, ctypes.byref(n), ctypes.byref(d)))
        return n.value, d.value

    def decompress(self, data: bytes, dtype=np.float64, layout: int = CHAIN_AOS) -> np.ndarray:
        n, d, _ = peek(data)
        out = np.empty((n, d) if layout == CHAIN_AOS else (d, n), dtype)
        src = ctypes.create_string_buffer(data, len(data))
        self.decompress_ptr(ctypes.addressof(src), len(data), out.ctypes.data, out.nbytes,
                            CHAIN_F64 if out.dtype == np.float64 else CHAIN_F32, layout)
        return out


def peek(data: bytes):
    L = load()
    n, d, t = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_int()
    src = ctypes.create_string_buffer(data, len(data))
    _check(L.chain_peek(ctypes.addressof(src), len(data), ctypes.byref(n), ctypes.byref(d), ctypes.byref(t)))
    return n.value, d.value, t.value


def decompress_noalloc_ptr(src_ptr: int, length: int, out_ptr: int, capacity: int, dtype: int = CHAIN_F64,
                           layout: int = CHAIN_AOS, stream: int = 0):
    """chain_decompress_noalloc on the current CUDA device: no context, no allocation."""
    L = load()
    n, d = ctypes.c_uint64(), ctypes.c_uint32()
    _check(L.chain_decompress_noalloc(ctypes.c_void_p(src_ptr), length, dtype, layout, ctypes.c_void_p(out_ptr),
                                      capacity, ctypes.byref(n), ctypes.byref(d), ctypes.c_void_p(stream)))
    return n.value, d.value


class Batch:
    """chain_batch: `workers` contexts on one device, driven by host threads."""

    def __init__(self, device: int = 0, workers: int = 4):
        self.L = load()
        h = ctypes.c_void_p()
        _check(self.L.chain_batch_create(device, workers, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.chain_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compress_items(self, items, opts: ChainOpts | None = None):
        arr = (BatchItem * len(items))(*items)
        _check(self.L.chain_batch_compress(self.h, arr, len(items), ctypes.byref(opts) if opts else None))
        return arr

    def decompress_items(self, items):
        arr = (BatchItem * len(items))(*items)
        _check(self.L.chain_batch_decompress(self.h, arr, len(items)))
        return arr

    def tune_items(self, items) -> dict:
        """chain_batch_tune on compress items (their outputs are overwritten)."""
        arr = (BatchItem * len(items))(*items)
        r = TuneResult()
        _check(self.L.chain_batch_tune(self.h, arr, len(items), ctypes.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def tune(self, frames, layout: int = CHAIN_SOA) -> dict:
        """chain_batch_tune on a sample of frames (the compress() form)."""
        keep, items = [], []
        for pts, eb, p, t in frames:
            pts = np.ascontiguousarray(pts)
            n, d = (pts.shape[1], pts.shape[0]) if layout == CHAIN_SOA else pts.shape
            cap = compress_bound(n, d)
            out = np.empty(cap, np.uint8)
            keep.append((pts, out))
            items.append(BatchItem(input=pts.ctypes.data, dtype=CHAIN_F32 if pts.dtype == np.float32 else CHAIN_F64,
                                   layout=layout, n=n, dims=d, eb=float(eb), p=int(p), threshold=int(t),
                                   output=out.ctypes.data, output_capacity=cap))
        return self.tune_items(items)

    def compress(self, frames, layout: int = CHAIN_SOA) -> list[bytes]:
        """frames: list of (points, eb, p, threshold) with numpy points ((D, N) for SoA)."""
        keep, items, outs = [], [], []
        for pts, eb, p, t in frames:
            pts = np.ascontiguousarray(pts)
            n, d = (pts.shape[1], pts.shape[0]) if layout == CHAIN_SOA else pts.shape
            cap = compress_bound(n, d)
            out = np.empty(cap, np.uint8)
            keep.append(pts)
            outs.append(out)
            items.append(BatchItem(input=pts.ctypes.data, dtype=CHAIN_F32 if pts.dtype == np.float32 else CHAIN_F64,
                                   layout=layout, n=n, dims=d, eb=float(eb), p=int(p), threshold=int(t),
                                   output=out.ctypes.data, output_capacity=cap))
        arr = self.compress_items(items)
        return [outs[i][: arr[i].output_bytes].tobytes() for i in range(len(items))]

    def decompress(self, containers, dtype=np.float64, layout: int = CHAIN_AOS) -> list[np.ndarray]:
        keep, items, outs = [], [], []
        for data in containers:
            n, d, _ = peek(data)
            out = np.empty((n, d) if layout == CHAIN_AOS else (d, n), dtype)
            src = np.frombuffer(data, np.uint8)
            keep.append(src)
            outs.append(out)
            items.append(BatchItem(input=src.ctypes.data, input_bytes=len(data),
                                   dtype=CHAIN_F64 if out.dtype == np.float64 else CHAIN_F32, layout=layout,
                                   output=out.ctypes.data, output_capacity=out.nbytes))
        self.decompress_items(items)
        return outs


class Server:
    """chain_server: FIFO admission of compress (op 0) / decompress (op 1) requests onto
    `workers` resident contexts under a device-memory budget."""

    COMPRESS, DECOMPRESS = 0, 1

    def __init__(self, device: int = 0, workers: int = 8, memory_budget_bytes: int = 40 << 30):
        self.L = load()
        h = ctypes.c_void_p()
        _check(self.L.chain_server_create(device, workers, memory_budget_bytes, None, ctypes.byref(h)))
        self.h = h
        self._items = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.chain_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, op: int, item: BatchItem) -> int:
        """The item (and the buffers it points to) must stay alive until wait()."""
        t = ctypes.c_uint64()
        _check(self.L.chain_server_submit(self.h, op, ctypes.byref(item), ctypes.byref(t)))
        self._items[t.value] = item
        return t.value

    def wait(self, ticket: int, check: bool = True):
        """-> (status, queue_ms, service_ms, item)"""
        q, s = ctypes.c_double(), ctypes.c_double()
        st = self.L.chain_server_wait(self.h, ticket, ctypes.byref(q), ctypes.byref(s))
        item = self._items.pop(ticket, None)
        if check:
            _check(st)
        return st, q.value, s.value, item


def transcode_lcp2(data: bytes) -> bytes:
    """LCG2 container -> the reference CPU Chain's LCP2 bitstream (chain_transcode_lcp2)."""
    L = load()
    src = np.frombuffer(data, np.uint8)
    need = ctypes.c_size_t()
    st = L.chain_transcode_lcp2(src.ctypes.data, src.nbytes, None, 0, ctypes.byref(need))
    if st not in (CHAIN_OK, CHAIN_ERR_BUFFER_TOO_SMALL):
        _check(st)
    out = np.empty(max(1, need.value), np.uint8)
    _check(L.chain_transcode_lcp2(src.ctypes.data, src.nbytes, out.ctypes.data, out.nbytes, ctypes.byref(need)))
    return out[: need.value].tobytes()


def launch_count() -> int:
    """Kernel launches issued by the library in this process so far."""
    return load().chain_launch_count()


def alloc_count() -> int:
    """cudaMalloc / cudaMallocHost calls made by the library in this process so far."""
    return load().chain_alloc_count()


def compress_bound(n: int, dims: int) -> int:
    return load().chain_compress_bound(n, dims)
