// Python module `lcps_gpu_cpp`: the reference GPU encoder's surface
// (cu/chain/lcps_gpu_cpp.cu:1095-1102), wrapped by chain_caller.chain_gpu
// (chain_caller.py:38-40), backed by libchain_b200.
//
//   lcps_compress2_gpu(points, eb, p, threshold, diff) -> bytes
//
// `points` is the reference's C-contiguous (D, N) SoA array.  Differences from the
// reference, all needed for bit-exact parity with the CPU Chain path:
//   * float32 and float64 inputs are taken as they are (the reference casts to
//     float32); other dtypes are converted to float64;
//   * eb is a Python float (double), p and threshold are 64-bit;
//   * the result is an LCG2 version-2 container (FP64 header fields, exact
//     corrections, interleaved-rANS sections) instead of LCG2 v1 with nvCOMP sections.
// `diff` is accepted and ignored, as in the reference (lcps_gpu_cpp.cu:721).
#include "pymod_common.h"

namespace py = pybind11;
using namespace chain_py;

static py::bytes compress_impl(py::array arr, double eb, int64_t p, int64_t threshold, chain_layout layout, bool bl,
                               bool l1, bool l2, uint32_t bytes_per_lane) {
    py::array a;
    chain_dtype dt;
    if (py::isinstance<py::array_t<float>>(arr) && (arr.flags() & py::array::c_style)) {
        a = arr;
        dt = CHAIN_F32;
    } else if (arr.dtype().is(py::dtype::of<float>())) {
        a = py::array_t<float, py::array::c_style | py::array::forcecast>::ensure(arr);
        dt = CHAIN_F32;
    } else {
        a = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(arr);
        dt = CHAIN_F64;
    }
    if (!a || a.ndim() != 2)
        throw std::invalid_argument(layout == CHAIN_SOA ? "points must be a 2-D array of shape (D, N)"
                                                        : "points must be a 2-D ndarray with shape (N, D)");
    const uint64_t n = static_cast<uint64_t>(layout == CHAIN_SOA ? a.shape(1) : a.shape(0));
    const uint32_t d = static_cast<uint32_t>(layout == CHAIN_SOA ? a.shape(0) : a.shape(1));
    chain_opts opts{};
    opts.struct_size = sizeof(chain_opts);
    opts.bl = bl;
    opts.l1 = l1;
    opts.l2 = l2;
    opts.rans_bytes_per_lane = bytes_per_lane;
    std::lock_guard<std::mutex> lock(contexts().mu);
    chain_ctx* ctx = context_for_current_device();
    size_t len = 0;
    chain_status st;
    {
        py::gil_scoped_release nogil;
        st = chain_compress(ctx, a.data(), dt, layout, n, d, eb, p, threshold, &opts, &len);
    }
    check(st);
    PyObject* obj = PyBytes_FromStringAndSize(nullptr, static_cast<Py_ssize_t>(len));
    if (!obj) throw py::error_already_set();
    py::bytes out = py::reinterpret_steal<py::bytes>(obj);
    {
        py::gil_scoped_release nogil;
        st = chain_result_copy(ctx, PyBytes_AS_STRING(obj), len);
    }
    check(st);
    return out;
}

PYBIND11_MODULE(lcps_gpu_cpp, m) {
    m.doc() = "B200 Chain compressor: FP64 quantization, Z-order block sort, chaining, "
              "interleaved rANS; LCG2 v2 bytes (bit-exact integers vs the CPU Chain).";
    m.def(
        "lcps_compress2_gpu",
        [](py::array points, double eb, int64_t p, int64_t threshold, int64_t diff, bool bl, bool l1, bool l2,
           uint32_t rans_bytes_per_lane) {
            (void)diff;
            return compress_impl(points, eb, p, threshold, CHAIN_SOA, bl, l1, l2, rans_bytes_per_lane);
        },
        py::arg("points"), py::arg("eb"), py::arg("p"), py::arg("threshold"), py::arg("diff"),
        py::arg("bl") = true, py::arg("l1") = true, py::arg("l2") = true, py::arg("rans_bytes_per_lane") = 0,
        "Compress (D, N) float32/float64 coordinates into one self-contained LCG2 v2 bytes object.");
    m.def(
        "lcps_compress2_gpu_aos",
        [](py::array points, double eb, int64_t p, int64_t threshold, int64_t diff, bool bl, bool l1, bool l2,
           uint32_t rans_bytes_per_lane) {
            (void)diff;
            return compress_impl(points, eb, p, threshold, CHAIN_AOS, bl, l1, l2, rans_bytes_per_lane);
        },
        py::arg("points"), py::arg("eb"), py::arg("p"), py::arg("threshold"), py::arg("diff") = 0,
        py::arg("bl") = true, py::arg("l1") = true, py::arg("l2") = true, py::arg("rans_bytes_per_lane") = 0,
        "Same as lcps_compress2_gpu for (N, D) coordinates (the CPU entry point's layout).");
}
