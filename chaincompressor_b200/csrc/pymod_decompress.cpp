// Python module `lcps_gpu_decompress_ans`: the reference GPU decoder's surface
// (cu/decompress/lcps_gpu_decompress_ans.cu:2898-2921), wrapped by
// chain_caller.gpu_decompress (chain_caller.py:33-35), backed by libchain_b200.
//
//   lcps_decompress_gpu(compressed_data, output_soa=False) -> ndarray
//
// Returns C-contiguous (N, D), or (D, N) when output_soa is true.  The values are
// float64 and equal, bit for bit, to what the reference CPU decoder produces for the
// same integers (the reference GPU decoder returns float32 and cannot keep |err| <= eb
// against float64 input).  dtype="float32" rounds them to float32 instead.
#include "pymod_common.h"

namespace py = pybind11;
using namespace chain_py;

static py::array decompress_impl(py::bytes data, bool output_soa, const std::string& dtype) {
    char* buf = nullptr;
    Py_ssize_t len = 0;
    if (PyBytes_AsStringAndSize(data.ptr(), &buf, &len) != 0) throw py::error_already_set();
    const bool f32 = dtype == "float32";
    if (!f32 && dtype != "float64") throw std::invalid_argument("dtype must be 'float64' or 'float32'");
    uint64_t n = 0;
    uint32_t d = 0;
    check(chain_peek(buf, static_cast<size_t>(len), &n, &d, nullptr));
    std::vector<py::ssize_t> shape = output_soa ? std::vector<py::ssize_t>{(py::ssize_t)d, (py::ssize_t)n}
                                                : std::vector<py::ssize_t>{(py::ssize_t)n, (py::ssize_t)d};
    py::array out = f32 ? py::array(py::array_t<float>(shape)) : py::array(py::array_t<double>(shape));
    const size_t cap = static_cast<size_t>(n) * d * (f32 ? 4 : 8);
    std::lock_guard<std::mutex> lock(contexts().mu);
    chain_ctx* ctx = context_for_current_device();
    chain_status st;
    {
        py::gil_scoped_release nogil;
        st = chain_decompress(ctx, buf, static_cast<size_t>(len), f32 ? CHAIN_F32 : CHAIN_F64,
                              output_soa ? CHAIN_SOA : CHAIN_AOS, out.mutable_data(), cap, &n, &d);
    }
    check(st);
    return out;
}

PYBIND11_MODULE(lcps_gpu_decompress_ans, m) {
    m.doc() = "B200 Chain decompressor for LCG2 v2 containers (bit-exact FP64 reconstruction).";
    m.def("lcps_decompress_gpu", &decompress_impl, py::arg("compressed_data"), py::arg("output_soa") = false,
          py::arg("dtype") = "float64",
          "Decompress an LCG2 v2 container into coordinates in the original particle order. "
          "output_soa=False returns (N, D); True returns (D, N), both C-contiguous.");
}
