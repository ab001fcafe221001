// Test-only extractor over the reference CPU encoder (oracle side; never shipped).
//
// This translation unit compiles the reference's own cpp/chain/lcps_cpp.cpp (included
// from where it lies in the reference checkout, path given by LCPS_CPP_SOURCE) and
// exposes, as the Python module `lcps_ref_streams`, the reference's LCP2 component
// decoder (decode_component_matrix_cpp, lcps_cpp.cpp:1715-1825).  It turns an LCP2
// bitstream produced by the reference encoder into its five integer streams
// (idrel, diff, keep, choice2, rel), the exact-coordinate corrections and the header
// fields, which are the bit-exact targets for the GPU encoder.
#include LCPS_CPP_SOURCE

namespace {

py::array_t<std::int64_t> matrix_to_array(const LcpsIntegerMatrixCpp& m) {
    const std::size_t dims = m.size();
    const std::size_t n = dims ? m[0].size() : 0;
    py::array_t<std::int64_t> out({static_cast<py::ssize_t>(dims), static_cast<py::ssize_t>(n)});
    auto* dst = out.mutable_data();
    for (std::size_t d = 0; d < dims; ++d)
        std::memcpy(dst + d * n, m[d].data(), n * sizeof(std::int64_t));
    return out;
}

py::dict decode_streams(const py::bytes& bitstream) {
    const std::string bytes = bitstream;
    LcpsReaderCpp reader(bytes);
    const auto magic = reader.Bytes(4);
    require_lcps_cpp(magic == "LCP2" || magic == "LCP3", "expected LCP2/LCP3");
    const std::size_t dims = reader.U32();
    const std::size_t n = reader.Size();
    const auto p = reader.I64();
    const double eb = reader.Double();
    const auto wrap_min = reader.I64();
    const auto wrap_max = reader.I64();
    std::vector<double> mins(dims);
    for (auto& m : mins) m = reader.Double();
    const char* names[5] = {"idrel", "diff", "keep", "choice2", "rel"};
    const std::size_t comp_dims[5] = {1, dims, dims, 1, dims};
    py::dict out;
    py::list magics, sizes;
    for (int s = 0; s < 5; ++s) {
        const auto blob = reader.Blob();
        magics.append(py::str(std::string(blob.substr(0, std::min<std::size_t>(4, blob.size())))));
        sizes.append(blob.size());
        out[names[s]] = matrix_to_array(decode_component_matrix_cpp(blob, comp_dims[s], n));
    }
    const auto exact_count = reader.Size();
    const auto exact_bytes = reader.Blob();
    reader.End();
    py::array_t<std::uint64_t> ex_idx(static_cast<py::ssize_t>(exact_count));
    py::array_t<double> ex_val(static_cast<py::ssize_t>(exact_count));
    if (exact_count) {
        std::string raw = magic == "LCP2" ? zstd_decompress_cpp(exact_bytes, exact_count * 16)
                                          : std::string(exact_bytes);
        LcpsReaderCpp r(raw);
        for (std::size_t i = 0; i < exact_count; ++i) {
            ex_idx.mutable_data()[i] = r.U64();
            ex_val.mutable_data()[i] = r.Double();
        }
    }
    out["dims"] = dims;
    out["n"] = n;
    out["p"] = p;
    out["eb"] = eb;
    out["wrap_min"] = wrap_min;
    out["wrap_max"] = wrap_max;
    out["mins"] = mins;
    out["magics"] = magics;
    out["sizes"] = sizes;
    out["exact_index"] = ex_idx;
    out["exact_value"] = ex_val;
    out["exact_bytes"] = exact_bytes.size();
    return out;
}

}  // namespace

PYBIND11_MODULE(lcps_ref_streams, m) {
    m.doc() = "Oracle-only: integer streams of a reference LCP2 bitstream.";
    m.def("decode_streams", &decode_streams, py::arg("bitstream"));
}
