// Shared helpers of the two pybind11 modules: one library context per CUDA device,
// status -> Python exception mapping (std::invalid_argument -> ValueError, everything
// else -> RuntimeError, as the reference modules raise them).
#pragma once

#include <cuda_runtime.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "chain_b200.h"

namespace chain_py {

namespace py = pybind11;

inline void check(chain_status st) {
    if (st == CHAIN_OK) return;
    const std::string msg = chain_last_error_message();
    if (st == CHAIN_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

struct Contexts {
    std::mutex mu;
    std::map<int, chain_ctx*> by_device;
};

inline Contexts& contexts() {
    static Contexts* c = new Contexts();  // never destroyed: CUDA may be torn down first
    return *c;
}

// Returns the context of the current CUDA device, creating it on first use.  The
// caller holds contexts().mu for the duration of its call.
inline chain_ctx* context_for_current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("no CUDA device available");
    }
    auto& m = contexts().by_device;
    auto it = m.find(dev);
    if (it != m.end()) return it->second;
    chain_ctx* ctx = nullptr;
    check(chain_ctx_create(dev, nullptr, &ctx));
    m[dev] = ctx;
    return ctx;
}

}  // namespace chain_py
