// Host-side helpers shared by the C-ABI translation units: error types that
// the entry points turn into gs_status codes, CUDA checks and a grow-only
// device buffer.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace gsb {
namespace host {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct InvalidArg : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct StateError : std::logic_error {
    using std::logic_error::logic_error;
};
// A bounded device-side wait gave up (its kernel set the device error word).
struct TimeoutError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw CudaError(std::string("gsplat_b200: ") + what + ": " + cudaGetErrorString(e));
}
inline void req(bool ok, const char* what) {
    if (!ok)
        throw InvalidArg(std::string("gsplat_b200: ") + what);
}

inline size_t align_up(size_t v, size_t a = 256) { return (v + a - 1) / a * a; }

struct DevBuf {
    char* p = nullptr;
    size_t bytes = 0;
    // Grow-only; new storage is zeroed when `zero` (used for accumulators).
    char* ensure(size_t need, cudaStream_t s, bool zero = false) {
        if (need <= bytes && p)
            return p;
        if (p) {
            ck(cudaStreamSynchronize(s), "sync before workspace growth");
            ck(cudaFree(p), "workspace free");
            p = nullptr;
            bytes = 0;
        }
        const size_t cap = align_up(need + need / 4 + 4096);
        ck(cudaMalloc(&p, cap), "workspace cudaMalloc");
        bytes = cap;
        if (zero)
            ck(cudaMemsetAsync(p, 0, cap, s), "workspace zero");
        return p;
    }
    // Exactly `need` bytes (rounded to 256) when it must grow; for large
    // planned buffers where growth headroom would waste memory.
    char* exact(size_t need, cudaStream_t s, bool zero = false) {
        if (need <= bytes && p) {
            if (zero)
                ck(cudaMemsetAsync(p, 0, need, s), "workspace zero");
            return p;
        }
        if (p) {
            ck(cudaStreamSynchronize(s), "sync before workspace growth");
            ck(cudaFree(p), "workspace free");
            p = nullptr;
            bytes = 0;
        }
        const size_t cap = align_up(need > 0 ? need : 256);
        ck(cudaMalloc(&p, cap), "workspace cudaMalloc");
        bytes = cap;
        if (zero)
            ck(cudaMemsetAsync(p, 0, cap, s), "workspace zero");
        return p;
    }
    void release() {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

inline int msb_bits(unsigned v) {
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

} // namespace host
} // namespace gsb
