// Allocation-free exclusive scan: the same decoupled look-back scan kernel as
// gs_exclusive_scan_u32, with its scratch in a fixed device array that is
// part of the loaded library instead of context workspace.
//
// Who needs it: code that must not call cudaMalloc at the point where it
// scans. cudaMalloc synchronises the device (a stall in a real-time render
// or training loop), and it is off limits to plugins whose host application
// owns all device memory through its own allocator. Such callers pass their
// input and output buffers and get the scan without any allocation.
//
// Scratch: one u64 look-back word per 2048-element tile plus two u32 words
// (tile counter, error word), for at most kNoAllocMaxElements elements. Every
// device that loads the library keeps this array (about 128 KiB) until the
// process exits. All calls share it: two calls whose work overlaps on the GPU
// (different streams, no ordering between them) race on it and both results
// are undefined; calls on one stream, or otherwise ordered, are safe. The
// array keeps the last call's contents; each call clears the part it uses
// (an asynchronous memset, which allocates nothing) before its kernel runs.
//
// A scan whose look-back wait gave up (a broken invariant, never expected)
// leaves a partial prefix and sets the array's error word; the call itself
// only enqueues work, so gs_exclusive_scan_u32_noalloc_status copies that word
// into a buffer the caller owns, ordered after the scan on the same stream.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gsplat_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace gsb {

// One look-back word per tile of the scan kernel; the element bound follows
// from the kernel's own tile size, so the words can never run past the array.
constexpr int kNoAllocMaxTiles = 16384;
constexpr long long kNoAllocMaxElements = 1ll * kNoAllocMaxTiles * kScanTile; // 33,554,432
static_assert(kNoAllocMaxElements == (1ll << 25), "the header states a 2^25-element bound");

// [0, kNoAllocMaxTiles): look-back words; [kNoAllocMaxTiles]: tile counter
// (low word) and error word (high word); [kNoAllocMaxTiles + 1]: where the
// total goes when the caller asks for none.
static __device__ __align__(256) unsigned long long g_noalloc_scan_scratch[kNoAllocMaxTiles + 2];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned long long* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device. Resolved once per
// device: the array's name is only a host-side handle, not a device address.
cudaError_t scratch_on_current_device(unsigned long long** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= kMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
        if (e != cudaSuccess)
            return e;
        g_scratch_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

} // namespace
} // namespace gsb

extern "C" gs_status gs_exclusive_scan_u32_noalloc(const unsigned* in, unsigned* out, int n,
                                                   unsigned* total_out, void* stream) {
    using namespace gsb;
    if (n < 0 || (n > 0 && (!in || !out)))
        return GS_ERR_INVALID;
    if (static_cast<long long>(n) > kNoAllocMaxElements)
        return GS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long* scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess)
        return GS_ERR_CUDA;
    if (n == 0) {
        if (total_out && cudaMemsetAsync(total_out, 0, sizeof(unsigned), s) != cudaSuccess)
            return GS_ERR_CUDA;
        return GS_OK;
    }
    unsigned* words = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxTiles);
    unsigned* tile_counter = words;
    unsigned* err = words + 1;
    unsigned* total =
        total_out ? total_out : reinterpret_cast<unsigned*>(scratch + kNoAllocMaxTiles + 1);
    // Clear the tile counter and error word; launch_scan clears the look-back
    // words of the tiles this call uses (and the tile counter again).
    if (cudaMemsetAsync(words, 0, 2 * sizeof(unsigned), s) != cudaSuccess)
        return GS_ERR_CUDA;
    launch_scan(s, n, in, nullptr, out, scratch, tile_counter, total, err);
    return cudaGetLastError() == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}

extern "C" gs_status gs_exclusive_scan_u32_noalloc_status(unsigned* status_out, void* stream) {
    using namespace gsb;
    if (!status_out)
        return GS_ERR_INVALID;
    unsigned long long* scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess)
        return GS_ERR_CUDA;
    const unsigned* err = reinterpret_cast<const unsigned*>(scratch + kNoAllocMaxTiles) + 1;
    // cudaMemcpyDefault: the caller's word may be device or host memory.
    return cudaMemcpyAsync(status_out, err, sizeof(unsigned), cudaMemcpyDefault,
                           static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? GS_OK
               : GS_ERR_CUDA;
}
