// sort_noalloc.cu -- the radix sort of particle cell keys with no device
// allocation at all.
//
// Who needs this: callers that hand the library device buffers they own and
// do not let it allocate -- a host application whose device memory comes from
// its own pool or a fixed budget reserved at start-up, or a latency-sensitive
// loop where cudaMalloc/cudaFree may implicitly synchronize the device.  They
// pass the input keys and the output buffers; the sort's working memory (one
// ping-pong pair of key/value buffers, the per-tile digit histogram and the
// scan partials) lives in one fixed, file-scope device array instead.
//
// That array is part of the library image: every GPU that loads the library
// holds it (MPM_SORT_NOALLOC_MAX_KEYS keys, about 8.9 MB) until the process
// exits.  All calls share it, so calls whose work overlaps on the GPU race
// with each other; serialize them (one stream, or events).  Every word a call
// reads from the array is first written by that same call (the histogram by
// the upsweep, the partials by the scan, the ping-pong pair by the scatter),
// so nothing carries over between calls and nothing needs clearing.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/mpm_b200.h"
#include "engine_host.hpp"

namespace mpm {

mpm_status recordError(mpm_status st, const char* msg);

namespace {

constexpr size_t kMaxKeys = MPM_SORT_NOALLOC_MAX_KEYS;
constexpr size_t kTilesMax = (kMaxKeys + kSortTileKeys - 1) / kSortTileKeys;  // radix tiles
constexpr size_t kHistWords = 256 * kTilesMax;
constexpr size_t kPartialWords = 64;                    // >= scan chunks of the histogram + 1
static_assert(kPartialWords >= (kHistWords + 4095) / 4096 + 1, "scan partials too small");
constexpr size_t kScratchWords = 2 * kMaxKeys + kHistWords + kPartialWords;

// The scratch: [tmp keys | tmp values | histogram | scan partials].
static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
uint32_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  Host code may
// not use `g_sort_scratch` itself: on the host that name is only a stand-in
// for the symbol, not a device address.  Resolved once per device, on the
// first call made with that device current, and cached for the life of the
// process: a cudaDeviceReset unloads the library's module on that device, so
// the cached address is not valid across a reset.
mpm_status scratchForCurrentDevice(uint32_t** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return recordError(MPM_ERR_CUDA, "mpm_sort_keys_device_noalloc: no current CUDA device");
    }
    if (dev < 0 || dev >= kMaxDevices)
        return recordError(MPM_ERR_UNSUPPORTED, "mpm_sort_keys_device_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return recordError(MPM_ERR_CUDA, (std::string("mpm_sort_keys_device_noalloc: cudaGetSymbolAddress: ") +
                                              cudaGetErrorString(e)).c_str());
        }
        g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_ptr[dev];
    return MPM_OK;
}

// True when the n-word ranges starting at a and b share a word.
bool rangesOverlap(const uint32_t* a, const uint32_t* b, uint32_t n) {
    const uintptr_t pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = (uintptr_t)n * sizeof(uint32_t);
    return pa < pb + len && pb < pa + len;
}

// The scratch address is the current device's, so the stream must belong to
// that device: a stream of another device would run the passes on that device
// against this device's scratch.  The legacy and per-thread default streams
// (passed as null or their handles) belong to the current device.
mpm_status checkStreamDevice(cudaStream_t stream) {
    if (stream == nullptr || stream == cudaStreamLegacy || stream == cudaStreamPerThread) return MPM_OK;
    int cur = -1, sdev = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e == cudaSuccess) e = cudaStreamGetDevice(stream, &sdev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return recordError(MPM_ERR_INVALID_ARG, (std::string("mpm_sort_keys_device_noalloc: invalid stream: ") +
                                                 cudaGetErrorString(e)).c_str());
    }
    if (sdev != cur)
        return recordError(MPM_ERR_INVALID_ARG,
                           ("mpm_sort_keys_device_noalloc: the stream belongs to device " + std::to_string(sdev) +
                            " but device " + std::to_string(cur) +
                            " is current; make the stream's device current (mpm_set_device) before the call")
                               .c_str());
    return MPM_OK;
}

}  // namespace
}  // namespace mpm

extern "C" mpm_status mpm_sort_keys_device_noalloc(const uint32_t* keys, uint32_t n, int32_t bits,
                                                   uint32_t* sorted_keys, uint32_t* perm, void* stream) {
    if (bits < 1 || bits > 32)
        return mpm::recordError(MPM_ERR_INVALID_ARG, "mpm_sort_keys_device_noalloc: bits must be in [1, 32]");
    if ((size_t)n > mpm::kMaxKeys)
        return mpm::recordError(MPM_ERR_INVALID_ARG,
                                ("mpm_sort_keys_device_noalloc: n = " + std::to_string(n) +
                                 " exceeds the fixed scratch capacity of MPM_SORT_NOALLOC_MAX_KEYS = " +
                                 std::to_string(mpm::kMaxKeys) + " keys; use mpm_sort_keys for larger inputs")
                                    .c_str());
    if (n == 0) return MPM_OK;
    if (!keys || !sorted_keys || !perm)
        return mpm::recordError(MPM_ERR_INVALID_ARG, "mpm_sort_keys_device_noalloc: null buffer");
    // The first pass reads `keys` while it scatters into the outputs (or into
    // the scratch pair, which later passes scatter back into the outputs), so
    // the three buffers must be distinct: an in-place call would sort wrongly.
    if (mpm::rangesOverlap(keys, sorted_keys, n) || mpm::rangesOverlap(keys, perm, n) ||
        mpm::rangesOverlap(sorted_keys, perm, n))
        return mpm::recordError(MPM_ERR_INVALID_ARG,
                                "mpm_sort_keys_device_noalloc: keys, sorted_keys and perm must not overlap");
    mpm_status st = mpm::checkStreamDevice(static_cast<cudaStream_t>(stream));
    if (st != MPM_OK) return st;
    uint32_t* scratch = nullptr;
    st = mpm::scratchForCurrentDevice(&scratch);
    if (st != MPM_OK) return st;
    uint32_t* tmp_keys = scratch;
    uint32_t* tmp_vals = scratch + mpm::kMaxKeys;
    uint32_t* hist = scratch + 2 * mpm::kMaxKeys;
    uint32_t* partials = hist + mpm::kHistWords;
    cudaError_t e = mpm::radixSortPairsInto(keys, sorted_keys, perm, tmp_keys, tmp_vals, n, bits, hist, partials,
                                            static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return mpm::recordError(MPM_ERR_CUDA,
                                (std::string("mpm_sort_keys_device_noalloc: ") + cudaGetErrorString(e)).c_str());
    }
    return MPM_OK;
}
