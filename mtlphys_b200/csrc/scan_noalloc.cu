// scan_noalloc.cu — mp_exclusive_scan_noalloc: the single-pass exclusive scan
// with its scratch in a fixed, file-scope device array instead of caller- or
// library-allocated memory.
//
// Some callers cannot allocate device memory at the point where they need a
// scan: a frame loop that has a fixed per-frame memory budget and must not
// call cudaMalloc/cudaFree between frames, or a host framework whose own
// caching allocator owns the whole device heap and forbids raw allocations
// from plugins.  This entry point needs nothing from them beyond the input
// and output arrays.
//
// The scratch (a tile ticket, an error word and one look-back descriptor per
// 4096-element tile) lives in g_scan_scratch below: 33,024 bytes that every
// GPU which loads the library holds until the process exits.  That bounds n
// at kNoAllocMaxN = 2^24 elements.  A look-back that gives up sets the error
// word; mp_exclusive_scan_status(NULL, stream) reads and clears it (the next
// call's own clearing of the header would otherwise hide it).
#include "../../include/mtlphys_b200.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "pbf_kernels.h"

namespace {

constexpr uint32_t kNoAllocMaxN = 1u << 24;                           // 16,777,216 elements
constexpr uint32_t kNoAllocTiles = kNoAllocMaxN / mpb::kScanTile;      // 4096 descriptors
constexpr uint32_t kHeaderWords = 32;                                  // 256 bytes: ticket, error word

// [0] tile ticket, [1] error word (low 32 bits), [32 ...] tile descriptors.
static __device__ __align__(256) unsigned long long g_scan_scratch[kHeaderWords + kNoAllocTiles];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_addr[kMaxDevices] = {};

int report(int code, const char* msg) {
    mpb::record_error(msg);
    return code;
}

// Device address of g_scan_scratch on the current device.  In host code the
// symbol's name is only a host-side stand-in.  The address is looked up with
// the device current on every call made outside stream capture (a few
// microseconds), so it follows the module if the device was reset; a call
// made while `s` is being captured uses the address of the last call outside
// capture on this device, so the first call on a device must come before any
// capture.
int scratch_address(int dev, cudaStream_t s, void** out) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    const cudaError_t qe = cudaStreamIsCapturing(s, &cap);
    if (qe != cudaSuccess) cudaGetLastError();  // drop the failed query's error; treat as capturing
    const bool capturing = qe != cudaSuccess || cap != cudaStreamCaptureStatusNone;
    std::lock_guard<std::mutex> guard(g_lock);
    if (!capturing) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
        if (e != cudaSuccess) {
            char buf[256];
            std::snprintf(buf, sizeof(buf), "cudaGetSymbolAddress(g_scan_scratch): %s",
                          cudaGetErrorString(e));
            return report(MP_ERR_CUDA, buf);
        }
        g_addr[dev] = p;
    } else if (!g_addr[dev]) {
        return report(MP_ERR_INVALID_ARGUMENT,
                      "first mp_exclusive_scan_noalloc call on this device is inside a stream "
                      "capture: make one call outside capture first");
    }
    *out = g_addr[dev];
    return MP_OK;
}

int current_device(int* dev) {
    const cudaError_t e = cudaGetDevice(dev);
    if (e != cudaSuccess) return report(MP_ERR_CUDA, cudaGetErrorString(e));
    if (*dev < 0 || *dev >= kMaxDevices) return report(MP_ERR_UNSUPPORTED, "device index too large");
    return MP_OK;
}

}  // namespace

extern "C" int mp_exclusive_scan_noalloc(const uint32_t* in, uint32_t* out, uint32_t n,
                                         mp_stream stream) {
    if (n == 0) return MP_OK;
    if (!in || !out) return report(MP_ERR_INVALID_ARGUMENT, "in/out is NULL");
    if (n > kNoAllocMaxN) {
        char buf[160];
        std::snprintf(buf, sizeof(buf),
                      "n = %u exceeds the %u-element limit of the static scan scratch; use "
                      "mp_exclusive_scan with caller scratch",
                      n, kNoAllocMaxN);
        return report(MP_ERR_INVALID_ARGUMENT, buf);
    }
    int dev = -1;
    int rc = current_device(&dev);
    if (rc != MP_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* base = nullptr;
    rc = scratch_address(dev, s, &base);
    if (rc != MP_OK) return rc;
    const uint32_t tiles = mpb::scan_tiles_for(n);
    cudaError_t e;
    // The array keeps the previous call's ticket and descriptors: clear the
    // header and the descriptors this call uses.
    e = cudaMemsetAsync(base, 0, (kHeaderWords + size_t(tiles)) * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return report(MP_ERR_CUDA, cudaGetErrorString(e));
    auto* words = static_cast<unsigned long long*>(base);
    e = mpb::launch_scan(in, out, n, words + kHeaderWords, words, tiles, false,
                         reinterpret_cast<uint32_t*>(words + 1), s);
    if (e != cudaSuccess) return report(MP_ERR_CUDA, cudaGetErrorString(e));
    return MP_OK;
}

// The error word (words[1]) of the static scratch, for mp_exclusive_scan_status.
int mpb::noalloc_scan_error_word(cudaStream_t s, uint32_t** word) {
    int dev = -1;
    int rc = current_device(&dev);
    if (rc != MP_OK) return rc;
    void* base = nullptr;
    rc = scratch_address(dev, s, &base);
    if (rc != MP_OK) return rc;
    *word = reinterpret_cast<uint32_t*>(static_cast<unsigned long long*>(base) + 1);
    return MP_OK;
}
