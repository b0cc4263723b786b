// host_common.h — host-side helpers shared by the single-scene engine
// (engine.cpp) and the multi-scene batch (batch.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/mtlphys_b200.h"
#include "pbf_device.cuh"
#include "pbf_kernels.h"

namespace mpb {

// Records a formatted message for mp_last_error() and returns `code`.
int fail(int code, const char* fmt, ...);
const char* last_error();

#define MP_CUDA(call)                                                                          \
    do {                                                                                       \
        const cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                                 \
            return ::mpb::fail(e_ == cudaErrorMemoryAllocation ? MP_ERR_OUT_OF_MEMORY : MP_ERR_CUDA, \
                               "%s: %s", #call, cudaGetErrorString(e_));                       \
    } while (0)

// Device allocation through the installed allocator (dev_alloc): returns
// from the calling function with the status on failure.
#define MP_ALLOC(ptr, bytes, device)                                                           \
    do {                                                                                       \
        void* p_ = nullptr;                                                                    \
        const int rc_ = ::mpb::dev_alloc(&p_, (bytes), (device));                              \
        if (rc_ != MP_OK) return rc_;                                                          \
        (ptr) = static_cast<decltype(ptr)>(p_);                                                \
    } while (0)

// Makes `dev` current for the scope and restores the previous device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

inline uint32_t round_up(uint32_t n, uint32_t m) { return ((n + m - 1) / m) * m; }

// Dense hash grid of buildSpatialBuffers (Engine.cpp:398-403, 443-451).
int make_grid(const mp_pbf_params& p, GridDev& g);
int validate_params(const mp_pbf_params& p);
// Engine::seedParticles (Engine.cpp:454-549) and the jittered lattice.
int seed_scene(const mp_pbf_params& p, uint32_t scene, const mp_scene_desc& d, uint32_t n,
               std::vector<float>& pos);
void fill_default_params(mp_pbf_params& p);
void fill_default_desc(mp_scene_desc& d);
size_t elem_bytes(uint32_t which);
StepConsts make_consts(const mp_pbf_params& p, const GridDev& g, uint32_t n, float dt, bool sphere);

}  // namespace mpb
