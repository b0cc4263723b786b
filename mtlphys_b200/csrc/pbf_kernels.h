// pbf_kernels.h — host-side launchers of the PBF step kernels (sm_100a).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_device.cuh"

namespace mpb {

// Device buffers of one scene (all sized for n particles / cells+1 cells).
struct DevState {
    float4* pos;            // positions, original order (predicted during a step)
    float4* vel;            // velocities
    float4* prev;           // positions at the start of the step
    float4* sorted_a;       // sorted positions: hash-time gather, solver iterate
    float4* sorted_b;       // sorted (position, lambda) written by the lambda pass
    uint32_t* hash;         // cell hash per particle
    uint32_t* off;          // rank of the particle's atomic increment in its cell
    uint32_t* tmp;          // unstable cell-grouped order (before the stable fix-up)
    uint32_t* sidx;         // sortedIndex: slot -> particle, stable within a cell
    uint32_t* scell;        // hash cell per sorted slot (anchor of the solver state)
    uint32_t* row_masks;            // 9 x mask_stride in-range bits per stencil row
    uint32_t* mask_overflow;        // bit r: row r exceeded 32 candidates (delta re-tests the rest)
    uint32_t mask_stride;
    uint32_t* ncount;       // neighbour count per particle
    float* lambdas;         // last lambda per particle
    float* foam;            // foam intensity per particle
    uint32_t* counts;       // cells+1 per-cell counts (all zero between passes)
    uint32_t* cstart;       // cells+1 exclusive scan of counts
    uint32_t* long_list;    // cells whose segment exceeds kSegMax
    uint32_t* long_count;   // entries in long_list
    unsigned long long* scan_status;  // look-back tile descriptors
    unsigned long long* scan_ticket;  // monotonic tile ticket
    uint32_t scan_tiles;
    uint32_t* err;          // device error word (kDevErr*)
    SphereState* sphere;    // sphere state (scene 2)
};

constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItemsPerThread = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItemsPerThread;  // 4096
constexpr uint32_t kSegMax = 256;  // longest cell segment ranked in place

inline uint32_t scan_tiles_for(uint64_t n) { return uint32_t((n + kScanTile - 1) / kScanTile); }

// Optional per-kernel timing: the launchers call begin() before and end()
// after every kernel they enqueue (CUDA events on the same stream).
struct KernelTimer {
    virtual void begin(cudaStream_t s) = 0;
    virtual void end(const char* kernel, cudaStream_t s) = 0;
    virtual ~KernelTimer() = default;
};

// Bounds, in polls, of the device-side waits (the scan's look-back, the batch
// kernel's grid barrier).  mp_set_spin_limit() changes them process-wide;
// launchers read them when they enqueue a kernel, and engines and batches
// re-capture their CUDA graphs when spin_limit_epoch() has moved on.
constexpr uint32_t kDefaultScanSpinLimit = 1u << 22;     // ~0.1-1 s of 32 ns naps
constexpr uint32_t kDefaultBarrierSpinLimit = 1u << 24;  // ~1-10 s of 64 ns naps
uint32_t scan_spin_limit();
uint32_t barrier_spin_limit();
uint32_t spin_limit_epoch();

// Device memory of engines and batches: through the allocator installed
// with mp_set_device_allocator (cudaMalloc/cudaFree by default).  Each block
// is freed by the allocator that made it.  dev_alloc returns MP_OK or
// MP_ERR_OUT_OF_MEMORY (message recorded).
int dev_alloc(void** p, size_t bytes, int device);
void dev_free(void* p);

// Exclusive scan with decoupled look-back.  `status` holds `tiles` words and
// `ticket` one word, both from an earlier call with the same tile count or
// zeroed.  zero_input: write 0 over `in` after reading it.  A look-back that
// waits longer than scan_spin_limit() polls sets kDevErrSpin in *err and
// gives that tile a wrong prefix (every write stays inside `out`).
cudaError_t launch_scan(const uint32_t* in, uint32_t* out, uint32_t n, unsigned long long* status,
                        unsigned long long* ticket, uint32_t tiles, bool zero_input, uint32_t* err,
                        cudaStream_t s, KernelTimer* t = nullptr);

// Timer helpers for the launchers.
inline void tbegin(KernelTimer* t, cudaStream_t s) {
    if (t) t->begin(s);
}
inline void tend(KernelTimer* t, const char* k, cudaStream_t s) {
    if (t) t->end(k, s);
}

// Spatial hash of the current (predict = false) or predicted (predict =
// true) positions: fills hash, cstart, sidx, sorted_a (and counts back to
// zero).  With predict, the sphere (if any) is advanced first.
cudaError_t launch_hash_pass(const StepConsts& c, const DevState& d, bool predict, cudaStream_t s,
                             KernelTimer* t = nullptr);
// countNeighbors on sorted_a (buildSpatialHash only; the step fuses it).
cudaError_t launch_count_neighbors(const StepConsts& c, const DevState& d, cudaStream_t s,
                                   KernelTimer* t = nullptr);
// K solver iterations + scatter-back + finalize + foam.
cudaError_t launch_solver(const StepConsts& c, const DevState& d, uint32_t iterations,
                          cudaStream_t s, KernelTimer* t = nullptr);

// Number of kernel launches one step issues (for the benchmark's count).
uint32_t step_launch_count(uint32_t iterations);

// Legacy integrator (Integrate.metal SimParams, Shared.h:28-35).
struct IntegrateConsts {
    uint32_t n;
    float dt, damping, restitution;
    float gx, gy, gz;
    float bminx, bminy, bminz, bmaxx, bmaxy, bmaxz;
};
cudaError_t launch_integrate(const IntegrateConsts& c, float4* pos, float4* vel, cudaStream_t s);

// Mouse pulse (MousePulseUniforms, Constraints.metal:222-229).
struct MouseConsts {
    uint32_t n;
    float ox, oy, oz, dx, dy, dz, fx, fy, fz;
    float radius, falloff;
};
cudaError_t launch_mouse_pulse(const MouseConsts& c, float4* vel, const float4* pos, cudaStream_t s);

// Sets the message mp_last_error() returns on this thread.
void record_error(const char* msg);

// Device address of the error word of mp_exclusive_scan_noalloc's static
// scratch on the current device (MP_OK or an MP_ERR_* status).
int noalloc_scan_error_word(cudaStream_t s, uint32_t** word);

}  // namespace mpb
