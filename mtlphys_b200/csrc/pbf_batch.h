// pbf_batch.h — device-side layout and launcher of the multi-scene step.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_device.cuh"

namespace mpb {

// Per-scene record in device memory.  `c` holds the scene's constants; its
// sub-grid fields (c.g.lx .. c.g.cells, c.g.cell0) are rewritten by every
// step from the bounding box `bb` of the scene's predicted cells.
struct SceneDev {
    StepConsts c;
    uint32_t p0;         // first particle (and first sorted slot) of the scene
    uint32_t bb[6];      // min x, y, z / max x, y, z dense cell of this step
    uint32_t pad;
    SphereState sphere;  // used when c.sphere != 0
};

// Recording of one step for the adjoint (lam == nullptr: not recording).
// The step's prev, sidx, scell and cstart arrays are kept as well: for a
// recorded step the host points BatchArgs at the record's own copies.
struct BatchRecord {
    SceneDev* scenes;      // scene table once the sub-grids are set (sphere advanced)
    SphereState* sphere0;  // every scene's sphere before the advance
    float4* lam;           // iterations x stride: (l, lambda) written by each lambda pass
    float4* delta;         // iterations x stride: unclamped correction of each delta pass
    uint32_t* masks;       // iterations x 9 x mask_stride: row masks of each lambda pass
    uint32_t* overflow;    // iterations x mask_stride: bit r set for a long row r
    uint32_t stride;       // slots per lam / delta array
};

struct BatchArgs {
    SceneDev* scenes;
    uint32_t scene_begin, scene_end;  // scenes of this launch
    const uint32_t* scene_of;         // scene of every particle / slot
    uint32_t p_begin, p_end;          // particles (= slots) of this launch
    uint32_t iterations;
    float4 *pos, *vel, *prev, *sorted_a, *sorted_b;
    uint32_t *hash, *off, *tmp, *sidx, *scell, *ncount;
    float *lambdas, *foam;
    uint32_t *counts, *cstart, *tile_sums;
    uint32_t max_cells;               // capacity of counts / cstart minus one
    uint32_t *long_list, *long_count;
    uint32_t *row_masks, *mask_overflow;
    uint32_t mask_stride;
    uint32_t* total_cells;
    unsigned *bar_count, *bar_gen;
    uint32_t* err;
    // Bounded grid barrier: a block waits at most spin_limit polls.  One
    // that gives up sets kDevErrSpin and *abort, and every block then leaves
    // the launch at its next barrier; a launch that starts with *abort set
    // does nothing (the host clears it in mp_batch_check_errors).
    // bar_extra (a test hook, normally 0) makes every barrier wait for that
    // many more blocks than the launch has, so that each wait runs out.
    uint32_t* abort;
    uint32_t spin_limit, bar_extra;
    uint32_t scorr4;  // 1: every scene's s_corr exponent is 4 (the kernel fixes it at compile time)
    BatchRecord rec;
};

// Cooperative launch of one step of scenes [scene_begin, scene_end) with
// `blocks` blocks of `block` (128, 256 or 512) threads.
cudaError_t launch_batch_step(const BatchArgs& args, uint32_t block, uint32_t blocks, cudaStream_t s);
// Resident blocks per SM of the step kernel at that block size (0: unsupported).
int batch_max_blocks_per_sm(uint32_t block);

}  // namespace mpb
