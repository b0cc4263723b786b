// ref_spatial.cpp — compiles the reference's engine/shaders/Spatial.metal
// unchanged as host C++ (through the metal_stdlib shim in this folder) and
// exposes one loop per kernel: call k runs GPU thread gid = k.
//
// TEST INFRASTRUCTURE ONLY (the "_ref" cross-check of the oracle).
#include "Spatial.metal"

#include "ref_harness.h"

extern "C" {

void ref_k_hash_cells(const float* pos4, uint32_t* hashes, const void* sp, uint32_t threads) {
    const auto& p = *static_cast<const SpatialParams*>(sp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        hashCells(reinterpret_cast<const float4*>(pos4), hashes, p, uint(g));
}

void ref_k_count_cells(const uint32_t* hashes, uint32_t* counts, const void* sp, uint32_t threads) {
    const auto& p = *static_cast<const SpatialParams*>(sp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        countCells(hashes, reinterpret_cast<atomic_uint*>(counts), p, uint(g));
}

void ref_k_scatter_particles(const uint32_t* hashes, const uint32_t* cell_start, uint32_t* cursor,
                             uint32_t* sorted_index, const void* sp, uint32_t threads) {
    const auto& p = *static_cast<const SpatialParams*>(sp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        scatterParticles(hashes, cell_start, reinterpret_cast<atomic_uint*>(cursor), sorted_index,
                         p, uint(g));
}

void ref_k_gather_positions(const float* pos4, const uint32_t* sorted_index, float* sorted4,
                            const void* sp, uint32_t threads) {
    const auto& p = *static_cast<const SpatialParams*>(sp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        gatherPositions(reinterpret_cast<const float4*>(pos4), sorted_index,
                        reinterpret_cast<float4*>(sorted4), p, uint(g));
}

void ref_k_count_neighbors(const float* pos4, const uint32_t* cell_start,
                           const uint32_t* sorted_index, uint32_t* counts, const void* sp,
                           const float* sorted4, uint32_t threads) {
    const auto& p = *static_cast<const SpatialParams*>(sp);
#pragma omp parallel for schedule(dynamic, 1024) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        countNeighbors(reinterpret_cast<const float4*>(pos4), cell_start, sorted_index, counts, p,
                       reinterpret_cast<const float4*>(sorted4), uint(g));
}

size_t ref_sizeof_spatial_params(void) { return sizeof(SpatialParams); }

void ref_fill_spatial_params(void* out, const float origin[3], float cell, float inv_cell,
                             float radius_sq, uint32_t n, uint32_t total_cells,
                             const uint32_t dims[3], uint32_t max_nbr) {
    auto& sp = *static_cast<SpatialParams*>(out);
    sp.gridOrigin = float3(origin[0], origin[1], origin[2]);
    sp.cellSize = cell;
    sp.invCellSize = inv_cell;
    sp.neighborRadiusSq = radius_sq;
    sp.particleCount = n;
    sp.totalCells = total_cells;
    sp.gridDim = uint3(dims[0], dims[1], dims[2]);
    sp.maxNeighborsForViz = max_nbr;
}

}  // extern "C"
