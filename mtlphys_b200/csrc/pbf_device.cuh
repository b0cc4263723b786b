// pbf_device.cuh — device-side types and per-particle math of the PBF step.
//
// The arithmetic follows the reference shaders:
//   cell coordinates / hash ........ engine/shaders/Spatial.metal:35-43
//   poly6 / spiky gradient ......... engine/shaders/Constraints.metal:29-39
//   lambda ......................... Constraints.metal:124-127
//   position correction + s_corr ... Constraints.metal:170-198
//   sphere push .................... Constraints.metal:262-277
//   finalize ....................... Constraints.metal:305-353
//   foam ........................... Constraints.metal:287-299
// Every constant the reference hard-codes in a shader is a field of
// StepConsts (filled from mp_pbf_params on the host).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mpb {

// Uniform hash grid: SpatialParams (engine/shaders/Shared.h:40-49).  A
// particle's cell is computed on the dense grid (origin, cell size, dense
// dims) exactly as the reference does; the cells that are stored may be a
// box-shaped sub-grid of it (lower corner l, dims g, stored from cell0 on),
// with the same x-fastest order, so the sorted order does not change.  The
// single-scene engine stores the whole dense grid (l = 0, g = dense dims,
// cell0 = 0); the batched engine stores each scene's bounding box of cells.
struct GridDev {
    float ox, oy, oz;    // gridOrigin (= bounds_min)
    float inv;           // invCellSize = 1.0f / cellSize, rounded on the host
    float cs;            // cellSize
    int dgx, dgy, dgz;   // dense gridDim: cell coordinates are clamped to it
    int lx, ly, lz;      // sub-grid lower corner, in dense cell coordinates
    int gx, gy, gz;      // sub-grid dims
    uint32_t cell0;      // index of the sub-grid's first cell in the cell arrays
    uint32_t cells;      // gx * gy * gz
};

// Per-launch constants of one step (PBFParams, Shared.h:53-71, plus the
// shader literals).  Passed by value.
struct StepConsts {
    GridDev g;
    uint32_t n;
    float h, h2, poly6, spiky;
    float inv_rho0, eps;
    float scorr_k, inv_wq, max_step;
    uint32_t scorr_n;
    float scorr_pq;     // poly6 / W(dq): s_corr's ratio is d^3 * scorr_pq
    float delta_scale;  // -spiky / rho0: the position correction's common factor
    float bminx, bminy, bminz, bmaxx, bmaxy, bmaxz;
    float gravx, gravy, gravz;
    float dt, inv_dt, damping, vmax, vmax_frac;
    float wall_eps, floor_fric, wall_fric;
    float foam_maxn, foam_lo, foam_hi;
    int sphere;  // 1: sphere-drop scene (sphere state lives in device memory)
    float sph_gravity, sph_drag, sph_rest;
};

// Device-resident sphere state: center xyz, velocity xyz, radius.
struct SphereState {
    float c[3];
    float v[3];
    float r;
    float pad;
};

constexpr uint32_t kDevErrSpin = 0x1u;
constexpr uint32_t kDevErrNaN = 0x2u;
constexpr uint32_t kDevErrIndex = 0x4u;

#ifdef __CUDACC__
// ---- spatial hash -----------------------------------------------------------

// cellCoordOf: q = (p - origin) * invCellSize, floor, clamp to [0, dim-1].
// Explicit round-to-nearest ops keep the two roundings of the reference
// formula (no contraction), and cvt.rmi saturates (NaN -> 0) so that every
// input maps to a valid cell.
__device__ __forceinline__ int cell_axis(float p, float o, float inv, int dim) {
    const float q = __fmul_rn(__fsub_rn(p, o), inv);
    const int c = __float2int_rd(q);
    return min(max(c, 0), dim - 1);
}

// Linear id of sub-grid cell (x, y, z), x fastest (cellHashOf).
__device__ __forceinline__ uint32_t cell_local(const GridDev& g, int x, int y, int z) {
    return uint32_t(x) + uint32_t(y) * uint32_t(g.gx) + uint32_t(z) * uint32_t(g.gx) * uint32_t(g.gy);
}

// Index of sub-grid cell (x, y, z) in the cell arrays.
__device__ __forceinline__ uint32_t cell_hash(const GridDev& g, int x, int y, int z) {
    return g.cell0 + cell_local(g, x, y, z);
}

// Cell of a position, in sub-grid coordinates (inside the sub-grid for every
// position its bounding box was built from).
__device__ __forceinline__ void cell_of(const GridDev& g, float px, float py, float pz, int& cx,
                                        int& cy, int& cz) {
    cx = cell_axis(px, g.ox, g.inv, g.dgx) - g.lx;
    cy = cell_axis(py, g.oy, g.inv, g.dgy) - g.ly;
    cz = cell_axis(pz, g.oz, g.inv, g.dgz) - g.lz;
}

__device__ __forceinline__ void decode_cell(const GridDev& g, uint32_t local, int& x, int& y, int& z) {
    const uint32_t gx = uint32_t(g.gx), gy = uint32_t(g.gy);
    x = int(local % gx);
    const uint32_t t = local / gx;
    y = int(t % gy);
    z = int(t / gy);
}

// Lower corner of sub-grid cell index c along one axis: origin + (l + c) * cellSize.
__device__ __forceinline__ float anchor_x(const GridDev& g, int c) {
    return __fmaf_rn(float(c + g.lx), g.cs, g.ox);
}
__device__ __forceinline__ float anchor_y(const GridDev& g, int c) {
    return __fmaf_rn(float(c + g.ly), g.cs, g.oy);
}
__device__ __forceinline__ float anchor_z(const GridDev& g, int c) {
    return __fmaf_rn(float(c + g.lz), g.cs, g.oz);
}

// Squared distance with one fixed rounding order, shared by the neighbour
// count and the solver so that integer outputs are reproducible.
__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// ---- SPH helpers ------------------------------------------------------------

__device__ __forceinline__ float smoothstep_f(float e0, float e1, float x) {
    float t = __fdiv_rn(__fsub_rn(x, e0), __fsub_rn(e1, e0));
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    return __fmul_rn(__fmul_rn(t, t), __fmaf_rn(-2.0f, t, 3.0f));
}

#endif  // __CUDACC__

}  // namespace mpb
