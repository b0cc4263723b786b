/*
 * pbf_oracle.h — CPU oracle for the PBF simulation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: only the tests, the smoke
 * check and the CPU-baseline leg of the benchmark load it.  The product path
 * (libmtlphys_b200.so) never links or calls it.
 *
 * It restates, in FP64, the reference engine's simulation step
 * (engine/src/Engine.cpp:685-811) and spatial hash (Engine.cpp:601-679) from
 * the shader sources engine/shaders/Spatial.metal and Constraints.metal.
 * The integer outputs (cell hashes, cell starts, sorted order, neighbour
 * counts) are computed in FP32 with the exact operation order the CUDA path
 * uses, so they are bit-exact references; the solver (densities, lambdas,
 * position corrections, finalize, foam) runs in FP64.
 *
 * Parity is pinned by the reference's own shader code compiled as C++
 * (oracle/ref, built into oracle/_ref/) and by the golden vectors in
 * tests/golden/ generated from it.
 */
#ifndef PBF_ORACLE_H
#define PBF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/mtlphys_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Uniform grid of the spatial hash: SpatialParams (Shared.h:40-49) as the
 * reference derives it in buildSpatialBuffers (Engine.cpp:398-452). */
typedef struct or_grid {
    float    origin[3];   /* = bounds_min                        */
    float    cell;        /* cell size                           */
    float    inv_cell;    /* 1.0f / cell in FP32 (Engine.cpp:446) */
    uint32_t dims[3];     /* ceil(extent / cell) in FP32          */
    uint32_t cells;       /* dims.x * dims.y * dims.z             */
} or_grid;

int  or_make_grid(const mp_pbf_params* p, or_grid* g);

/* cellCoordOf + cellHashOf (Spatial.metal:35-43) on FP32 positions. */
void or_hash_f32(const float* pos4, uint32_t n, const or_grid* g, uint32_t* hashes);
/* cpuExclusiveScan (tests/TestUtils.hpp:52-61), modulo 2^32. */
void or_exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n);
/* countCells + scan + scatterParticles (Spatial.metal:63-180) with the
 * intra-cell order fixed to ascending particle index (stable sort). */
void or_counting_sort(const uint32_t* hashes, uint32_t n, uint32_t cells,
                      uint32_t* cell_start /* cells+1 */, uint32_t* sorted_index);
/* countNeighbors (Spatial.metal:207-243) in FP32: j != i in the 27 cells
 * around i's cell with |p_j - p_i|^2 < r2max, r^2 = fma(dz,dz,fma(dy,dy,dx*dx)). */
void or_count_neighbors_f32(const float* pos4, uint32_t n, const or_grid* g, float r2max,
                            const uint32_t* cell_start, const uint32_t* sorted_index,
                            uint32_t* counts);
/* predictPositions (Constraints.metal:54-66) in FP32 with the product's
 * rounding: v' = fma(g, dt, v), p' = fma(v', dt, p), w kept. */
void or_predict_f32(const float* pos4, const float* vel4, uint32_t n, const float g[3],
                    float dt, float* pred4);

/* Scene seeding of Engine::seedParticles (Engine.cpp:454-549) and the
 * explicit jittered lattice of mp_scene_desc.  Writes n float4 positions
 * (w = 1); returns 0 or MP_ERR_INVALID_ARGUMENT. */
int or_seed_scene(const mp_pbf_params* p, uint32_t scene, const mp_scene_desc* d,
                  uint32_t n, float* pos4);

/* Engine::integrate (Engine.cpp:578-596, Integrate.metal:11-42) in FP32, in
 * place on n float4 positions / velocities. */
void or_integrate_f32(const mp_pbf_params* p, float dt, uint32_t n, float* pos4, float* vel4);
/* Engine::applyMousePulse (Engine.cpp:813-841, Constraints.metal:231-253) in
 * FP32, in place on n float4 velocities. */
void or_mouse_pulse_f32(const mp_pbf_params* p, const float origin[3], const float dir[3],
                        const float force[3], float radius, uint32_t n, const float* pos4,
                        float* vel4);

/* Sphere kinematics of Engine::step (Engine.cpp:693-712) in FP64.
 * s = {cx, cy, cz, vx, vy, vz, radius}. */
void or_sphere_advance(const mp_pbf_params* p, double dt, double* s);

/* Outputs of one step.  Any pointer may be NULL. */
typedef struct or_step_out {
    double*   pos3;          /* final positions, original order, xyz         */
    double*   vel3;          /* final velocities                              */
    double*   lambda;        /* last iteration's lambda per particle          */
    double*   foam;          /* foam intensity                                */
    uint32_t* neighbor_counts;
    uint32_t* hashes;        /* N                                             */
    uint32_t* cell_start;    /* cells + 1                                     */
    uint32_t* sorted_index;  /* N                                             */
    float*    pred4;         /* FP32 predicted positions the hash was built on */
} or_step_out;

/*
 * One Engine::step in FP64 from an FP32 particle state (float4 x n).
 *   sphere: NULL unless the scene is the sphere drop; advanced in place.
 * The hash is built on FP32 predicted positions (or_predict_f32) so that its
 * integer outputs match the CUDA path bit for bit, and the FP64 solver starts
 * from those same FP32 predicted positions (the reference computes its
 * prediction in FP32; everything after it is FP64 here).
 */
int or_step(const mp_pbf_params* p, float dt, uint32_t n, const float* pos4, const float* vel4,
            double* sphere, or_step_out* out);

/*
 * One step with an FP64 state (xyz triples) in and out: the prediction is
 * FP64 and the hash is built on it rounded to FP32.  Used for FP64 rollouts
 * (finite differences of the adjoint).  pos3/vel3 are updated in place.
 */
int or_step_f64(const mp_pbf_params* p, double dt, uint32_t n, double* pos3, double* vel3,
                double* sphere);

/* Number of OpenMP threads the oracle uses (0 -> runtime default). */
/* Test hook: plant a deliberate mistake in the oracle's step so that a test
 * can show the parity checks reject it.  1: the density starts at the
 * particle's own W(0) only when its slot lies in the stencil of its current
 * cell (instead of always, Constraints.metal:99-108).  0: none. */
void or_plant_fault(int which);
void or_set_threads(int n);
int  or_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* PBF_ORACLE_H */
