/*
 * ref_harness.h — drives the reference's compute shaders, compiled as host
 * C++ (ref_spatial.cpp, ref_constraints.cpp, ref_integrate.cpp), in the
 * dispatch order of the reference's Engine (engine/src/Engine.cpp).
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from
 * the reference sources where they lie; used to validate the FP64 oracle, to
 * generate the golden vectors under tests/golden/, and as the timed
 * reference CPU arm of the benchmark.  FP32 throughout (the shaders' own
 * arithmetic, without Metal's fast-math).
 */
#ifndef REF_HARNESS_H
#define REF_HARNESS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ref_config {
    float    bounds_min[3];   /* kBoundsMin (Engine.cpp:23)           */
    float    bounds_max[3];   /* kBoundsMax (Engine.cpp:24)           */
    float    cell;            /* kCellSize (Engine.cpp:25)            */
    float    h;               /* kSmoothingH (Engine.cpp:29)          */
    float    rest_density;    /* kRestDensity (Engine.cpp:32)         */
    float    epsilon;         /* kEpsilonCFM (Engine.cpp:35)          */
    float    damping;         /* kPBFDamping (Engine.cpp:36)          */
    float    gravity[3];      /* Engine.cpp:558                       */
    uint32_t iterations;      /* kSolverIters (Engine.cpp:39)         */
    uint32_t max_neighbors;   /* kMaxNeighborsForViz (Engine.cpp:27)  */
    uint32_t sphere;          /* 1: sphere-drop scene                 */
    float    sphere_center[3];   /* in/out, Engine.hpp:182            */
    float    sphere_velocity[3]; /* in/out, Engine.hpp:183            */
    float    sphere_radius;      /* Engine.hpp:184                    */
} ref_config;

/* Kernel loops run with OpenMP when threads > 1 (atomics then make the
 * intra-cell scatter order nondeterministic, as on the GPU). */
void     ref_set_threads(int n);
int      ref_parallel(void);
int      ref_threads(void);

/* Grid of buildSpatialBuffers (Engine.cpp:398-403); returns total cells. */
uint32_t ref_grid(const ref_config* c, uint32_t dims[3]);

/* Engine::buildSpatialHash (Engine.cpp:601-679) on pos4. */
void ref_build_spatial_hash(const ref_config* c, uint32_t n, const float* pos4, uint32_t* hashes,
                            uint32_t* cell_start, uint32_t* sorted_index, float* sorted4,
                            uint32_t* ncount);

/* Engine::step (Engine.cpp:685-811).  pos4/vel4 are updated in place; any
 * other output may be NULL.  The sphere state in *c is advanced. */
void ref_step(ref_config* c, float dt, uint32_t n, float* pos4, float* vel4, float* prev4,
              float* lambdas, uint32_t* ncount, float* foam, uint32_t* hashes,
              uint32_t* cell_start, uint32_t* sorted_index);

/* Engine::integrate (Engine.cpp:578-595), legacy integrator. */
void ref_integrate(float* pos4, float* vel4, const float gravity[3], float dt, const float bmin[3],
                   const float bmax[3], float damping, uint32_t n);

/* Engine::applyMousePulse (Engine.cpp:813-841). */
void ref_k_mouse_pulse(float* vel4, const float* pos4, const float origin[3], const float dir[3],
                       const float force[3], float radius, uint32_t count, uint32_t threads);

/* ---- per-kernel loops (one call per GPU thread id) ---- */
size_t ref_sizeof_spatial_params(void);
size_t ref_sizeof_pbf_params(void);
void ref_fill_spatial_params(void* out, const float origin[3], float cell, float inv_cell,
                             float radius_sq, uint32_t n, uint32_t total_cells,
                             const uint32_t dims[3], uint32_t max_nbr);
void ref_fill_pbf_params(void* out, const float gravity[3], float dt, const float bmin[3],
                         const float bmax[3], float h, float h2, float poly6_norm,
                         float spiky_norm, float rest_density, float epsilon, float damping,
                         uint32_t n);
void ref_k_hash_cells(const float* pos4, uint32_t* hashes, const void* sp, uint32_t threads);
void ref_k_count_cells(const uint32_t* hashes, uint32_t* counts, const void* sp, uint32_t threads);
void ref_k_scatter_particles(const uint32_t* hashes, const uint32_t* cell_start, uint32_t* cursor,
                             uint32_t* sorted_index, const void* sp, uint32_t threads);
void ref_k_gather_positions(const float* pos4, const uint32_t* sorted_index, float* sorted4,
                            const void* sp, uint32_t threads);
void ref_k_count_neighbors(const float* pos4, const uint32_t* cell_start,
                           const uint32_t* sorted_index, uint32_t* counts, const void* sp,
                           const float* sorted4, uint32_t threads);
void ref_k_predict(float* pos4, const float* vel4, float* prev4, const void* pp, uint32_t threads);
void ref_k_density_lambda(const float* sorted4, const uint32_t* cell_start,
                          const uint32_t* sorted_index, float* sorted_lambda, float* lambdas,
                          const void* sp, const void* pp, uint32_t threads);
void ref_k_apply_delta(const float* sorted4, const uint32_t* cell_start,
                       const float* sorted_lambda, float* next4, const void* sp, const void* pp,
                       uint32_t threads);
void ref_k_sphere_collision(float* buf4, const void* sp, const float center[3], float radius,
                            uint32_t threads);
void ref_k_scatter_to_original(const float* sorted4, const uint32_t* sorted_index, float* pos4,
                               const void* sp, uint32_t threads);
void ref_k_finalize(float* pos4, float* vel4, const float* prev4, const void* pp, uint32_t threads);
void ref_k_compute_foam(const float* vel4, const uint32_t* ncount, float* foam, uint32_t count,
                        float max_neighbors, uint32_t threads);

#ifdef __cplusplus
}
#endif

#endif /* REF_HARNESS_H */
