/*
 * mtlphys_b200.h — C ABI of the B200 Position-Based Fluids engine.
 *
 * This is the drop-in boundary for the simulation step of the reference
 * engine.  Every entry point below replaces one member of the reference's
 * C++ `mtlphys::Engine` class (engine/include/mtlphys/Engine.hpp) or one
 * method of its Obj-C++ bridge (app/bridge/EngineBridge.h); the citation is
 * given beside each declaration.
 *
 * Conventions
 *  - Every call returns an int status: MP_OK (0) or one of MP_ERR_*.  The
 *    reference aborts on fatal errors (engine/src/Engine.cpp:72-83, 407-413,
 *    849-854); this ABI returns a status instead and keeps a per-thread
 *    message readable with mp_last_error().
 *  - The engine owns its device buffers (like the reference owns its
 *    MTL::Buffer objects).  mp_engine_buffer() hands out borrowed device
 *    pointers; mp_engine_upload()/mp_engine_download() copy host data.
 *  - GPU work is enqueued asynchronously on the caller's CUDA stream
 *    (`mp_stream`, a cudaStream_t passed as void*; NULL = legacy default
 *    stream).  This replaces the caller-supplied MTL::CommandBuffer of the
 *    reference: step() only encodes, the caller decides when to wait.
 *    Only download, mp_engine_synchronize and mp_engine_check_errors block.
 *  - Not thread-safe: one host thread per engine (Engine.hpp:4-6).
 *  - Particle state is float4 per particle (x, y, z, w) in original
 *    particle order, as the reference's positions/velocities buffers.
 */
#ifndef MTLPHYS_B200_H
#define MTLPHYS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define MP_OK                    0
#define MP_ERR_INVALID_ARGUMENT  1   /* bad handle, size, scene id, ...        */
#define MP_ERR_OUT_OF_MEMORY     2   /* device or host allocation failed       */
#define MP_ERR_CUDA              3   /* a CUDA runtime call failed             */
#define MP_ERR_DEVICE            4   /* a kernel set the device error word     */
#define MP_ERR_SPIN_LIMIT        5   /* a bounded device-side wait gave up     */
#define MP_ERR_UNSUPPORTED       6   /* feature not available in this build    */

/* bits of the device error word (mp_engine_check_errors) */
#define MP_DEVERR_SPIN_LIMIT     0x1u  /* scan look-back / grid barrier timed out */
#define MP_DEVERR_NAN            0x2u  /* a non-finite position or velocity entered or left a step */
#define MP_DEVERR_INDEX          0x4u  /* an index check failed (debug checks)    */

/* ---- scenes: Engine.hpp:37-39 ------------------------------------------- */
#define MP_SCENE_CUBE_DROP    0u
#define MP_SCENE_DAM_BREAK    1u
#define MP_SCENE_SPHERE_DROP  2u

/* ---- buffers: Engine.hpp:83-90 accessors (+ foam, sorted state) --------- */
#define MP_BUF_POSITIONS        0u  /* float4[N]  positionsBuffer()      */
#define MP_BUF_VELOCITIES       1u  /* float4[N]  velocitiesBuffer()     */
#define MP_BUF_PREV_POSITIONS   2u  /* float4[N]  prevPositionsBuffer()  */
#define MP_BUF_CELL_HASHES      3u  /* uint32[N]  cellHashesBuffer()     */
#define MP_BUF_CELL_START       4u  /* uint32[C+1] cellStartBuffer()     */
#define MP_BUF_SORTED_INDEX     5u  /* uint32[N]  sortedIndexBuffer()    */
#define MP_BUF_NEIGHBOR_COUNTS  6u  /* uint32[N]  neighborCountsBuffer() */
#define MP_BUF_LAMBDAS          7u  /* float[N]   lambdasBuffer()        */
#define MP_BUF_FOAM             8u  /* float[N]   _foamIntensity         */
#define MP_BUF_SORTED_POSITIONS 9u  /* float4[N]  _sortedPositions (hash-time gather) */
#define MP_BUF_COUNT           10u

typedef void* mp_stream;             /* cudaStream_t */
typedef struct mp_engine mp_engine;  /* opaque */

/*
 * Simulation parameters.  The reference hard-codes these as constexpr
 * tunables (engine/src/Engine.cpp:22-39, 551-572) and as literals inside its
 * shaders (engine/shaders/Constraints.metal:158-160, 190, 297, 325, 341-347);
 * here every one of them is a field.  mp_default_params() fills the
 * reference's values.  `size` must be sizeof(mp_pbf_params).
 */
typedef struct mp_pbf_params {
    uint32_t size;               /* sizeof(mp_pbf_params)                          */
    uint32_t solver_iterations;  /* kSolverIters = 5      (Engine.cpp:39)          */
    float    h;                  /* kSmoothingH = 0.10    (Engine.cpp:29)          */
    float    cell_size;          /* kCellSize = 0.10      (Engine.cpp:25)          */
    float    rest_density;       /* kRestDensity = 8000   (Engine.cpp:32)          */
    float    epsilon;            /* kEpsilonCFM = 800     (Engine.cpp:35)          */
    float    damping;            /* kPBFDamping = 0.996   (Engine.cpp:36)          */
    float    gravity[3];         /* (0,-9.81,0)           (Engine.cpp:558)         */
    float    bounds_min[3];      /* kBoundsMin (-3,-3,-3) (Engine.cpp:23)          */
    float    bounds_max[3];      /* kBoundsMax (3,6,3)    (Engine.cpp:24)          */
    float    scorr_k;            /* kSCorrK = 1e-4        (Constraints.metal:158)  */
    uint32_t scorr_n;            /* ratio^4               (Constraints.metal:179)  */
    float    scorr_dq;           /* 0.2 (x h)             (Constraints.metal:159)  */
    float    max_delta;          /* 0.3 (x h)             (Constraints.metal:190)  */
    float    vmax;               /* 1.0 (x h/dt)          (Constraints.metal:347)  */
    float    wall_eps;           /* 1e-3                  (Constraints.metal:325)  */
    float    floor_friction;     /* 0.55                  (Constraints.metal:341)  */
    float    wall_friction;      /* 0.97                  (Constraints.metal:344)  */
    float    foam_max_neighbors; /* kMaxNeighborsForViz=96 (Engine.cpp:27, 806)   */
    float    foam_speed_lo;      /* 1.2                   (Constraints.metal:297)  */
    float    foam_speed_hi;      /* 4.5                   (Constraints.metal:297)  */
    float    sphere_radius;      /* 0.6                   (Engine.hpp:184)         */
    float    sphere_gravity;     /* -9.81                 (Engine.cpp:694)         */
    float    sphere_drag;        /* 0.998 per step        (Engine.cpp:695-697)     */
    float    sphere_restitution; /* 0.4                   (Engine.cpp:702-707)     */
    float    integrate_damping;  /* 0.999 legacy integrator (Engine.cpp:584)      */
    float    integrate_restitution; /* 0.4                (Integrate.metal:29)      */
    float    mouse_falloff;      /* 0.4: exp(-r^2/(R^2 f)) (Constraints.metal:250)  */
} mp_pbf_params;

/*
 * Scene description for mp_engine_reset_scene().  With lattice == 0 the
 * reference's own placement for the scene is used (Engine.cpp:454-549).
 * With lattice == 1 particles are placed on a dims[0] x dims[1] x dims[2]
 * lattice with lower corner `origin`, x fastest, then z, then y (the
 * reference's loop order), each component jittered by a uniform value in
 * [-jitter, +jitter) drawn from std::mt19937_64(seed) as
 * ((draw >> 11) * 2^-53 * 2 - 1) * jitter, x then y then z per particle.
 * `size` must be sizeof(mp_scene_desc).
 */
typedef struct mp_scene_desc {
    uint32_t size;
    uint32_t lattice;            /* 0: reference placement, 1: explicit lattice   */
    uint64_t seed;               /* jitter seed                                   */
    uint32_t dims[3];            /* lattice counts along x, y, z                  */
    float    origin[3];          /* lattice lower corner                          */
    float    spacing;            /* lattice spacing (0 -> 0.5 h, Engine.cpp:457)  */
    float    jitter;             /* absolute jitter amplitude per component       */
    float    sphere_center[3];   /* scene 2: sphere start (Engine.cpp:523-525)    */
    float    sphere_velocity[3]; /* scene 2: sphere start velocity (0 in ref)     */
} mp_scene_desc;

/* ---- library ------------------------------------------------------------ */
/* Last error message of the calling thread ("" if none). */
const char* mp_last_error(void);
/* ABI version: increases when a struct or signature changes. */
uint32_t mp_abi_version(void);
/* Reference defaults: Engine.cpp:22-39, 551-572; Constraints.metal literals. */
int mp_default_params(mp_pbf_params* out);
/* Defaults for mp_scene_desc (reference placement). */
int mp_default_scene_desc(mp_scene_desc* out);
/* Rest density of an interior lattice site at `spacing` for smoothing length
 * h: FP64 sum of Poly6 over the lattice (the quantity Engine.cpp:30-31
 * approximates as ~8072 before hard-coding 8000). */
double mp_lattice_rest_density(double h, double spacing);

/* ---- failure handling (no reference counterpart: the reference aborts the
 *      process, engine/src/Engine.cpp:72-83, 407-413, 849-854, and creates its
 *      buffers unchecked, :390-395) ------------------------------------------
 * Device allocations.  Every device buffer of engines and batches is made by
 * `alloc` and given back with `free_fn` (the one that made it, even after the
 * allocator is replaced, and only once the device is idle).  alloc returns 0
 * and a device pointer on `device`, or non-zero when it cannot: the call that
 * needed the memory then returns MP_ERR_OUT_OF_MEMORY and leaves the engine or
 * batch empty (no particles; steps do nothing) but usable: a later reset
 * allocates again.  NULL restores cudaMalloc / cudaFree.  Process-wide;
 * install it before the calls whose allocations it should see. */
typedef int (*mp_device_alloc_fn)(void** ptr, size_t bytes, int device, void* user);
typedef void (*mp_device_free_fn)(void* ptr, int device, void* user);
int mp_set_device_allocator(mp_device_alloc_fn alloc, mp_device_free_fn free_fn, void* user);
/* Bound, in polls, of every device-side wait of kernels enqueued after the
 * call: the scan's decoupled look-back and the batch kernel's grid barrier
 * (each poll naps 32-64 ns).  0 restores the defaults (2^22 and 2^24 polls).
 * A wait that runs out sets MP_DEVERR_SPIN_LIMIT instead of hanging; see
 * mp_exclusive_scan_status and mp_batch_check_errors.  Process-wide; engines
 * and batches re-capture their CUDA graphs at their next step. */
int mp_set_spin_limit(uint32_t polls);

/* ---- engine lifetime: Engine.hpp:29-30, 41-44 ---------------------------- */
/* Engine(MTL::Device*) — binds `device`, then reset(200'000) like
 * Engine.cpp:97-102. */
int mp_engine_create(int device, mp_engine** out);
/* ~Engine() (Engine.cpp:104-123). NULL is accepted. */
int mp_engine_destroy(mp_engine* e);
/* Replaces the constexpr tunables; takes effect at the next reset/step
 * (a change of bounds or cell size re-derives the grid at the next reset). */
int mp_engine_set_params(mp_engine* e, const mp_pbf_params* p);
int mp_engine_get_params(const mp_engine* e, mp_pbf_params* out);
/* reset(particleCount) — keeps the current scene (Engine.cpp:125-127). */
int mp_engine_reset(mp_engine* e, uint32_t n);
/* reset(particleCount, sceneIdx) (Engine.cpp:129-134); desc may be NULL. */
int mp_engine_reset_scene(mp_engine* e, uint32_t n, uint32_t scene, const mp_scene_desc* desc);

/* ---- simulation: Engine.hpp:52, 56 --------------------------------------- */
/* step(cmd, dt): predict -> spatial hash -> K solver iterations -> scatter
 * back -> finalize -> foam (Engine.cpp:685-811).  dt <= 0 is a no-op that
 * returns MP_OK (Engine.cpp:686). */
int mp_engine_step(mp_engine* e, float dt, mp_stream stream);
/* buildSpatialHash(cmd): hash, count, scan, scatter, gather, neighbour
 * count of the current positions (Engine.cpp:601-679).  The intra-cell
 * order of sortedIndex is ascending particle index (deterministic). */
int mp_engine_build_spatial_hash(mp_engine* e, mp_stream stream);
/* Capture step() into a CUDA graph and replay it (1) or launch kernel by
 * kernel (0, default).  Results are identical either way. */
int mp_engine_set_graph_mode(mp_engine* e, int enable);

/* ---- tracing (no reference counterpart: the reference reads only
 *      command-buffer timestamps, tests/bench_engine.cpp:43) ---------------- */
typedef struct mp_kernel_time {
    char     name[32];   /* kernel kind, e.g. "lambda", "delta", "scan"   */
    uint32_t launches;   /* launches timed since the last read            */
    double   ms;         /* total device time of those launches           */
} mp_kernel_time;
/* Time every kernel the engine launches with CUDA events on its stream
 * (1), or stop (0).  While profiling, step() runs kernel by kernel, or, in
 * graph mode, as one graph captured with the timing events as event nodes
 * (instantiated per step; the times then exclude the host's launch gaps). */
int mp_engine_set_profiling(mp_engine* e, int enable);
/* Wait for the timed work and return per-kernel totals (up to `capacity`
 * entries; *count = number of kernel kinds); the totals are then cleared. */
int mp_engine_kernel_times(mp_engine* e, mp_kernel_time* out, uint32_t capacity, uint32_t* count);
/* Kernel launches one step() issues for `iterations` solver iterations. */
uint32_t mp_step_launch_count(uint32_t iterations);

/* ---- queries: Engine.hpp:44, 78-80 --------------------------------------- */
uint32_t mp_engine_particle_count(const mp_engine* e);
uint32_t mp_engine_total_cells(const mp_engine* e);
float    mp_engine_cell_size(const mp_engine* e);
uint32_t mp_engine_current_scene(const mp_engine* e);
/* Grid dimensions of the spatial hash (SpatialParams::gridDim, Shared.h:47). */
int mp_engine_grid_dims(const mp_engine* e, uint32_t dims[3]);

/* ---- buffers: Engine.hpp:83-90 ------------------------------------------- */
/* Borrowed device pointer and byte size of buffer `which` (MP_BUF_*). */
int mp_engine_buffer(mp_engine* e, uint32_t which, void** dptr, size_t* bytes);
/* Copy `count` elements (float4, uint32 or float per the buffer's type)
 * between host memory and buffer `which`.  upload is ordered on `stream`
 * and returns once the host memory may be reused; download synchronizes. */
int mp_engine_upload(mp_engine* e, uint32_t which, const void* host, size_t count, mp_stream stream);
int mp_engine_download(mp_engine* e, uint32_t which, void* host, size_t count, mp_stream stream);
/* Engine::integrate(cmd, dt) (Engine.cpp:578-596, Integrate.metal:11-42): the
 * legacy semi-implicit Euler step with box bounds, kept by the reference for
 * its integrator tests: v = (v + g dt) * integrate_damping, p += v dt, then
 * per axis a position outside [bounds_min, bounds_max] is clamped and its
 * velocity reflected with integrate_restitution.  Asynchronous on `stream`;
 * dt <= 0 is a no-op. */
int mp_engine_integrate(mp_engine* e, float dt, mp_stream stream);
/* Engine::applyMousePulse(cmd, rayOrigin, rayDir, force, radius)
 * (Engine.cpp:813-841, Constraints.metal:231-253): every particle in front of
 * the ray origin within `radius` of the ray (ray_dir normalized by the
 * caller) gets force * exp(-r^2 / (radius^2 mouse_falloff)) added to its
 * velocity.  Asynchronous on `stream`. */
int mp_engine_apply_mouse_pulse(mp_engine* e, const float ray_origin[3], const float ray_dir[3],
                                const float force[3], float radius, mp_stream stream);
/* ---- headless rendering: Engine::render (Engine.cpp:884-1020) ------------
 * The reference draws its particles with a Metal screen-space-fluid pipeline
 * (engine/shaders/Render.metal) into the app's drawable.  Here the same
 * passes run as CUDA kernels into device image buffers, no graphics API:
 * sphere-billboard depth (closest wins) and additive thickness, a masked
 * 9x9 Gaussian of the depth, the composite (normals from screen derivatives,
 * reflected / refracted procedural sky, Beer-Lambert absorption, Schlick
 * Fresnel, sun glint), then the box wireframe, the sphere (scene 2) and foam
 * sprites.  The output is linear RGBA float in [0, 1] per pixel, row-major
 * with y = 0 on the top row (the reference's target stores the same values
 * as 8-bit sRGB). */
typedef struct mp_render_params {
    uint32_t size;               /* sizeof(mp_render_params)                     */
    uint32_t width, height;      /* pixels                                       */
    uint32_t flags;              /* MP_RENDER_* passes after the composite       */
    float    eye[3], target[3];  /* lookAt(eye, target, +y)  (Engine.cpp:894-899) */
    float    fov_y;              /* 1.0 rad                  (Engine.cpp:893)    */
    float    z_near, z_far;      /* 0.1, 100                 (Engine.cpp:900)    */
    float    particle_radius;    /* 0.022 * 1.3              (Engine.cpp:26, 902) */
    float    foam_radius_scale;  /* 0.25                     (Render.metal:363)  */
} mp_render_params;
#define MP_RENDER_BOX     1u  /* bounding-box wireframe (Engine.cpp:985-995)  */
#define MP_RENDER_SPHERE  2u  /* the sphere, scene 2 only (:997-1008)          */
#define MP_RENDER_FOAM    4u  /* foam sprites (:1010-1018)                     */
/* Image buffers of the last render (mp_engine_render_buffer). */
#define MP_RENDER_BUF_COLOR     0u  /* float4[W*H] linear RGBA                    */
#define MP_RENDER_BUF_DEPTH     1u  /* float[W*H]  closest view distance, 3.39e38 = none */
#define MP_RENDER_BUF_SMOOTHED  2u  /* float[W*H]  smoothed view distance, 0 = none */
#define MP_RENDER_BUF_THICKNESS 3u  /* float[W*H]  summed thickness              */
#define MP_RENDER_BUF_NDC_DEPTH 4u  /* float[W*H]  NDC depth of the final image  */
/* Defaults: 1280 x 720, the app's start-up orbit camera
 * (app/MetalView.swift:93-96), all passes. */
int mp_default_render_params(mp_render_params* rp);
/* The camera matrices of a render (column-major 4x4): no GPU needed. */
int mp_render_camera(const mp_render_params* rp, float view[16], float proj[16]);
/* Render the engine's current particles.  rgba: device buffer of
 * width * height float4 to receive the image, or NULL (then read it with
 * mp_engine_render_buffer).  Asynchronous on `stream`. */
int mp_engine_render(mp_engine* e, const mp_render_params* rp, float* rgba, mp_stream stream);
int mp_engine_render_buffer(mp_engine* e, uint32_t which, void** dptr, size_t* bytes);
/* Sphere state of scene 2 (Engine.hpp:182-184). */
int mp_engine_set_sphere(mp_engine* e, const float center[3], const float velocity[3], float radius);
int mp_engine_get_sphere(mp_engine* e, float center[3], float velocity[3], float* radius);
/* Wait for the engine's queued work and report the device error word
 * (MP_DEVERR_* in *bits, may be NULL); the word is cleared. */
int mp_engine_check_errors(mp_engine* e, uint32_t* bits);
int mp_engine_synchronize(mp_engine* e);

/* ---- batch of independent scenes (no reference counterpart: the reference
 *      steps one scene per Engine) -------------------------------------------
 * All scenes advance in one persistent, cooperative launch per step (or, in
 * serial mode, the same kernel launched once per scene).  Each scene has its
 * own parameters, dt, seeding and sphere, and gives the results a
 * single-scene engine would give (the same particle order and arithmetic).
 * Particles of scene s are the contiguous range mp_batch_scene_range(s) of
 * the batch's buffers (MP_BUF_* as for an engine; MP_BUF_CELL_START holds the
 * scenes' bounding boxes of cells laid end to end). */
typedef struct mp_batch mp_batch;
typedef struct mp_batch_tuning {
    uint32_t block;          /* threads per block: 128, 256 or 512     */
    uint32_t blocks_per_sm;  /* resident blocks per SM of the launch   */
    float    ms_per_step;    /* measured by mp_batch_autotune          */
} mp_batch_tuning;
int mp_batch_create(int device, mp_batch** out);
int mp_batch_destroy(mp_batch* b);
/* nscenes scenes: counts[s] particles, scene_ids[s] (MP_SCENE_*, NULL = cube
 * drop), params[s], descs[s] (NULL = reference placement), dts[s] > 0.  All
 * scenes use the same solver_iterations. */
int mp_batch_reset(mp_batch* b, uint32_t nscenes, const uint32_t* counts, const uint32_t* scene_ids,
                   const mp_pbf_params* params, const mp_scene_desc* descs, const float* dts);
int mp_batch_set_dts(mp_batch* b, const float* dts);
/* One step of every scene, asynchronous on `stream`. */
int mp_batch_step(mp_batch* b, mp_stream stream);
/* 0: one launch for all scenes (default); 1: the same kernel once per scene. */
int mp_batch_set_mode(mp_batch* b, int serial);
/* Capture a step into a CUDA graph and replay it (1), or launch directly (0). */
int mp_batch_set_graph_mode(mp_batch* b, int enable);
/* Launch shape (block = 128/256/512, blocks_per_sm 0 = as many as fit). */
int mp_batch_set_launch(mp_batch* b, uint32_t block, uint32_t blocks_per_sm);
int mp_batch_get_launch(const mp_batch* b, uint32_t* block, uint32_t* blocks);
/* Time `steps` steps for every launch shape from the same saved state
 * (restored afterwards), keep the fastest, and remember it for batches of
 * the same scene count and particle-count bucket.  Results are identical for
 * every shape. */
int mp_batch_autotune(mp_batch* b, uint32_t steps, mp_batch_tuning* best);
uint32_t mp_batch_scene_count(const mp_batch* b);
uint32_t mp_batch_particle_count(const mp_batch* b);
int mp_batch_scene_range(const mp_batch* b, uint32_t scene, uint32_t* first, uint32_t* count);
int mp_batch_buffer(mp_batch* b, uint32_t which, void** dptr, size_t* bytes);
int mp_batch_upload(mp_batch* b, uint32_t which, const void* host, size_t count, mp_stream stream);
int mp_batch_download(mp_batch* b, uint32_t which, void* host, size_t count, mp_stream stream);
int mp_batch_set_sphere(mp_batch* b, uint32_t scene, const float center[3], const float velocity[3],
                        float radius);
int mp_batch_get_sphere(mp_batch* b, uint32_t scene, float center[3], float velocity[3], float* radius);
/* Replace scene `scene`'s parameters; the box, cell size and
 * solver_iterations must stay the same (the hash grid does not change). */
int mp_batch_set_params(mp_batch* b, uint32_t scene, const mp_pbf_params* params);
int mp_batch_get_params(const mp_batch* b, uint32_t scene, mp_pbf_params* params);
/* Wait for the batch's queued work and report its device error word (as
 * mp_engine_check_errors).  When a grid barrier gave up (MP_ERR_SPIN_LIMIT),
 * the launch left every block at its next barrier, so the state of that step
 * is invalid, and every step after it did nothing; this call re-arms the
 * batch, which steps again from its (invalid) state: restore or reset it. */
int mp_batch_check_errors(mp_batch* b, uint32_t* bits);
/* Test hook: every grid barrier of the following steps waits for `extra`
 * more blocks than the launch has (0 = normal), so every wait runs out after
 * the mp_set_spin_limit bound.  For failure-path tests only. */
int mp_batch_debug_barrier_extra(mp_batch* b, uint32_t extra);

/* ---- differentiable rollouts (no reference counterpart: the reference
 *      engine is not differentiable) ------------------------------------------
 * mp_batch_rollout_forward advances every scene `steps` steps (as
 * mp_batch_step would) and keeps a checkpoint of the state (positions,
 * velocities, spheres) every `checkpoint_every` steps.
 * mp_batch_rollout_backward then takes dL/d(final positions) and dL/d(final
 * velocities) (device arrays of N float4, w ignored; NULL = zero) and writes
 * dL/d(initial positions), dL/d(initial velocities) (N float4) and, per scene,
 * MP_SCENE_GRADS doubles (MP_GRAD_*): dL/d s_corr k and dL/d the initial
 * sphere center, velocity and radius.  It recomputes each segment between
 * checkpoints with every step recorded (neighbour lists, iterates,
 * corrections) and runs the adjoint kernels over it in reverse, the
 * neighbour topology and clamp states of each step held fixed.  Outputs may
 * be NULL.  The state is left at the end of the rollout; the scratch buffers
 * (MP_BUF_PREV, cell and sort arrays, lambdas) then hold values of the
 * recomputation.  All work is asynchronous on `stream`.  Any other call that
 * changes the state (step, upload, set_sphere, set_params, set_dts, reset)
 * ends the rollout: a later backward call fails with MP_ERR_INVALID_ARGUMENT.
 * Hash grids must be at most 2048 x 2048 x 1024 cells (MP_ERR_UNSUPPORTED). */
#define MP_SCENE_GRADS   8
#define MP_GRAD_SCORR_K  0
#define MP_GRAD_CENTER   1 /* 3 values */
#define MP_GRAD_VELOCITY 4 /* 3 values */
#define MP_GRAD_RADIUS   7
int mp_batch_rollout_forward(mp_batch* b, uint32_t steps, uint32_t checkpoint_every, mp_stream stream);
int mp_batch_rollout_backward(mp_batch* b, const float* dpos, const float* dvel, float* dpos0,
                              float* dvel0, double* dscene, mp_stream stream);
/* Kernel launches of a backward pass over `steps` steps (recomputation
 * included). */
uint32_t mp_batch_rollout_launch_count(const mp_batch* b, uint32_t steps);

/* ---- state snapshots (no reference counterpart: the reference keeps its
 *      state only in its Metal buffers) ------------------------------------------
 * A snapshot is a self-describing byte string: a 64-byte header ("MTLPSNAP",
 * version, kind, scene and particle counts, struct sizes), one record per
 * scene (mp_pbf_params, mp_scene_desc, scene id, particle count, dt, sphere
 * center/velocity/radius), then every particle's position and velocity
 * (float4, original order).  *_snapshot_size gives the bytes needed;
 * *_snapshot waits for queued work and copies the state into `host`;
 * *_restore re-creates the engine or batch from a snapshot (parameters,
 * scenes, buffers, state), after which stepping continues exactly as from
 * the saved state.  mtlphys_b200/snapshot.py reads and writes the format. */
size_t mp_engine_snapshot_size(const mp_engine* e);
int mp_engine_snapshot(mp_engine* e, void* host, size_t bytes);
int mp_engine_restore(mp_engine* e, const void* host, size_t bytes);
size_t mp_batch_snapshot_size(const mp_batch* b);
int mp_batch_snapshot(mp_batch* b, void* host, size_t bytes);
int mp_batch_restore(mp_batch* b, const void* host, size_t bytes);

/* ---- scan: Engine.hpp:92-100 --------------------------------------------- */
/* runExclusiveScan(cmd, in, out, chunkSums, n) (Engine.cpp:843-882): out[i]
 * = sum of in[0..i) modulo 2^32, single pass with decoupled look-back; no
 * 1024^2 length cap.  `in` and `out` are device pointers; `scratch` is a
 * device buffer of at least mp_exclusive_scan_scratch_bytes(n) bytes.
 * n == 0 is a no-op (Engine.cpp:848).  in == out is allowed. */
size_t mp_exclusive_scan_scratch_bytes(uint32_t n);
int mp_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n,
                      void* scratch, size_t scratch_bytes, mp_stream stream);
/* Waits for `stream` and reports whether the last scan that used `scratch`
 * (NULL: the static scratch of mp_exclusive_scan_noalloc) completed:
 * MP_ERR_SPIN_LIMIT when its look-back wait gave up (that scan's output is
 * wrong), MP_OK otherwise; the error word is cleared.  The scans themselves
 * are asynchronous and return MP_OK once enqueued. */
int mp_exclusive_scan_status(const void* scratch, mp_stream stream);
/* Test hook: mp_exclusive_scan with the tile ticket starting at
 * `first_ticket`.  A ticket that is not a multiple of the tile count splits
 * the tiles across two epochs, so the look-back of the first tile launched
 * waits for descriptors no tile writes and gives up after the
 * mp_set_spin_limit bound.  For failure-path tests only. */
int mp_debug_exclusive_scan_from_ticket(const uint32_t* in, uint32_t* out, uint32_t n, void* scratch,
                                        size_t scratch_bytes, uint64_t first_ticket, mp_stream stream);

/* The same exclusive scan without any device allocation, for callers that
 * cannot allocate when they need it (a frame loop with a fixed per-frame
 * memory budget, a host framework whose allocator owns the device heap).
 * It has no counterpart in the reference.  Its scratch is a 33,024-byte
 * static device array held by every GPU that loads this library, which
 * limits n to 16,777,216 (2^24) elements: larger n returns
 * MP_ERR_INVALID_ARGUMENT.  `in` and `out` are device pointers on the current
 * device.  The first call on each device looks up the array's address (set-up
 * with that device current); make that first call before any stream capture.
 * Calls outside stream capture look the address up again, so it follows a
 * device reset.  A look-back that gives up is reported by
 * mp_exclusive_scan_status(NULL, stream).
 * All calls share the one array, so calls that overlap on the GPU (other
 * streams, other host threads) race: order them on one stream. */
int mp_exclusive_scan_noalloc(const uint32_t* in, uint32_t* out, uint32_t n, mp_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* MTLPHYS_B200_H */
