// engine.cpp — the C++ Engine behind the C ABI of include/mtlphys_b200.h.
//
// Host-side counterpart of the reference's mtlphys::Engine
// (engine/include/mtlphys/Engine.hpp, engine/src/Engine.cpp): it owns the
// particle and hash buffers on one GPU, seeds the three scenes, derives the
// per-step constants from mp_pbf_params, and enqueues the sm_100a kernels of
// pbf_hash.cu / pbf_solver.cu on the caller's CUDA stream (the reference
// encodes Metal dispatches into the caller's command buffer).  Optionally the
// whole step is captured once into a CUDA graph and replayed.
#include "../../include/mtlphys_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "host_common.h"
#include "pbf_render.h"
#include "snapshot.h"
#include "pbf_kernels.h"

using namespace mpb;
using mpb::DevState;
using mpb::GridDev;
using mpb::StepConsts;

namespace mpb {

constexpr uint32_t kAbiVersion = 1;
constexpr float kPi = 3.14159265358979323846f;
constexpr uint32_t kPad = 256;  // Engine.cpp:19 pads buffers to the threadgroup size

namespace {
thread_local std::string g_err;
}  // namespace

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// Lets the other translation units of the library report through
// mp_last_error().
void record_error(const char* msg) { g_err = msg; }

const char* last_error() { return g_err.c_str(); }

// ---- bounds of the device-side waits (mp_set_spin_limit) --------------------
namespace {
std::atomic<uint32_t> g_scan_spins{kDefaultScanSpinLimit};
std::atomic<uint32_t> g_barrier_spins{kDefaultBarrierSpinLimit};
std::atomic<uint32_t> g_spin_epoch{0};
}  // namespace

uint32_t scan_spin_limit() { return g_scan_spins.load(); }
uint32_t barrier_spin_limit() { return g_barrier_spins.load(); }
uint32_t spin_limit_epoch() { return g_spin_epoch.load(); }

// ---- device allocations (mp_set_device_allocator) ---------------------------
namespace {
struct Allocator {
    mp_device_alloc_fn alloc = nullptr;  // nullptr: cudaMalloc / cudaFree
    mp_device_free_fn free = nullptr;
    void* user = nullptr;
};
std::mutex g_alloc_lock;
Allocator g_alloc;
// who made each live block (it is given back to the same allocator)
std::unordered_map<void*, std::pair<Allocator, int>> g_blocks;
}  // namespace

int dev_alloc(void** p, size_t bytes, int device) {
    *p = nullptr;
    Allocator a;
    {
        std::lock_guard<std::mutex> lock(g_alloc_lock);
        a = g_alloc;
    }
    void* ptr = nullptr;
    if (a.alloc) {
        if (a.alloc(&ptr, bytes, device, a.user) != 0 || !ptr)
            return fail(MP_ERR_OUT_OF_MEMORY, "device allocator refused %zu bytes on device %d", bytes,
                        device);
    } else {
        const cudaError_t e = cudaMalloc(&ptr, bytes);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? MP_ERR_OUT_OF_MEMORY : MP_ERR_CUDA,
                        "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    std::lock_guard<std::mutex> lock(g_alloc_lock);
    g_blocks[ptr] = {a, device};
    *p = ptr;
    return MP_OK;
}

void dev_free(void* p) {
    if (!p) return;
    std::pair<Allocator, int> owner;
    {
        std::lock_guard<std::mutex> lock(g_alloc_lock);
        auto it = g_blocks.find(p);
        if (it == g_blocks.end()) return;
        owner = it->second;
        g_blocks.erase(it);
    }
    if (owner.first.alloc) {
        // a caller's allocator may hand the block out again at once: give it
        // back only when no queued kernel can still use it (cudaFree waits
        // by itself)
        DeviceGuard g(owner.second);
        cudaDeviceSynchronize();
        if (owner.first.free) owner.first.free(p, owner.second, owner.first.user);
    } else {
        cudaFree(p);
    }
}

// Grid of buildSpatialBuffers (Engine.cpp:398-403, 443-451).
int make_grid(const mp_pbf_params& p, GridDev& g) {
    if (!(p.cell_size > 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "cell_size must be > 0");
    uint64_t cells = 1;
    uint32_t dims[3];
    for (int a = 0; a < 3; ++a) {
        const float extent = p.bounds_max[a] - p.bounds_min[a];
        const float d = std::ceil(extent / p.cell_size);
        if (!(d >= 1.0f) || d > 65536.0f)
            return fail(MP_ERR_INVALID_ARGUMENT, "bounds/cell_size give grid dimension %g on axis %d",
                        double(d), a);
        dims[a] = uint32_t(d);
        cells *= dims[a];
    }
    if (cells >= (1ull << 31))
        return fail(MP_ERR_INVALID_ARGUMENT, "grid of %llu cells is too large",
                    static_cast<unsigned long long>(cells));
    g.ox = p.bounds_min[0];
    g.oy = p.bounds_min[1];
    g.oz = p.bounds_min[2];
    g.inv = 1.0f / p.cell_size;
    g.cs = p.cell_size;
    g.gx = g.dgx = int(dims[0]);
    g.gy = g.dgy = int(dims[1]);
    g.gz = g.dgz = int(dims[2]);
    g.lx = g.ly = g.lz = 0;
    g.cell0 = 0;
    g.cells = uint32_t(cells);
    return MP_OK;
}

int validate_params(const mp_pbf_params& p) {
    if (p.size != sizeof(mp_pbf_params))
        return fail(MP_ERR_INVALID_ARGUMENT, "mp_pbf_params.size is %u, expected %zu", p.size,
                    sizeof(mp_pbf_params));
    if (!(p.h > 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "h must be > 0");
    if (!(p.rest_density > 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "rest_density must be > 0");
    if (!(p.epsilon >= 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "epsilon must be >= 0");
    if (p.solver_iterations > 1000)
        return fail(MP_ERR_INVALID_ARGUMENT, "solver_iterations %u > 1000", p.solver_iterations);
    if (p.scorr_n > 16) return fail(MP_ERR_INVALID_ARGUMENT, "scorr_n %u > 16", p.scorr_n);
    if (!(p.foam_speed_hi > p.foam_speed_lo))
        return fail(MP_ERR_INVALID_ARGUMENT, "foam_speed_hi must exceed foam_speed_lo");
    if (!(p.foam_max_neighbors > 0.0f))
        return fail(MP_ERR_INVALID_ARGUMENT, "foam_max_neighbors must be > 0");
    for (int a = 0; a < 3; ++a)
        if (!(p.bounds_max[a] > p.bounds_min[a]))
            return fail(MP_ERR_INVALID_ARGUMENT, "bounds_max must exceed bounds_min");
    GridDev g;
    return make_grid(p, g);
}

// Scene seeding: Engine::seedParticles (Engine.cpp:454-549), generalised to
// a box that is not centred on the origin (the cube and the dam column are
// centred on the box's x/z centre, which is 0 for the reference box), plus
// the explicit jittered lattice of mp_scene_desc.
int seed_scene(const mp_pbf_params& p, uint32_t scene, const mp_scene_desc& d, uint32_t n,
               std::vector<float>& pos) {
    pos.assign(4 * size_t(n), 0.0f);
    const float spacing_ref = p.h * 0.5f;  // Engine.cpp:457
    uint32_t i = 0;
    if (d.lattice) {
        const double sp = d.spacing > 0.0f ? double(d.spacing) : double(spacing_ref);
        const uint64_t cap = uint64_t(d.dims[0]) * d.dims[1] * d.dims[2];
        if (cap < n)
            return fail(MP_ERR_INVALID_ARGUMENT, "lattice %ux%ux%u holds fewer than %u particles",
                        d.dims[0], d.dims[1], d.dims[2], n);
        std::mt19937_64 rng(d.seed);
        auto jit = [&]() {
            const double u = double(rng() >> 11) * 0x1.0p-53;
            return (2.0 * u - 1.0) * double(d.jitter);
        };
        for (uint32_t y = 0; y < d.dims[1] && i < n; ++y)
            for (uint32_t z = 0; z < d.dims[2] && i < n; ++z)
                for (uint32_t x = 0; x < d.dims[0] && i < n; ++x, ++i) {
                    const double jx = jit(), jy = jit(), jz = jit();
                    pos[4 * i + 0] = float(double(d.origin[0]) + double(x) * sp + jx);
                    pos[4 * i + 1] = float(double(d.origin[1]) + double(y) * sp + jy);
                    pos[4 * i + 2] = float(double(d.origin[2]) + double(z) * sp + jz);
                    pos[4 * i + 3] = 1.0f;
                }
        return MP_OK;
    }
    const float spacing = spacing_ref;
    const float* bmin = p.bounds_min;
    const float* bmax = p.bounds_max;
    const float cx = 0.5f * (bmin[0] + bmax[0]);
    const float cz = 0.5f * (bmin[2] + bmax[2]);
    if (scene == MP_SCENE_DAM_BREAK) {
        const uint32_t nLayers = uint32_t(5.5f / spacing);
        if (nLayers == 0) return fail(MP_ERR_INVALID_ARGUMENT, "h too large for the dam column");
        const uint32_t perLayer = (n + nLayers - 1) / nLayers;
        const uint32_t side = uint32_t(std::ceil(std::sqrt(double(perLayer))));
        const float baseExtent = float(side - 1) * spacing;
        const float xMin = bmin[0] + 0.05f;
        const float yMin = bmin[1] + 0.05f;
        const float zStart = cz - baseExtent * 0.5f;
        for (uint32_t y = 0; y < nLayers && i < n; ++y)
            for (uint32_t z = 0; z < side && i < n; ++z)
                for (uint32_t x = 0; x < side && i < n; ++x, ++i) {
                    pos[4 * i + 0] = xMin + float(x) * spacing;
                    pos[4 * i + 1] = yMin + float(y) * spacing;
                    pos[4 * i + 2] = zStart + float(z) * spacing;
                    pos[4 * i + 3] = 1.0f;
                }
        return MP_OK;
    }
    if (scene == MP_SCENE_SPHERE_DROP) {
        const float xMin = bmin[0] + 0.05f, xMax = bmax[0] - 0.05f;
        const float zMin = bmin[2] + 0.05f, zMax = bmax[2] - 0.05f;
        const float yMin = bmin[1] + 0.05f;
        const uint32_t nx = uint32_t((xMax - xMin) / spacing);
        const uint32_t nz = uint32_t((zMax - zMin) / spacing);
        for (uint32_t y = 0;; ++y) {
            const float yPos = yMin + float(y) * spacing;
            if (yPos > bmax[1] - 0.5f || i >= n) break;
            for (uint32_t z = 0; z < nz && i < n; ++z)
                for (uint32_t x = 0; x < nx && i < n; ++x, ++i) {
                    pos[4 * i + 0] = xMin + float(x) * spacing;
                    pos[4 * i + 1] = yPos;
                    pos[4 * i + 2] = zMin + float(z) * spacing;
                    pos[4 * i + 3] = 1.0f;
                }
            if (nx == 0 || nz == 0) break;
        }
        return MP_OK;
    }
    if (scene != MP_SCENE_CUBE_DROP) return fail(MP_ERR_INVALID_ARGUMENT, "unknown scene %u", scene);
    const uint32_t side = uint32_t(std::ceil(std::cbrt(double(n))));
    const float halfBlk = 0.5f * float(side - 1) * spacing;
    const float topY = 2.0f;
    for (uint32_t y = 0; y < side && i < n; ++y)
        for (uint32_t z = 0; z < side && i < n; ++z)
            for (uint32_t x = 0; x < side && i < n; ++x, ++i) {
                pos[4 * i + 0] = cx - halfBlk + float(x) * spacing;
                pos[4 * i + 1] = topY - float(y) * spacing;
                pos[4 * i + 2] = cz - halfBlk + float(z) * spacing;
                pos[4 * i + 3] = 1.0f;
            }
    return MP_OK;
}

void fill_default_params(mp_pbf_params& p) {
    std::memset(&p, 0, sizeof(p));
    p.size = sizeof(mp_pbf_params);
    p.solver_iterations = 5;       // Engine.cpp:39
    p.h = 0.10f;                   // Engine.cpp:29
    p.cell_size = 0.10f;           // Engine.cpp:25
    p.rest_density = 8000.0f;      // Engine.cpp:32
    p.epsilon = 800.0f;            // Engine.cpp:35
    p.damping = 0.996f;            // Engine.cpp:36
    p.gravity[0] = 0.0f;           // Engine.cpp:558
    p.gravity[1] = -9.81f;
    p.gravity[2] = 0.0f;
    for (int a = 0; a < 3; ++a) p.bounds_min[a] = -3.0f;  // Engine.cpp:23
    p.bounds_max[0] = 3.0f;        // Engine.cpp:24
    p.bounds_max[1] = 6.0f;
    p.bounds_max[2] = 3.0f;
    p.scorr_k = 1e-4f;             // Constraints.metal:158
    p.scorr_n = 4;                 // Constraints.metal:179-180
    p.scorr_dq = 0.2f;             // Constraints.metal:159
    p.max_delta = 0.3f;            // Constraints.metal:190
    p.vmax = 1.0f;                 // Constraints.metal:347
    p.wall_eps = 1e-3f;            // Constraints.metal:325
    p.floor_friction = 0.55f;      // Constraints.metal:341-342
    p.wall_friction = 0.97f;       // Constraints.metal:344
    p.foam_max_neighbors = 96.0f;  // Engine.cpp:27, 806
    p.foam_speed_lo = 1.2f;        // Constraints.metal:297
    p.foam_speed_hi = 4.5f;
    p.sphere_radius = 0.6f;        // Engine.hpp:184
    p.sphere_gravity = -9.81f;     // Engine.cpp:694
    p.sphere_drag = 0.998f;        // Engine.cpp:695-697
    p.sphere_restitution = 0.4f;   // Engine.cpp:702-707
    p.integrate_damping = 0.999f;  // Engine.cpp:584
    p.integrate_restitution = 0.4f;  // Integrate.metal:29
    p.mouse_falloff = 0.4f;        // Constraints.metal:250
}

void fill_default_desc(mp_scene_desc& d) {
    std::memset(&d, 0, sizeof(d));
    d.size = sizeof(mp_scene_desc);
    d.sphere_center[1] = 4.5f;  // Engine.cpp:523-525
}

size_t elem_bytes(uint32_t which) {
    switch (which) {
        case MP_BUF_POSITIONS:
        case MP_BUF_VELOCITIES:
        case MP_BUF_PREV_POSITIONS:
        case MP_BUF_SORTED_POSITIONS:
            return 16;
        default:
            return 4;
    }
}

// writePBFParams (Engine.cpp:551-572) and the shader literals, in FP32 like
// the reference, for a scene of n particles on grid g stepped by dt.
StepConsts make_consts(const mp_pbf_params& p, const GridDev& g, uint32_t n, float dt, bool sphere) {
    StepConsts c{};
    c.g = g;
    c.n = n;
    const float h = p.h, h2 = h * h, h3 = h2 * h, h6 = h3 * h3, h9 = h6 * h3;
    c.h = h;
    c.h2 = h2;
    c.poly6 = 315.0f / (64.0f * kPi * h9);
    c.spiky = 45.0f / (kPi * h6);
    c.inv_rho0 = 1.0f / p.rest_density;
    c.eps = p.epsilon;
    c.scorr_k = p.scorr_k;
    c.scorr_n = p.scorr_n;
    // invWq = 1 / poly6((dq*h)^2) (Constraints.metal:159-160)
    const float dq = p.scorr_dq * h;
    const float dq2 = dq * dq;
    const float wd = h2 - dq2;
    const float wq = dq2 < h2 ? c.poly6 * wd * wd * wd : 0.0f;
    c.inv_wq = wq > 0.0f ? 1.0f / wq : 0.0f;
    c.scorr_pq = c.poly6 * c.inv_wq;
    c.delta_scale = -c.spiky * c.inv_rho0;
    c.max_step = p.max_delta * h;
    c.bminx = p.bounds_min[0];
    c.bminy = p.bounds_min[1];
    c.bminz = p.bounds_min[2];
    c.bmaxx = p.bounds_max[0];
    c.bmaxy = p.bounds_max[1];
    c.bmaxz = p.bounds_max[2];
    c.gravx = p.gravity[0];
    c.gravy = p.gravity[1];
    c.gravz = p.gravity[2];
    c.dt = dt;
    c.inv_dt = 1.0f / dt;
    c.damping = p.damping;
    c.vmax = p.vmax * h * c.inv_dt;
    c.vmax_frac = p.vmax;
    c.wall_eps = p.wall_eps;
    c.floor_fric = p.floor_friction;
    c.wall_fric = p.wall_friction;
    c.foam_maxn = p.foam_max_neighbors;
    c.foam_lo = p.foam_speed_lo;
    c.foam_hi = p.foam_speed_hi;
    c.sphere = sphere ? 1 : 0;
    c.sph_gravity = p.sphere_gravity;
    c.sph_drag = p.sphere_drag;
    c.sph_rest = p.sphere_restitution;
    return c;
}

}  // namespace mpb

namespace {

// Per-kernel CUDA-event timing (mp_engine_set_profiling): two events per
// launch on the launching stream, reduced to totals per kernel name when read.
struct EventTimer final : mpb::KernelTimer {
    std::vector<cudaEvent_t> pool;
    size_t used = 0, open = 0;
    struct Mark {
        const char* name;
        size_t b, e;
    };
    std::vector<Mark> marks;
    std::map<std::string, std::pair<uint32_t, double>> totals;
    cudaError_t status = cudaSuccess;

    cudaEvent_t next() {
        if (used == pool.size()) {
            cudaEvent_t ev = nullptr;
            const cudaError_t e = cudaEventCreate(&ev);
            if (e != cudaSuccess) status = e;
            pool.push_back(ev);
        }
        return pool[used++];
    }
    // graphs of profiled steps, kept until their events are read
    std::vector<std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;

    // Under stream capture the record becomes an event node of the graph
    // (cudaEventRecordExternal), so the events time the kernels as the graph
    // runs them, without the host's launch gaps between them.
    static void record(cudaEvent_t ev, cudaStream_t s) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
            cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal);
        else
            cudaEventRecord(ev, s);
    }
    void begin(cudaStream_t s) override {
        open = used;
        record(next(), s);
    }
    void end(const char* kernel, cudaStream_t s) override {
        const size_t e = used;
        record(next(), s);
        marks.push_back({kernel, open, e});
    }
    void release_graphs() {
        if (!graphs.empty()) cudaDeviceSynchronize();
        for (auto& g : graphs) {
            if (g.second) cudaGraphExecDestroy(g.second);
            if (g.first) cudaGraphDestroy(g.first);
        }
        graphs.clear();
    }
    cudaError_t collect() {
        for (const Mark& m : marks) {
            cudaError_t e = cudaEventSynchronize(pool[m.e]);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, pool[m.b], pool[m.e]);
            if (e != cudaSuccess) return e;
            auto& t = totals[m.name];
            t.first += 1;
            t.second += ms;
        }
        marks.clear();
        used = 0;
        release_graphs();
        return status;
    }
    ~EventTimer() override {
        release_graphs();
        for (cudaEvent_t ev : pool)
            if (ev) cudaEventDestroy(ev);
    }
};

}  // namespace

struct mp_engine {
    int device = 0;
    mp_pbf_params params{};
    mp_scene_desc desc{};
    uint32_t scene = MP_SCENE_CUBE_DROP;
    uint32_t n = 0;
    GridDev grid{};
    DevState d{};
    uint32_t n_alloc = 0;      // particle capacity of the buffers
    uint32_t cells_alloc = 0;  // grid cells the cell buffers were sized for (0: none)
    void* particle_block = nullptr;
    void* list_block = nullptr;  // in-range row masks of the solver
    void* cell_block = nullptr;
    void* small_block = nullptr;
    mpb::SphereState sphere_init{};
    // graph mode
    bool graph_mode = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    float graph_dt = 0.0f;
    uint32_t graph_spin_epoch = 0;  // spin limits the captured graph was made with
    // profiling
    EventTimer* timer = nullptr;
    // render targets (Engine::ensureRenderTargets, Engine.cpp:351-377)
    void* render_block = nullptr;
    uint32_t render_w = 0, render_h = 0;
    mpb::RenderBuffers rb{};

    int ensure_render_targets(uint32_t w, uint32_t h) {
        if (render_block && w == render_w && h == render_h) return MP_OK;
        dev_free(render_block);
        render_block = nullptr;
        const size_t px = size_t(w) * h, plane = (px * 4 + 255) & ~size_t(255);
        MP_ALLOC(render_block, 4 * plane + 4 * plane, device);
        char* p = static_cast<char*>(render_block);
        rb.depth = reinterpret_cast<uint32_t*>(p);
        rb.thick = reinterpret_cast<float*>(p + plane);
        rb.smoothed = reinterpret_cast<float*>(p + 2 * plane);
        rb.ndc = reinterpret_cast<float*>(p + 3 * plane);
        rb.rgba = reinterpret_cast<float4*>(p + 4 * plane);
        render_w = w;
        render_h = h;
        return MP_OK;
    }

    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    }
    void free_particles() {
        dev_free(particle_block);
        dev_free(list_block);
        particle_block = nullptr;
        list_block = nullptr;
        d.pos = d.vel = d.prev = d.sorted_a = d.sorted_b = nullptr;
        d.hash = d.off = d.tmp = d.sidx = d.scell = d.ncount = d.long_list = nullptr;
        d.lambdas = d.foam = nullptr;
        d.row_masks = nullptr;
        d.mask_overflow = nullptr;
        d.mask_stride = 0;
        n_alloc = 0;
    }
    void free_cells() {
        dev_free(cell_block);
        cell_block = nullptr;
        d.counts = d.cstart = nullptr;
        d.scan_ticket = d.scan_status = nullptr;
        cells_alloc = 0;
    }
    ~mp_engine() {
        DeviceGuard g(device);
        delete timer;
        drop_graph();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        free_particles();
        free_cells();
        dev_free(small_block);
        dev_free(render_block);
    }

    int alloc_particles(uint32_t count) {
        const uint32_t cap = round_up(count ? count : 1u, kPad);
        if (cap == n_alloc) return MP_OK;
        free_particles();
        const size_t v4 = size_t(cap) * 16, u = size_t(cap) * 4;
        const size_t longs = (size_t(cap) / mpb::kSegMax + 2) * 4;
        const size_t total = 5 * v4 + 8 * u + longs + 16 * 256;
        MP_ALLOC(particle_block, total, device);
        char* b = static_cast<char*>(particle_block);
        auto take = [&](size_t bytes) {
            char* r = b;
            b += (bytes + 255) & ~size_t(255);
            return r;
        };
        d.pos = reinterpret_cast<float4*>(take(v4));
        d.vel = reinterpret_cast<float4*>(take(v4));
        d.prev = reinterpret_cast<float4*>(take(v4));
        d.sorted_a = reinterpret_cast<float4*>(take(v4));
        d.sorted_b = reinterpret_cast<float4*>(take(v4));
        d.hash = reinterpret_cast<uint32_t*>(take(u));
        d.off = reinterpret_cast<uint32_t*>(take(u));
        d.tmp = reinterpret_cast<uint32_t*>(take(u));
        d.sidx = reinterpret_cast<uint32_t*>(take(u));
        d.scell = reinterpret_cast<uint32_t*>(take(u));
        d.ncount = reinterpret_cast<uint32_t*>(take(u));
        d.lambdas = reinterpret_cast<float*>(take(u));
        d.foam = reinterpret_cast<float*>(take(u));
        d.long_list = reinterpret_cast<uint32_t*>(take(longs));
        MP_CUDA(cudaMemset(particle_block, 0, total));
        // 9 row masks (4 bytes each) + an overflow flag per particle
        MP_ALLOC(list_block, 10 * u, device);
        d.row_masks = static_cast<uint32_t*>(list_block);
        d.mask_overflow = d.row_masks + 9 * size_t(cap);
        d.mask_stride = cap;
        n_alloc = cap;
        return MP_OK;
    }

    int alloc_cells(uint32_t cells) {
        if (cells == cells_alloc && cell_block) return MP_OK;
        free_cells();
        const size_t len = size_t(cells) + 1;
        const uint32_t tiles = mpb::scan_tiles_for(len);
        const size_t cb = ((len * 4 + 255) & ~size_t(255));
        const size_t total = 2 * cb + size_t(tiles) * 8 + 256;
        MP_ALLOC(cell_block, total, device);
        MP_CUDA(cudaMemset(cell_block, 0, total));
        char* b = static_cast<char*>(cell_block);
        d.counts = reinterpret_cast<uint32_t*>(b);
        d.cstart = reinterpret_cast<uint32_t*>(b + cb);
        d.scan_ticket = reinterpret_cast<unsigned long long*>(b + 2 * cb);
        d.scan_status = reinterpret_cast<unsigned long long*>(b + 2 * cb + 256);
        d.scan_tiles = tiles;
        cells_alloc = cells;
        return MP_OK;
    }

    int alloc_small() {
        if (small_block) return MP_OK;
        MP_ALLOC(small_block, 256, device);
        MP_CUDA(cudaMemset(small_block, 0, 256));
        char* b = static_cast<char*>(small_block);
        d.long_count = reinterpret_cast<uint32_t*>(b);
        d.err = reinterpret_cast<uint32_t*>(b + 4);
        d.sphere = reinterpret_cast<mpb::SphereState*>(b + 64);
        return MP_OK;
    }

    // false after an allocation failed: the engine holds no particles and
    // launches nothing until a reset or set_params allocates again
    bool ready() const { return particle_block && cell_block && small_block; }

    // a failed allocation leaves the engine empty, not half-built
    int emptied(int rc) {
        drop_graph();
        n = 0;
        return rc;
    }

    StepConsts consts(float dt) const {
        return mpb::make_consts(params, grid, n, dt, scene == MP_SCENE_SPHERE_DROP);
    }

    int enqueue_step(float dt, cudaStream_t s, mpb::KernelTimer* t = nullptr) {
        const StepConsts c = consts(dt);
        cudaError_t e = mpb::launch_hash_pass(c, d, true, s, t);
        if (e == cudaSuccess) e = mpb::launch_solver(c, d, params.solver_iterations, s, t);
        if (e != cudaSuccess) return fail(MP_ERR_CUDA, "step launch: %s", cudaGetErrorString(e));
        return MP_OK;
    }
};

extern "C" {

const char* mp_last_error(void) { return mpb::last_error(); }

}  // extern "C"

extern "C" {

uint32_t mp_abi_version(void) { return kAbiVersion; }

int mp_default_params(mp_pbf_params* out) {
    if (!out) return fail(MP_ERR_INVALID_ARGUMENT, "out is NULL");
    fill_default_params(*out);
    return MP_OK;
}

int mp_default_scene_desc(mp_scene_desc* out) {
    if (!out) return fail(MP_ERR_INVALID_ARGUMENT, "out is NULL");
    fill_default_desc(*out);
    return MP_OK;
}

double mp_lattice_rest_density(double h, double spacing) {
    if (!(h > 0.0) || !(spacing > 0.0)) return 0.0;
    const double pi = 3.14159265358979323846;
    const double norm = 315.0 / (64.0 * pi * std::pow(h, 9));
    const int R = int(std::ceil(h / spacing)) + 1;
    double rho = 0.0;
    for (int z = -R; z <= R; ++z)
        for (int y = -R; y <= R; ++y)
            for (int x = -R; x <= R; ++x) {
                const double r2 = spacing * spacing * double(x * x + y * y + z * z);
                if (r2 < h * h) {
                    const double d = h * h - r2;
                    rho += norm * d * d * d;
                }
            }
    return rho;
}

int mp_engine_create(int device, mp_engine** out) {
    if (!out) return fail(MP_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int count = 0;
    MP_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
        return fail(MP_ERR_INVALID_ARGUMENT, "device %d not in [0, %d)", device, count);
    auto* e = new (std::nothrow) mp_engine();
    if (!e) return fail(MP_ERR_OUT_OF_MEMORY, "host allocation failed");
    e->device = device;
    fill_default_params(e->params);
    fill_default_desc(e->desc);
    DeviceGuard g(device);
    int rc = e->alloc_small();
    if (rc == MP_OK) rc = make_grid(e->params, e->grid);
    // Engine(MTL::Device*) seeds 200K particles (Engine.cpp:101).
    if (rc == MP_OK) rc = mp_engine_reset_scene(e, 200000, MP_SCENE_CUBE_DROP, nullptr);
    if (rc != MP_OK) {
        const std::string msg = g_err;
        delete e;
        g_err = msg;
        return rc;
    }
    *out = e;
    return MP_OK;
}

int mp_engine_destroy(mp_engine* e) {
    delete e;
    return MP_OK;
}

int mp_engine_set_params(mp_engine* e, const mp_pbf_params* p) {
    if (!e || !p) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    int rc = validate_params(*p);
    if (rc != MP_OK) return rc;
    DeviceGuard g(e->device);
    GridDev grid;
    rc = make_grid(*p, grid);
    if (rc != MP_OK) return rc;
    rc = e->alloc_cells(grid.cells);
    if (rc != MP_OK) return e->emptied(rc);
    e->params = *p;
    e->grid = grid;
    e->drop_graph();
    return MP_OK;
}

int mp_engine_get_params(const mp_engine* e, mp_pbf_params* out) {
    if (!e || !out) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = e->params;
    return MP_OK;
}

int mp_engine_reset(mp_engine* e, uint32_t n) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    return mp_engine_reset_scene(e, n, e->scene, &e->desc);
}

int mp_engine_reset_scene(mp_engine* e, uint32_t n, uint32_t scene, const mp_scene_desc* desc) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    if (scene > MP_SCENE_SPHERE_DROP) return fail(MP_ERR_INVALID_ARGUMENT, "unknown scene %u", scene);
    if (n > (1u << 30)) return fail(MP_ERR_INVALID_ARGUMENT, "particle count %u too large", n);
    mp_scene_desc dd;
    if (desc) {
        if (desc->size != sizeof(mp_scene_desc))
            return fail(MP_ERR_INVALID_ARGUMENT, "mp_scene_desc.size is %u, expected %zu",
                        desc->size, sizeof(mp_scene_desc));
        dd = *desc;
    } else {
        fill_default_desc(dd);
    }
    std::vector<float> pos;
    int rc = seed_scene(e->params, scene, dd, n, pos);
    if (rc != MP_OK) return rc;
    DeviceGuard g(e->device);
    rc = make_grid(e->params, e->grid);
    if (rc != MP_OK) return rc;
    rc = e->alloc_cells(e->grid.cells);
    if (rc == MP_OK) rc = e->alloc_particles(n);
    if (rc != MP_OK) return e->emptied(rc);
    e->drop_graph();
    e->scene = scene;
    e->desc = dd;
    e->n = n;
    const size_t v4 = size_t(e->n_alloc) * 16, u = size_t(e->n_alloc) * 4;
    MP_CUDA(cudaMemset(e->d.vel, 0, v4));  // Engine.cpp:461
    MP_CUDA(cudaMemset(e->d.prev, 0, v4));
    MP_CUDA(cudaMemset(e->d.ncount, 0, u));
    MP_CUDA(cudaMemset(e->d.lambdas, 0, u));
    MP_CUDA(cudaMemset(e->d.foam, 0, u));
    MP_CUDA(cudaMemset(e->d.pos, 0, v4));
    if (n) MP_CUDA(cudaMemcpy(e->d.pos, pos.data(), 16 * size_t(n), cudaMemcpyHostToDevice));
    MP_CUDA(cudaMemset(e->d.counts, 0, (size_t(e->grid.cells) + 1) * 4));
    // Sphere reset (Engine.cpp:522-526).
    mpb::SphereState sph{};
    for (int a = 0; a < 3; ++a) {
        sph.c[a] = dd.sphere_center[a];
        sph.v[a] = dd.sphere_velocity[a];
    }
    sph.r = e->params.sphere_radius;
    MP_CUDA(cudaMemcpy(e->d.sphere, &sph, sizeof(sph), cudaMemcpyHostToDevice));
    MP_CUDA(cudaDeviceSynchronize());
    return MP_OK;
}

int mp_engine_step(mp_engine* e, float dt, mp_stream stream) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    if (!(dt > 0.0f)) return MP_OK;  // Engine.cpp:686
    if (!e->ready()) return MP_OK;   // emptied by a failed allocation
    DeviceGuard g(e->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (e->timer) {
        if (e->timer->marks.size() > 65536) {
            const cudaError_t ce = e->timer->collect();
            if (ce != cudaSuccess) return fail(MP_ERR_CUDA, "profiling: %s", cudaGetErrorString(ce));
        }
        if (!e->graph_mode) return e->enqueue_step(dt, s, e->timer);
        // graph mode: the step and its timing events captured as one graph
        // (instantiated per step, released when the times are read)
        if (!e->cap_stream) MP_CUDA(cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking));
        // a step that does not run leaves no marks behind (their events are
        // never recorded)
        const size_t marks0 = e->timer->marks.size(), used0 = e->timer->used;
        auto forget = [&] {
            e->timer->marks.resize(marks0);
            e->timer->used = used0;
        };
        MP_CUDA(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = e->enqueue_step(dt, e->cap_stream, e->timer);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(e->cap_stream, &graph);
        if (rc != MP_OK) {
            if (graph) cudaGraphDestroy(graph);
            forget();
            return rc;
        }
        if (ce != cudaSuccess) {
            forget();
            return fail(MP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        if (ie != cudaSuccess) {
            cudaGraphDestroy(graph);
            forget();
            return fail(MP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
        }
        e->timer->graphs.push_back({graph, exec});
        MP_CUDA(cudaGraphLaunch(exec, s));
        return MP_OK;
    }
    if (!e->graph_mode) return e->enqueue_step(dt, s);
    if (!e->gexec || e->graph_dt != dt || e->graph_spin_epoch != mpb::spin_limit_epoch()) {
        e->drop_graph();
        if (!e->cap_stream) MP_CUDA(cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking));
        MP_CUDA(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = e->enqueue_step(dt, e->cap_stream);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(e->cap_stream, &graph);
        if (rc != MP_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return fail(MP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        e->graph = graph;
        MP_CUDA(cudaGraphInstantiate(&e->gexec, e->graph, 0));
        e->graph_dt = dt;
        e->graph_spin_epoch = mpb::spin_limit_epoch();
    }
    MP_CUDA(cudaGraphLaunch(e->gexec, s));
    return MP_OK;
}

int mp_engine_build_spatial_hash(mp_engine* e, mp_stream stream) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    if (!e->ready()) return MP_OK;
    DeviceGuard g(e->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const StepConsts c = e->consts(1.0f);
    cudaError_t err = mpb::launch_hash_pass(c, e->d, false, s, e->timer);
    if (err == cudaSuccess) err = mpb::launch_count_neighbors(c, e->d, s, e->timer);
    if (err != cudaSuccess) return fail(MP_ERR_CUDA, "hash launch: %s", cudaGetErrorString(err));
    return MP_OK;
}

int mp_engine_set_graph_mode(mp_engine* e, int enable) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    DeviceGuard g(e->device);
    e->graph_mode = enable != 0;
    if (!e->graph_mode) e->drop_graph();
    return MP_OK;
}

int mp_engine_set_profiling(mp_engine* e, int enable) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    DeviceGuard g(e->device);
    if (enable && !e->timer) e->timer = new (std::nothrow) EventTimer();
    if (enable && !e->timer) return fail(MP_ERR_OUT_OF_MEMORY, "host allocation failed");
    if (!enable && e->timer) {
        MP_CUDA(cudaDeviceSynchronize());
        delete e->timer;
        e->timer = nullptr;
    }
    return MP_OK;
}

int mp_engine_kernel_times(mp_engine* e, mp_kernel_time* out, uint32_t capacity, uint32_t* count) {
    if (!e || !count || (capacity && !out)) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = 0;
    if (!e->timer) return MP_OK;
    DeviceGuard g(e->device);
    const cudaError_t ce = e->timer->collect();
    if (ce != cudaSuccess) return fail(MP_ERR_CUDA, "profiling: %s", cudaGetErrorString(ce));
    uint32_t i = 0;
    for (const auto& kv : e->timer->totals) {
        if (i < capacity) {
            std::memset(&out[i], 0, sizeof(mp_kernel_time));
            std::snprintf(out[i].name, sizeof(out[i].name), "%s", kv.first.c_str());
            out[i].launches = kv.second.first;
            out[i].ms = kv.second.second;
        }
        ++i;
    }
    *count = i;
    e->timer->totals.clear();
    return MP_OK;
}

uint32_t mp_step_launch_count(uint32_t iterations) { return mpb::step_launch_count(iterations); }

uint32_t mp_engine_particle_count(const mp_engine* e) { return e ? e->n : 0; }
uint32_t mp_engine_total_cells(const mp_engine* e) { return e ? e->grid.cells : 0; }
float mp_engine_cell_size(const mp_engine* e) { return e ? e->params.cell_size : 0.0f; }
uint32_t mp_engine_current_scene(const mp_engine* e) { return e ? e->scene : 0; }

int mp_engine_grid_dims(const mp_engine* e, uint32_t dims[3]) {
    if (!e || !dims) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    dims[0] = uint32_t(e->grid.gx);
    dims[1] = uint32_t(e->grid.gy);
    dims[2] = uint32_t(e->grid.gz);
    return MP_OK;
}

int mp_engine_buffer(mp_engine* e, uint32_t which, void** dptr, size_t* bytes) {
    if (!e || !dptr) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t n = e->n;
    void* p = nullptr;
    size_t count = n;
    switch (which) {
        case MP_BUF_POSITIONS: p = e->d.pos; break;
        case MP_BUF_VELOCITIES: p = e->d.vel; break;
        case MP_BUF_PREV_POSITIONS: p = e->d.prev; break;
        case MP_BUF_CELL_HASHES: p = e->d.hash; break;
        case MP_BUF_CELL_START: p = e->d.cstart; count = size_t(e->grid.cells) + 1; break;
        case MP_BUF_SORTED_INDEX: p = e->d.sidx; break;
        case MP_BUF_NEIGHBOR_COUNTS: p = e->d.ncount; break;
        case MP_BUF_LAMBDAS: p = e->d.lambdas; break;
        case MP_BUF_FOAM: p = e->d.foam; break;
        case MP_BUF_SORTED_POSITIONS: p = e->d.sorted_a; break;
        default: return fail(MP_ERR_INVALID_ARGUMENT, "unknown buffer %u", which);
    }
    *dptr = p;
    if (bytes) *bytes = count * elem_bytes(which);
    return MP_OK;
}

int mp_engine_upload(mp_engine* e, uint32_t which, const void* host, size_t count, mp_stream stream) {
    void* dptr = nullptr;
    size_t bytes = 0;
    int rc = mp_engine_buffer(e, which, &dptr, &bytes);
    if (rc != MP_OK) return rc;
    if (!host && count) return fail(MP_ERR_INVALID_ARGUMENT, "host is NULL");
    const size_t need = count * elem_bytes(which);
    if (need > bytes) return fail(MP_ERR_INVALID_ARGUMENT, "%zu elements exceed buffer %u", count, which);
    if (!need) return MP_OK;
    DeviceGuard g(e->device);
    MP_CUDA(cudaMemcpyAsync(dptr, host, need, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)));
    return MP_OK;
}

int mp_engine_download(mp_engine* e, uint32_t which, void* host, size_t count, mp_stream stream) {
    void* dptr = nullptr;
    size_t bytes = 0;
    int rc = mp_engine_buffer(e, which, &dptr, &bytes);
    if (rc != MP_OK) return rc;
    if (!host && count) return fail(MP_ERR_INVALID_ARGUMENT, "host is NULL");
    const size_t need = count * elem_bytes(which);
    if (need > bytes) return fail(MP_ERR_INVALID_ARGUMENT, "%zu elements exceed buffer %u", count, which);
    DeviceGuard g(e->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (need) MP_CUDA(cudaMemcpyAsync(host, dptr, need, cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

int mp_engine_set_sphere(mp_engine* e, const float center[3], const float velocity[3], float radius) {
    if (!e || !center || !velocity) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!(radius >= 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "radius must be >= 0");
    mpb::SphereState s{};
    for (int a = 0; a < 3; ++a) {
        s.c[a] = center[a];
        s.v[a] = velocity[a];
    }
    s.r = radius;
    DeviceGuard g(e->device);
    MP_CUDA(cudaDeviceSynchronize());
    MP_CUDA(cudaMemcpy(e->d.sphere, &s, sizeof(s), cudaMemcpyHostToDevice));
    return MP_OK;
}

int mp_engine_get_sphere(mp_engine* e, float center[3], float velocity[3], float* radius) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    mpb::SphereState s{};
    DeviceGuard g(e->device);
    MP_CUDA(cudaDeviceSynchronize());
    MP_CUDA(cudaMemcpy(&s, e->d.sphere, sizeof(s), cudaMemcpyDeviceToHost));
    for (int a = 0; a < 3; ++a) {
        if (center) center[a] = s.c[a];
        if (velocity) velocity[a] = s.v[a];
    }
    if (radius) *radius = s.r;
    return MP_OK;
}

int mp_engine_integrate(mp_engine* e, float dt, mp_stream stream) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    if (!(dt > 0.0f) || !e->ready()) return MP_OK;
    DeviceGuard g(e->device);
    const mp_pbf_params& p = e->params;
    mpb::IntegrateConsts c{};
    c.n = e->n;
    c.dt = dt;
    c.damping = p.integrate_damping;
    c.restitution = p.integrate_restitution;
    c.gx = p.gravity[0];
    c.gy = p.gravity[1];
    c.gz = p.gravity[2];
    c.bminx = p.bounds_min[0];
    c.bminy = p.bounds_min[1];
    c.bminz = p.bounds_min[2];
    c.bmaxx = p.bounds_max[0];
    c.bmaxy = p.bounds_max[1];
    c.bmaxz = p.bounds_max[2];
    const cudaError_t err = mpb::launch_integrate(c, e->d.pos, e->d.vel, static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return fail(MP_ERR_CUDA, "integrate launch: %s", cudaGetErrorString(err));
    return MP_OK;
}

int mp_engine_apply_mouse_pulse(mp_engine* e, const float ray_origin[3], const float ray_dir[3],
                                const float force[3], float radius, mp_stream stream) {
    if (!e || !ray_origin || !ray_dir || !force) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!e->ready()) return MP_OK;
    DeviceGuard g(e->device);
    mpb::MouseConsts c{};
    c.n = e->n;
    c.ox = ray_origin[0];
    c.oy = ray_origin[1];
    c.oz = ray_origin[2];
    c.dx = ray_dir[0];
    c.dy = ray_dir[1];
    c.dz = ray_dir[2];
    c.fx = force[0];
    c.fy = force[1];
    c.fz = force[2];
    c.radius = radius;
    c.falloff = e->params.mouse_falloff;
    const cudaError_t err = mpb::launch_mouse_pulse(c, e->d.vel, e->d.pos, static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return fail(MP_ERR_CUDA, "mouse pulse launch: %s", cudaGetErrorString(err));
    return MP_OK;
}

int mp_engine_render(mp_engine* e, const mp_render_params* rp, float* rgba, mp_stream stream) {
    if (!e || !rp) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!e->ready())
        return fail(MP_ERR_INVALID_ARGUMENT, "the engine holds no particles since an allocation failed");
    mpb::RenderConsts c;
    int rc = mpb::make_render_consts(*rp, e->params, e->n, e->scene == MP_SCENE_SPHERE_DROP, c);
    if (rc != MP_OK) return rc;
    DeviceGuard g(e->device);
    rc = e->ensure_render_targets(rp->width, rp->height);
    if (rc != MP_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const cudaError_t err = mpb::launch_render(c, e->rb, e->d.pos, e->d.foam, e->d.sphere, s);
    if (err != cudaSuccess) return fail(MP_ERR_CUDA, "render launch: %s", cudaGetErrorString(err));
    if (rgba)
        MP_CUDA(cudaMemcpyAsync(rgba, e->rb.rgba, size_t(rp->width) * rp->height * 16, cudaMemcpyDeviceToDevice, s));
    return MP_OK;
}

int mp_engine_render_buffer(mp_engine* e, uint32_t which, void** dptr, size_t* bytes) {
    if (!e || !dptr || !bytes) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!e->render_block) return fail(MP_ERR_INVALID_ARGUMENT, "nothing rendered yet");
    const size_t px = size_t(e->render_w) * e->render_h;
    switch (which) {
        case MP_RENDER_BUF_COLOR: *dptr = e->rb.rgba; *bytes = 16 * px; break;
        case MP_RENDER_BUF_DEPTH: *dptr = e->rb.depth; *bytes = 4 * px; break;
        case MP_RENDER_BUF_SMOOTHED: *dptr = e->rb.smoothed; *bytes = 4 * px; break;
        case MP_RENDER_BUF_THICKNESS: *dptr = e->rb.thick; *bytes = 4 * px; break;
        case MP_RENDER_BUF_NDC_DEPTH: *dptr = e->rb.ndc; *bytes = 4 * px; break;
        default: return fail(MP_ERR_INVALID_ARGUMENT, "unknown render buffer %u", which);
    }
    return MP_OK;
}

size_t mp_engine_snapshot_size(const mp_engine* e) {
    return e ? mpb::snapshot_bytes(1, e->n) : 0;
}

int mp_engine_snapshot(mp_engine* e, void* host, size_t bytes) {
    if (!e || !host) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t need = mpb::snapshot_bytes(1, e->n);
    if (bytes < need) return fail(MP_ERR_INVALID_ARGUMENT, "snapshot needs %zu bytes, got %zu", need, bytes);
    DeviceGuard g(e->device);
    MP_CUDA(cudaDeviceSynchronize());
    char* out = static_cast<char*>(host);
    mpb::SnapshotHeader h;
    mpb::snapshot_header(h, mpb::kSnapshotEngine, 1, e->n);
    std::memcpy(out, &h, sizeof(h));
    mpb::SnapshotScene sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.params = e->params;
    sc.desc = e->desc;
    sc.scene_id = e->scene;
    sc.count = e->n;
    mpb::SphereState sph{};
    MP_CUDA(cudaMemcpy(&sph, e->d.sphere, sizeof(sph), cudaMemcpyDeviceToHost));
    for (int a = 0; a < 3; ++a) {
        sc.sphere[a] = sph.c[a];
        sc.sphere[3 + a] = sph.v[a];
    }
    sc.sphere[6] = sph.r;
    std::memcpy(out + sizeof(h), &sc, sizeof(sc));
    char* arrays = out + sizeof(h) + sizeof(sc);
    if (e->n) {
        MP_CUDA(cudaMemcpy(arrays, e->d.pos, 16 * size_t(e->n), cudaMemcpyDeviceToHost));
        MP_CUDA(cudaMemcpy(arrays + 16 * size_t(e->n), e->d.vel, 16 * size_t(e->n), cudaMemcpyDeviceToHost));
    }
    return MP_OK;
}

int mp_engine_restore(mp_engine* e, const void* host, size_t bytes) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    if (const char* why = mpb::snapshot_check(host, bytes, mpb::kSnapshotEngine))
        return fail(MP_ERR_INVALID_ARGUMENT, "%s", why);
    const char* in = static_cast<const char*>(host);
    mpb::SnapshotHeader h;
    std::memcpy(&h, in, sizeof(h));
    if (h.nscenes != 1) return fail(MP_ERR_INVALID_ARGUMENT, "an engine snapshot holds one scene");
    mpb::SnapshotScene sc;
    std::memcpy(&sc, in + sizeof(h), sizeof(sc));
    if (sc.count != h.particles) return fail(MP_ERR_INVALID_ARGUMENT, "snapshot particle counts disagree");
    int rc = mp_engine_set_params(e, &sc.params);
    if (rc == MP_OK) rc = mp_engine_reset_scene(e, sc.count, sc.scene_id, &sc.desc);
    if (rc != MP_OK) return rc;
    DeviceGuard g(e->device);
    const char* arrays = in + sizeof(h) + sizeof(sc);
    if (e->n) {
        MP_CUDA(cudaMemcpy(e->d.pos, arrays, 16 * size_t(e->n), cudaMemcpyHostToDevice));
        MP_CUDA(cudaMemcpy(e->d.vel, arrays + 16 * size_t(e->n), 16 * size_t(e->n), cudaMemcpyHostToDevice));
    }
    return mp_engine_set_sphere(e, sc.sphere, sc.sphere + 3, sc.sphere[6]);
}

int mp_engine_check_errors(mp_engine* e, uint32_t* bits) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    DeviceGuard g(e->device);
    MP_CUDA(cudaDeviceSynchronize());
    uint32_t w = 0;
    MP_CUDA(cudaMemcpy(&w, e->d.err, 4, cudaMemcpyDeviceToHost));
    MP_CUDA(cudaMemset(e->d.err, 0, 4));
    if (bits) *bits = w;
    if (w & mpb::kDevErrSpin) return fail(MP_ERR_SPIN_LIMIT, "a bounded device wait gave up (bits 0x%x)", w);
    if (w) return fail(MP_ERR_DEVICE, "device error word 0x%x", w);
    return MP_OK;
}

int mp_engine_synchronize(mp_engine* e) {
    if (!e) return fail(MP_ERR_INVALID_ARGUMENT, "NULL engine");
    DeviceGuard g(e->device);
    MP_CUDA(cudaDeviceSynchronize());
    return MP_OK;
}

int mp_set_spin_limit(uint32_t polls) {
    g_scan_spins.store(polls ? polls : kDefaultScanSpinLimit);
    g_barrier_spins.store(polls ? polls : kDefaultBarrierSpinLimit);
    g_spin_epoch.fetch_add(1);
    return MP_OK;
}

int mp_set_device_allocator(mp_device_alloc_fn alloc, mp_device_free_fn free_fn, void* user) {
    if (alloc && !free_fn) return fail(MP_ERR_INVALID_ARGUMENT, "an allocator needs a free function");
    std::lock_guard<std::mutex> lock(g_alloc_lock);
    g_alloc.alloc = alloc;
    g_alloc.free = alloc ? free_fn : nullptr;
    g_alloc.user = alloc ? user : nullptr;
    return MP_OK;
}

size_t mp_exclusive_scan_scratch_bytes(uint32_t n) {
    return 256 + size_t(mpb::scan_tiles_for(n)) * 8;
}

int mp_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, void* scratch,
                      size_t scratch_bytes, mp_stream stream) {
    if (n == 0) return MP_OK;  // Engine.cpp:848
    if (!in || !out || !scratch) return fail(MP_ERR_INVALID_ARGUMENT, "NULL pointer");
    const size_t need = mp_exclusive_scan_scratch_bytes(n);
    if (scratch_bytes < need)
        return fail(MP_ERR_INVALID_ARGUMENT, "scratch of %zu bytes, need %zu", scratch_bytes, need);
    if (reinterpret_cast<uintptr_t>(scratch) & 7u)
        return fail(MP_ERR_INVALID_ARGUMENT, "scratch must be 8-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // scratch: [0,8) ticket, [8,12) error word, [256, ...) tile descriptors
    MP_CUDA(cudaMemsetAsync(scratch, 0, need, s));
    char* b = static_cast<char*>(scratch);
    const cudaError_t e = mpb::launch_scan(in, out, n, reinterpret_cast<unsigned long long*>(b + 256),
                                           reinterpret_cast<unsigned long long*>(b),
                                           mpb::scan_tiles_for(n), false,
                                           reinterpret_cast<uint32_t*>(b + 8), s);
    if (e != cudaSuccess) return fail(MP_ERR_CUDA, "scan launch: %s", cudaGetErrorString(e));
    return MP_OK;
}

int mp_debug_exclusive_scan_from_ticket(const uint32_t* in, uint32_t* out, uint32_t n, void* scratch,
                                        size_t scratch_bytes, uint64_t first_ticket, mp_stream stream) {
    if (n == 0) return MP_OK;
    if (!in || !out || !scratch) return fail(MP_ERR_INVALID_ARGUMENT, "NULL pointer");
    const size_t need = mp_exclusive_scan_scratch_bytes(n);
    if (scratch_bytes < need)
        return fail(MP_ERR_INVALID_ARGUMENT, "scratch of %zu bytes, need %zu", scratch_bytes, need);
    if (reinterpret_cast<uintptr_t>(scratch) & 7u)
        return fail(MP_ERR_INVALID_ARGUMENT, "scratch must be 8-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    MP_CUDA(cudaMemsetAsync(scratch, 0, need, s));
    // pageable source: the call returns once the value is staged
    const unsigned long long ticket = first_ticket;
    MP_CUDA(cudaMemcpyAsync(scratch, &ticket, sizeof(ticket), cudaMemcpyHostToDevice, s));
    char* b = static_cast<char*>(scratch);
    const cudaError_t e = mpb::launch_scan(in, out, n, reinterpret_cast<unsigned long long*>(b + 256),
                                           reinterpret_cast<unsigned long long*>(b),
                                           mpb::scan_tiles_for(n), false,
                                           reinterpret_cast<uint32_t*>(b + 8), s);
    if (e != cudaSuccess) return fail(MP_ERR_CUDA, "scan launch: %s", cudaGetErrorString(e));
    return MP_OK;
}

int mp_exclusive_scan_status(const void* scratch, mp_stream stream) {
    uint32_t* word = nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (scratch) {
        if (reinterpret_cast<uintptr_t>(scratch) & 7u)
            return fail(MP_ERR_INVALID_ARGUMENT, "scratch must be 8-byte aligned");
        word = reinterpret_cast<uint32_t*>(static_cast<char*>(const_cast<void*>(scratch)) + 8);
    } else {
        const int rc = mpb::noalloc_scan_error_word(s, &word);
        if (rc != MP_OK) return rc;
    }
    uint32_t w = 0;
    MP_CUDA(cudaMemcpyAsync(&w, word, sizeof(w), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (!w) return MP_OK;
    MP_CUDA(cudaMemsetAsync(word, 0, sizeof(w), s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (w & mpb::kDevErrSpin)
        return fail(MP_ERR_SPIN_LIMIT, "the scan's look-back wait gave up: its output is wrong (bits 0x%x)", w);
    return fail(MP_ERR_DEVICE, "scan error word 0x%x", w);
}

}  // extern "C"
