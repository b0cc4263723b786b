// batch.cpp — host side of the multi-scene batch (mp_batch_* in
// include/mtlphys_b200.h): buffers for all scenes, scene seeding, the
// per-step cooperative launch (optionally captured in a CUDA graph), the
// scene-by-scene serial mode and the launch-shape autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/mtlphys_b200.h"
#include "host_common.h"
#include "pbf_adjoint.h"
#include "pbf_batch.h"
#include "pbf_kernels.h"
#include "snapshot.h"

using namespace mpb;

namespace {

struct TuneKey {
    uint32_t n_bucket, scenes;
    bool operator<(const TuneKey& o) const {
        return n_bucket != o.n_bucket ? n_bucket < o.n_bucket : scenes < o.scenes;
    }
};
// Autotuned launch shapes, per particle-count bucket (power of two) and scene count.
std::mutex g_tune_lock;
std::map<TuneKey, std::pair<uint32_t, uint32_t>> g_tune_cache;

uint32_t pow2_bucket(uint32_t n) {
    uint32_t b = 1;
    while (b < n && b < (1u << 31)) b <<= 1;
    return b;
}

}  // namespace

struct mp_batch {
    int device = 0;
    uint32_t S = 0, N = 0, n_alloc = 0, iterations = 0;
    std::vector<uint32_t> counts, p0, scene_ids;
    std::vector<mp_pbf_params> params;
    std::vector<mp_scene_desc> descs;
    std::vector<float> dts;
    std::vector<SceneDev> host_scenes;
    uint32_t max_cells = 0;
    // device memory
    void* particle_block = nullptr;
    void* cell_block = nullptr;
    void* small_block = nullptr;
    SceneDev* scenes = nullptr;
    BatchArgs a{};
    // launch shape / modes
    uint32_t block = 256, blocks_per_sm = 0;
    bool serial = false, graph_mode = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    uint32_t graph_spin_epoch = 0;  // spin limits the captured graph was made with
    uint32_t bar_extra = 0;         // test hook: mp_batch_debug_barrier_extra

    // ---- differentiable rollouts ----
    // One recorded step: the record arrays of the step kernel plus its own
    // prev / sorted index / hash cell / cell start arrays.
    struct Slot {
        BatchRecord rec;
        float4* x0;
        uint32_t *sidx, *scell, *cstart;
    };
    // A saved state: positions, velocities and the scene table (spheres).
    struct Saved {
        float4 *pos, *vel;
        SceneDev* scenes;
    };
    void* tape_block = nullptr;
    std::vector<Slot> slots;
    void* ckpt_block = nullptr;
    std::vector<Saved> ckpts;  // checkpoints, then the saved final state
    void* adj_block = nullptr;
    AdjArgs adj{};
    uint32_t roll_steps = 0, roll_every = 0;
    bool roll_valid = false;

    size_t cap_slots() const { return round_up(std::max<uint32_t>(N, 1u), 256u); }
    static size_t al(size_t bytes) { return (bytes + 255) & ~size_t(255); }

    int ensure_tape(uint32_t nslots) {
        if (slots.size() >= nslots) return MP_OK;
        dev_free(tape_block);
        tape_block = nullptr;
        slots.clear();
        const size_t cap = cap_slots(), K = iterations, v4 = cap * 16, u = cap * 4;
        const size_t per = al(sizeof(SceneDev) * std::max<uint32_t>(S, 1u)) +
                           al(sizeof(SphereState) * std::max<uint32_t>(S, 1u)) + al(v4) + 2 * al(u) +
                           al((size_t(max_cells) + 1) * 4) + K * (2 * al(v4) + al(9 * u) + al(u));
        MP_ALLOC(tape_block, per * nslots, device);
        char* p = static_cast<char*>(tape_block);
        auto take = [&](size_t bytes) {
            char* r = p;
            p += al(bytes);
            return r;
        };
        for (uint32_t i = 0; i < nslots; ++i) {
            Slot sl{};
            sl.rec.scenes = reinterpret_cast<SceneDev*>(take(sizeof(SceneDev) * std::max<uint32_t>(S, 1u)));
            sl.rec.sphere0 = reinterpret_cast<SphereState*>(take(sizeof(SphereState) * std::max<uint32_t>(S, 1u)));
            sl.x0 = reinterpret_cast<float4*>(take(v4));
            sl.sidx = reinterpret_cast<uint32_t*>(take(u));
            sl.scell = reinterpret_cast<uint32_t*>(take(u));
            sl.cstart = reinterpret_cast<uint32_t*>(take((size_t(max_cells) + 1) * 4));
            sl.rec.lam = reinterpret_cast<float4*>(take(K * v4));
            sl.rec.delta = reinterpret_cast<float4*>(take(K * v4));
            sl.rec.masks = reinterpret_cast<uint32_t*>(take(K * 9 * u));
            sl.rec.overflow = reinterpret_cast<uint32_t*>(take(K * u));
            sl.rec.stride = uint32_t(cap);
            if (K == 0) sl.rec.lam = sl.rec.delta = nullptr, sl.rec.masks = sl.rec.overflow = nullptr;
            slots.push_back(sl);
        }
        return MP_OK;
    }

    int ensure_ckpts(uint32_t n) {
        if (ckpts.size() >= n) return MP_OK;
        dev_free(ckpt_block);
        ckpt_block = nullptr;
        ckpts.clear();
        const size_t v4 = cap_slots() * 16, sc = al(sizeof(SceneDev) * std::max<uint32_t>(S, 1u));
        const size_t per = 2 * al(v4) + sc;
        MP_ALLOC(ckpt_block, per * n, device);
        char* p = static_cast<char*>(ckpt_block);
        for (uint32_t i = 0; i < n; ++i) {
            Saved sv{reinterpret_cast<float4*>(p), reinterpret_cast<float4*>(p + al(v4)),
                     reinterpret_cast<SceneDev*>(p + 2 * al(v4))};
            ckpts.push_back(sv);
            p += per;
        }
        return MP_OK;
    }

    int ensure_adjoint() {
        if (adj_block) return MP_OK;
        const size_t cap = cap_slots(), v4 = al(cap * 16), u = al(cap * 4);
        const size_t gbytes = al(sizeof(double) * kGradStride * std::max<uint32_t>(S, 1u));
        // one-way pair inboxes and the overflow list; FP64 per-slot scene-gradient shares
        const size_t inbox = kInbox * (u + v4);
        const size_t ovf = 2 * al(4 * size_t(kInboxOverflow)) + al(16 * size_t(kInboxOverflow)) + 256;
        uint32_t most = 1;
        for (uint32_t c : counts) most = std::max(most, c);
        const uint32_t chunks = (most + kSumChunk - 1) / kSumChunk;
        const size_t accs = al(cap * 8) + al(cap * 32) + al(32 * size_t(chunks) * std::max<uint32_t>(S, 1u));
        const size_t total = 8 * v4 + 7 * u + gbytes + inbox + ovf + accs;
        MP_ALLOC(adj_block, total, device);
        MP_CUDA(cudaMemset(adj_block, 0, total));
        char* p = static_cast<char*>(adj_block);
        auto v = [&]() { float4* r = reinterpret_cast<float4*>(p); p += v4; return r; };
        auto w = [&]() { char* r = p; p += u; return r; };
        auto take = [&](size_t bytes) { char* r = p; p += al(bytes); return r; };
        adj = AdjArgs{};
        adj.pbar = v();
        adj.qbar = v();
        adj.dbar = v();
        adj.lbar = v();
        adj.gd = v();
        adj.p_extra = v();
        adj.xbar = v();
        adj.vbar = v();
        adj.qsc = reinterpret_cast<float*>(w());
        adj.lam_part = reinterpret_cast<float*>(w());
        adj.lam_extra = reinterpret_cast<float*>(w());
        adj.ccur = reinterpret_cast<uint32_t*>(w());
        adj.cpred = reinterpret_cast<uint32_t*>(w());
        adj.inbox_count = reinterpret_cast<uint32_t*>(w());
        adj.ovf_head = reinterpret_cast<uint32_t*>(w());
        MP_CUDA(cudaMemset(adj.ovf_head, 0xff, 4 * cap));  // kNoPost
        adj.inbox_src = reinterpret_cast<uint32_t*>(take(kInbox * u));
        adj.inbox_val = reinterpret_cast<float4*>(take(kInbox * v4));
        adj.ovf_count = reinterpret_cast<uint32_t*>(take(256));
        adj.ovf_src = reinterpret_cast<uint32_t*>(take(4 * size_t(kInboxOverflow)));
        adj.ovf_next = reinterpret_cast<uint32_t*>(take(4 * size_t(kInboxOverflow)));
        adj.ovf_val = reinterpret_cast<float4*>(take(16 * size_t(kInboxOverflow)));
        adj.kacc = reinterpret_cast<double*>(take(cap * 8));
        adj.sacc = reinterpret_cast<double4*>(take(cap * 32));
        adj.spart = reinterpret_cast<double4*>(take(32 * size_t(chunks) * std::max<uint32_t>(S, 1u)));
        adj.sum_chunks = chunks;
        adj.err = a.err;
        adj.grads = reinterpret_cast<double*>(p);
        adj.scene_of = a.scene_of;
        adj.n = N;
        adj.nscenes = S;
        adj.iterations = iterations;
        adj.stride = uint32_t(cap);
        adj.mask_stride = a.mask_stride;
        return MP_OK;
    }

    void free_rollout() {
        for (void* p : {tape_block, ckpt_block, adj_block}) dev_free(p);
        tape_block = ckpt_block = adj_block = nullptr;
        slots.clear();
        ckpts.clear();
        adj = AdjArgs{};
        roll_valid = false;
    }

    int save(const Saved& sv, cudaStream_t s) {
        const size_t v4 = size_t(N) * 16;
        MP_CUDA(cudaMemcpyAsync(sv.pos, a.pos, v4, cudaMemcpyDeviceToDevice, s));
        MP_CUDA(cudaMemcpyAsync(sv.vel, a.vel, v4, cudaMemcpyDeviceToDevice, s));
        MP_CUDA(cudaMemcpyAsync(sv.scenes, scenes, sizeof(SceneDev) * S, cudaMemcpyDeviceToDevice, s));
        return MP_OK;
    }
    int restore(const Saved& sv, cudaStream_t s) {
        const size_t v4 = size_t(N) * 16;
        MP_CUDA(cudaMemcpyAsync(a.pos, sv.pos, v4, cudaMemcpyDeviceToDevice, s));
        MP_CUDA(cudaMemcpyAsync(a.vel, sv.vel, v4, cudaMemcpyDeviceToDevice, s));
        MP_CUDA(cudaMemcpyAsync(scenes, sv.scenes, sizeof(SceneDev) * S, cudaMemcpyDeviceToDevice, s));
        return MP_OK;
    }

    // One step of every scene in one launch, kept in tape slot `i`.
    int enqueue_recorded(uint32_t i, cudaStream_t s) {
        const Slot& sl = slots[i];
        BatchArgs args = launch_args();
        args.scene_begin = 0;
        args.scene_end = S;
        args.p_begin = 0;
        args.p_end = N;
        args.prev = sl.x0;
        args.sidx = sl.sidx;
        args.scell = sl.scell;
        args.cstart = sl.cstart;
        args.rec = sl.rec;
        const cudaError_t e = launch_batch_step(args, block, blocks(), s);
        if (e != cudaSuccess) return fail(MP_ERR_CUDA, "recorded step launch: %s", cudaGetErrorString(e));
        return MP_OK;
    }

    // The reverse of the step kept in slot `i`, whose end positions are x1.
    int enqueue_adjoint(uint32_t i, const float4* x1, cudaStream_t s) {
        const Slot& sl = slots[i];
        AdjArgs ad = adj;
        ad.t = AdjStep{sl.rec.scenes, sl.rec.sphere0, sl.x0, x1, sl.sidx, sl.scell, sl.cstart,
                       sl.rec.lam, sl.rec.delta, sl.rec.masks, sl.rec.overflow};
        const cudaError_t e = launch_adjoint_step(ad, s);
        if (e != cudaSuccess) return fail(MP_ERR_CUDA, "adjoint step launch: %s", cudaGetErrorString(e));
        return MP_OK;
    }

    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    }
    void free_all() {
        drop_graph();
        for (void* p : {particle_block, cell_block, small_block, static_cast<void*>(scenes)}) dev_free(p);
        particle_block = cell_block = small_block = nullptr;
        scenes = nullptr;
        a = BatchArgs{};
    }
    ~mp_batch() {
        DeviceGuard g(device);
        free_rollout();
        free_all();
        if (cap_stream) cudaStreamDestroy(cap_stream);
    }

    uint32_t blocks() const {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int occ = batch_max_blocks_per_sm(block);
        const int per_sm = blocks_per_sm ? std::min<int>(int(blocks_per_sm), occ) : occ;
        return uint32_t(std::max(1, per_sm) * std::max(1, sms));
    }

    // launch arguments with the current bound of the barrier wait
    BatchArgs launch_args() const {
        BatchArgs args = a;
        args.spin_limit = barrier_spin_limit();
        args.bar_extra = bar_extra;
        return args;
    }

    int enqueue(cudaStream_t s) {
        if (N == 0) return MP_OK;
        const uint32_t nb = blocks();
        if (!serial) {
            BatchArgs args = launch_args();
            args.scene_begin = 0;
            args.scene_end = S;
            args.p_begin = 0;
            args.p_end = N;
            const cudaError_t e = launch_batch_step(args, block, nb, s);
            if (e != cudaSuccess) return fail(MP_ERR_CUDA, "batch step launch: %s", cudaGetErrorString(e));
            return MP_OK;
        }
        // The same kernel, one scene per launch, each on a grid no larger
        // than its particles need (a small scene's grid barriers are cheaper
        // on fewer blocks; the results do not depend on the grid).
        for (uint32_t sc = 0; sc < S; ++sc) {
            if (counts[sc] == 0) continue;
            const uint32_t need = uint32_t((uint64_t(counts[sc]) + block - 1) / block);
            BatchArgs args = launch_args();
            args.scene_begin = sc;
            args.scene_end = sc + 1;
            args.p_begin = p0[sc];
            args.p_end = p0[sc] + counts[sc];
            const cudaError_t e = launch_batch_step(args, block, std::min(nb, need), s);
            if (e != cudaSuccess) return fail(MP_ERR_CUDA, "batch step launch: %s", cudaGetErrorString(e));
        }
        return MP_OK;
    }

    // One step of every scene (graph replay in graph mode).
    int step(cudaStream_t s) {
        if (!graph_mode) return enqueue(s);
        if (gexec && graph_spin_epoch != spin_limit_epoch()) drop_graph();
        if (!gexec) {
            if (!cap_stream) MP_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
            MP_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue(cap_stream);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(cap_stream, &g);
            if (rc != MP_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ce != cudaSuccess) return fail(MP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
            graph = g;
            MP_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
            graph_spin_epoch = spin_limit_epoch();
        }
        MP_CUDA(cudaGraphLaunch(gexec, s));
        return MP_OK;
    }

    int upload_scenes() {
        MP_CUDA(cudaMemcpy(scenes, host_scenes.data(), sizeof(SceneDev) * S, cudaMemcpyHostToDevice));
        return MP_OK;
    }
};

namespace {

int batch_buffer(mp_batch* b, uint32_t which, void** dptr, size_t* bytes) {
    if (!b || !dptr) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    void* p = nullptr;
    size_t count = b->N;
    switch (which) {
        case MP_BUF_POSITIONS: p = b->a.pos; break;
        case MP_BUF_VELOCITIES: p = b->a.vel; break;
        case MP_BUF_PREV_POSITIONS: p = b->a.prev; break;
        case MP_BUF_CELL_HASHES: p = b->a.hash; break;
        case MP_BUF_CELL_START: p = b->a.cstart; count = size_t(b->max_cells) + 1; break;
        case MP_BUF_SORTED_INDEX: p = b->a.sidx; break;
        case MP_BUF_NEIGHBOR_COUNTS: p = b->a.ncount; break;
        case MP_BUF_LAMBDAS: p = b->a.lambdas; break;
        case MP_BUF_FOAM: p = b->a.foam; break;
        case MP_BUF_SORTED_POSITIONS: p = b->a.sorted_a; break;
        default: return fail(MP_ERR_INVALID_ARGUMENT, "unknown buffer %u", which);
    }
    *dptr = p;
    if (bytes) *bytes = count * elem_bytes(which);
    return MP_OK;
}

}  // namespace

extern "C" {

int mp_batch_create(int device, mp_batch** out) {
    if (!out) return fail(MP_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int count = 0;
    MP_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
        return fail(MP_ERR_INVALID_ARGUMENT, "device %d not in [0, %d)", device, count);
    int coop = 0;
    MP_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    if (!coop) return fail(MP_ERR_UNSUPPORTED, "device %d has no cooperative launch", device);
    auto* b = new (std::nothrow) mp_batch();
    if (!b) return fail(MP_ERR_OUT_OF_MEMORY, "host allocation failed");
    b->device = device;
    *out = b;
    return MP_OK;
}

int mp_batch_destroy(mp_batch* b) {
    delete b;
    return MP_OK;
}

int mp_batch_reset(mp_batch* b, uint32_t nscenes, const uint32_t* counts, const uint32_t* scene_ids,
                   const mp_pbf_params* params, const mp_scene_desc* descs, const float* dts) {
    if (!b || (nscenes && (!counts || !params || !dts)))
        return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    uint64_t total = 0;
    const uint32_t iters = nscenes ? params[0].solver_iterations : 0;
    uint64_t worst_cells = 0;
    std::vector<GridDev> grids(nscenes);
    for (uint32_t s = 0; s < nscenes; ++s) {
        int rc = validate_params(params[s]);
        if (rc != MP_OK) return rc;
        if (params[s].solver_iterations != iters)
            return fail(MP_ERR_INVALID_ARGUMENT, "all scenes must use the same solver_iterations");
        if (!(dts[s] > 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u: dt must be > 0", s);
        if (scene_ids && scene_ids[s] > MP_SCENE_SPHERE_DROP)
            return fail(MP_ERR_INVALID_ARGUMENT, "scene %u: unknown scene id %u", s, scene_ids[s]);
        if (descs && descs[s].size != sizeof(mp_scene_desc))
            return fail(MP_ERR_INVALID_ARGUMENT, "scene %u: mp_scene_desc.size mismatch", s);
        rc = make_grid(params[s], grids[s]);
        if (rc != MP_OK) return rc;
        total += counts[s];
        worst_cells += grids[s].cells;
    }
    if (total >= (1ull << 31)) return fail(MP_ERR_INVALID_ARGUMENT, "too many particles");
    if (worst_cells >= (1ull << 31) - 1) return fail(MP_ERR_INVALID_ARGUMENT, "scene grids too large");
    // seed every scene on the host
    std::vector<float> pos(4 * size_t(total), 0.0f), tmp;
    std::vector<uint32_t> scene_of(total);
    std::vector<SceneDev> hs(nscenes);
    uint64_t off = 0;
    for (uint32_t s = 0; s < nscenes; ++s) {
        mp_scene_desc d;
        if (descs) d = descs[s];
        else fill_default_desc(d);
        const uint32_t sid = scene_ids ? scene_ids[s] : MP_SCENE_CUBE_DROP;
        const int rc = seed_scene(params[s], sid, d, counts[s], tmp);
        if (rc != MP_OK) return rc;
        std::copy(tmp.begin(), tmp.end(), pos.begin() + 4 * off);
        std::fill(scene_of.begin() + off, scene_of.begin() + off + counts[s], s);
        std::memset(&hs[s], 0, sizeof(SceneDev));
        hs[s].c = make_consts(params[s], grids[s], counts[s], dts[s], sid == MP_SCENE_SPHERE_DROP);
        hs[s].p0 = uint32_t(off);
        for (int a = 0; a < 3; ++a) {
            hs[s].sphere.c[a] = d.sphere_center[a];
            hs[s].sphere.v[a] = d.sphere_velocity[a];
        }
        hs[s].sphere.r = params[s].sphere_radius;
        off += counts[s];
    }
    DeviceGuard g(b->device);
    b->free_rollout();
    b->free_all();
    b->S = nscenes;
    b->N = uint32_t(total);
    b->iterations = iters;
    b->counts.assign(counts, counts + nscenes);
    b->scene_ids.assign(nscenes, MP_SCENE_CUBE_DROP);
    if (scene_ids) b->scene_ids.assign(scene_ids, scene_ids + nscenes);
    b->params.assign(params, params + nscenes);
    b->descs.resize(nscenes);
    for (uint32_t s = 0; s < nscenes; ++s) {
        if (descs) b->descs[s] = descs[s];
        else fill_default_desc(b->descs[s]);
    }
    b->dts.assign(dts, dts + nscenes);
    b->p0.resize(nscenes);
    for (uint32_t s = 0; s < nscenes; ++s) b->p0[s] = hs[s].p0;
    b->host_scenes = hs;
    b->max_cells = uint32_t(worst_cells);
    // A failed allocation leaves the batch empty (no scenes), not half-built.
    const int arc = [&]() -> int {
        // particles
        const uint32_t cap = round_up(std::max<uint32_t>(b->N, 1u), 256u);
        const size_t v4 = size_t(cap) * 16, u = size_t(cap) * 4;
        const size_t longs = (size_t(cap) / kSegMax + 2) * 4;
        const size_t ptotal = 5 * v4 + 19 * u + longs + 32 * 256;
        MP_ALLOC(b->particle_block, ptotal, b->device);
        MP_CUDA(cudaMemset(b->particle_block, 0, ptotal));
        char* pb = static_cast<char*>(b->particle_block);
        auto take = [&](size_t bytes) {
            char* r = pb;
            pb += (bytes + 255) & ~size_t(255);
            return r;
        };
        BatchArgs& a = b->a;
        a.pos = reinterpret_cast<float4*>(take(v4));
        a.vel = reinterpret_cast<float4*>(take(v4));
        a.prev = reinterpret_cast<float4*>(take(v4));
        a.sorted_a = reinterpret_cast<float4*>(take(v4));
        a.sorted_b = reinterpret_cast<float4*>(take(v4));
        a.hash = reinterpret_cast<uint32_t*>(take(u));
        a.off = reinterpret_cast<uint32_t*>(take(u));
        a.tmp = reinterpret_cast<uint32_t*>(take(u));
        a.sidx = reinterpret_cast<uint32_t*>(take(u));
        a.scell = reinterpret_cast<uint32_t*>(take(u));
        a.ncount = reinterpret_cast<uint32_t*>(take(u));
        a.lambdas = reinterpret_cast<float*>(take(u));
        a.foam = reinterpret_cast<float*>(take(u));
        uint32_t* so = reinterpret_cast<uint32_t*>(take(u));
        a.scene_of = so;
        a.row_masks = reinterpret_cast<uint32_t*>(take(9 * u));
        a.mask_overflow = reinterpret_cast<uint32_t*>(take(u));
        a.mask_stride = cap;
        a.long_list = reinterpret_cast<uint32_t*>(take(longs));
        // cells: counts + cstart for the worst case (every scene's whole box)
        const size_t clen = size_t(b->max_cells) + 1;
        const size_t tiles = clen / 128 + 2;
        const size_t cbytes = ((clen * 4 + 255) & ~size_t(255));
        MP_ALLOC(b->cell_block, 2 * cbytes + tiles * 4, b->device);
        MP_CUDA(cudaMemset(b->cell_block, 0, 2 * cbytes + tiles * 4));
        a.counts = static_cast<uint32_t*>(b->cell_block);
        a.cstart = reinterpret_cast<uint32_t*>(static_cast<char*>(b->cell_block) + cbytes);
        a.tile_sums = reinterpret_cast<uint32_t*>(static_cast<char*>(b->cell_block) + 2 * cbytes);
        a.max_cells = b->max_cells;
        MP_ALLOC(b->small_block, 256, b->device);
        MP_CUDA(cudaMemset(b->small_block, 0, 256));
        uint32_t* sm = static_cast<uint32_t*>(b->small_block);
        a.long_count = sm + 0;
        a.total_cells = sm + 1;
        a.err = sm + 2;
        a.bar_count = reinterpret_cast<unsigned*>(sm + 32);
        a.bar_gen = reinterpret_cast<unsigned*>(sm + 33);
        a.abort = sm + 48;
        MP_ALLOC(b->scenes, sizeof(SceneDev) * std::max<uint32_t>(nscenes, 1u), b->device);
        a.scenes = b->scenes;
        a.iterations = iters;
        a.scorr4 = 1;
        for (uint32_t s = 0; s < nscenes; ++s)
            if (params[s].scorr_n != 4) a.scorr4 = 0;
        int rc = b->upload_scenes();
        if (rc != MP_OK) return rc;
        if (total) {
            MP_CUDA(cudaMemcpy(a.pos, pos.data(), 16 * size_t(total), cudaMemcpyHostToDevice));
            MP_CUDA(cudaMemcpy(so, scene_of.data(), 4 * size_t(total), cudaMemcpyHostToDevice));
        }
        return MP_OK;
    }();
    if (arc != MP_OK) {
        b->free_all();
        b->S = b->N = 0;
        b->counts.clear();
        b->p0.clear();
        b->scene_ids.clear();
        b->params.clear();
        b->descs.clear();
        b->dts.clear();
        b->host_scenes.clear();
        b->max_cells = 0;
        return arc;
    }
    // launch shape: the cached autotuning result for this size, if any
    {
        std::lock_guard<std::mutex> lock(g_tune_lock);
        auto it = g_tune_cache.find({pow2_bucket(b->N), b->S});
        if (it != g_tune_cache.end()) {
            b->block = it->second.first;
            b->blocks_per_sm = it->second.second;
        }
    }
    MP_CUDA(cudaDeviceSynchronize());
    return MP_OK;
}

int mp_batch_set_dts(mp_batch* b, const float* dts) {
    if (!b || (b->S && !dts)) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    for (uint32_t s = 0; s < b->S; ++s) {
        if (!(dts[s] > 0.0f)) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u: dt must be > 0", s);
    }
    DeviceGuard g(b->device);
    b->roll_valid = false;
    MP_CUDA(cudaDeviceSynchronize());
    // refresh the constants that depend on dt, keep the device-side sphere state
    std::vector<SceneDev> cur(b->S);
    if (b->S) MP_CUDA(cudaMemcpy(cur.data(), b->scenes, sizeof(SceneDev) * b->S, cudaMemcpyDeviceToHost));
    for (uint32_t s = 0; s < b->S; ++s) {
        GridDev g0;
        make_grid(b->params[s], g0);
        cur[s].c = make_consts(b->params[s], g0, b->counts[s], dts[s],
                               b->scene_ids[s] == MP_SCENE_SPHERE_DROP);
        b->dts[s] = dts[s];
    }
    if (b->S) MP_CUDA(cudaMemcpy(b->scenes, cur.data(), sizeof(SceneDev) * b->S, cudaMemcpyHostToDevice));
    b->drop_graph();
    return MP_OK;
}

int mp_batch_step(mp_batch* b, mp_stream stream) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    DeviceGuard g(b->device);
    b->roll_valid = false;
    return b->step(static_cast<cudaStream_t>(stream));
}

int mp_batch_set_mode(mp_batch* b, int serial) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    b->serial = serial != 0;
    b->drop_graph();
    return MP_OK;
}

int mp_batch_set_graph_mode(mp_batch* b, int enable) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    DeviceGuard g(b->device);
    b->graph_mode = enable != 0;
    b->drop_graph();
    return MP_OK;
}

int mp_batch_set_launch(mp_batch* b, uint32_t block, uint32_t blocks_per_sm) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    DeviceGuard g(b->device);
    const int occ = batch_max_blocks_per_sm(block);
    if (occ <= 0) return fail(MP_ERR_INVALID_ARGUMENT, "block size %u is not 128, 256 or 512", block);
    if (blocks_per_sm > uint32_t(occ))
        return fail(MP_ERR_INVALID_ARGUMENT, "%u blocks/SM exceed the %d that fit", blocks_per_sm, occ);
    b->block = block;
    b->blocks_per_sm = blocks_per_sm;
    b->drop_graph();
    return MP_OK;
}

int mp_batch_get_launch(const mp_batch* b, uint32_t* block, uint32_t* blocks) {
    if (!b || !block || !blocks) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    *block = b->block;
    *blocks = b->blocks();
    return MP_OK;
}

int mp_batch_autotune(mp_batch* b, uint32_t steps, mp_batch_tuning* best) {
    if (!b || steps == 0) return fail(MP_ERR_INVALID_ARGUMENT, "bad argument");
    DeviceGuard g(b->device);
    if (b->N == 0) return MP_OK;
    // Each candidate runs `steps` steps from the same saved state, which is
    // restored afterwards: tuning does not advance the simulation.
    const size_t v4 = size_t(b->N) * 16;
    void* save = nullptr;
    MP_ALLOC(save, 2 * v4 + sizeof(SceneDev) * b->S, b->device);
    auto snapshot = [&](bool restore) -> int {
        char* sv = static_cast<char*>(save);
        const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
        if (restore) {
            MP_CUDA(cudaMemcpy(b->a.pos, sv, v4, k));
            MP_CUDA(cudaMemcpy(b->a.vel, sv + v4, v4, k));
            MP_CUDA(cudaMemcpy(b->scenes, sv + 2 * v4, sizeof(SceneDev) * b->S, k));
        } else {
            MP_CUDA(cudaMemcpy(sv, b->a.pos, v4, k));
            MP_CUDA(cudaMemcpy(sv + v4, b->a.vel, v4, k));
            MP_CUDA(cudaMemcpy(sv + 2 * v4, b->scenes, sizeof(SceneDev) * b->S, k));
        }
        return MP_OK;
    };
    int rc = snapshot(false);
    const uint32_t saved_block = b->block, saved_bps = b->blocks_per_sm;
    const bool saved_graph = b->graph_mode;
    b->graph_mode = false;
    b->drop_graph();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_ms = 1e30f;
    uint32_t best_block = saved_block, best_bps = saved_bps;
    for (uint32_t block : {128u, 256u, 512u}) {
        const int occ = batch_max_blocks_per_sm(block);
        for (int bps = 1; rc == MP_OK && bps <= occ; ++bps) {
            b->block = block;
            b->blocks_per_sm = uint32_t(bps);
            rc = snapshot(true);
            if (rc != MP_OK) break;
            rc = b->enqueue(nullptr);  // warm-up step
            cudaEventRecord(e0);
            for (uint32_t i = 0; rc == MP_OK && i < steps; ++i) rc = b->enqueue(nullptr);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(MP_ERR_CUDA, "autotune sync failed");
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= float(steps);
            if (rc == MP_OK && ms < best_ms) {
                best_ms = ms;
                best_block = block;
                best_bps = uint32_t(bps);
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int rc2 = snapshot(true);
    dev_free(save);
    b->graph_mode = saved_graph;
    if (rc != MP_OK || rc2 != MP_OK) {
        b->block = saved_block;
        b->blocks_per_sm = saved_bps;
        return rc != MP_OK ? rc : rc2;
    }
    b->block = best_block;
    b->blocks_per_sm = best_bps;
    {
        std::lock_guard<std::mutex> lock(g_tune_lock);
        g_tune_cache[{pow2_bucket(b->N), b->S}] = {best_block, best_bps};
    }
    if (best) {
        best->block = best_block;
        best->blocks_per_sm = best_bps;
        best->ms_per_step = best_ms;
    }
    MP_CUDA(cudaDeviceSynchronize());
    return MP_OK;
}

uint32_t mp_batch_scene_count(const mp_batch* b) { return b ? b->S : 0; }
uint32_t mp_batch_particle_count(const mp_batch* b) { return b ? b->N : 0; }

int mp_batch_scene_range(const mp_batch* b, uint32_t scene, uint32_t* first, uint32_t* count) {
    if (!b || !first || !count) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (scene >= b->S) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u >= %u", scene, b->S);
    *first = b->p0[scene];
    *count = b->counts[scene];
    return MP_OK;
}

int mp_batch_buffer(mp_batch* b, uint32_t which, void** dptr, size_t* bytes) {
    return batch_buffer(b, which, dptr, bytes);
}

int mp_batch_upload(mp_batch* b, uint32_t which, const void* host, size_t count, mp_stream stream) {
    void* dptr = nullptr;
    size_t bytes = 0;
    int rc = batch_buffer(b, which, &dptr, &bytes);
    if (rc != MP_OK) return rc;
    const size_t need = count * elem_bytes(which);
    if (!host && count) return fail(MP_ERR_INVALID_ARGUMENT, "host is NULL");
    if (need > bytes) return fail(MP_ERR_INVALID_ARGUMENT, "%zu elements exceed buffer %u", count, which);
    if (!need) return MP_OK;
    DeviceGuard g(b->device);
    b->roll_valid = false;
    MP_CUDA(cudaMemcpyAsync(dptr, host, need, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)));
    return MP_OK;
}

int mp_batch_download(mp_batch* b, uint32_t which, void* host, size_t count, mp_stream stream) {
    void* dptr = nullptr;
    size_t bytes = 0;
    int rc = batch_buffer(b, which, &dptr, &bytes);
    if (rc != MP_OK) return rc;
    const size_t need = count * elem_bytes(which);
    if (!host && count) return fail(MP_ERR_INVALID_ARGUMENT, "host is NULL");
    if (need > bytes) return fail(MP_ERR_INVALID_ARGUMENT, "%zu elements exceed buffer %u", count, which);
    DeviceGuard g(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (need) MP_CUDA(cudaMemcpyAsync(host, dptr, need, cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

int mp_batch_set_sphere(mp_batch* b, uint32_t scene, const float center[3], const float velocity[3],
                        float radius) {
    if (!b || !center || !velocity) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (scene >= b->S) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u >= %u", scene, b->S);
    SphereState s{};
    for (int a = 0; a < 3; ++a) {
        s.c[a] = center[a];
        s.v[a] = velocity[a];
    }
    s.r = radius;
    DeviceGuard g(b->device);
    b->roll_valid = false;
    MP_CUDA(cudaDeviceSynchronize());
    MP_CUDA(cudaMemcpy(&b->scenes[scene].sphere, &s, sizeof(s), cudaMemcpyHostToDevice));
    return MP_OK;
}

int mp_batch_get_sphere(mp_batch* b, uint32_t scene, float center[3], float velocity[3], float* radius) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    if (scene >= b->S) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u >= %u", scene, b->S);
    SphereState s{};
    DeviceGuard g(b->device);
    MP_CUDA(cudaDeviceSynchronize());
    MP_CUDA(cudaMemcpy(&s, &b->scenes[scene].sphere, sizeof(s), cudaMemcpyDeviceToHost));
    for (int a = 0; a < 3; ++a) {
        if (center) center[a] = s.c[a];
        if (velocity) velocity[a] = s.v[a];
    }
    if (radius) *radius = s.r;
    return MP_OK;
}

int mp_batch_set_params(mp_batch* b, uint32_t scene, const mp_pbf_params* params) {
    if (!b || !params) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (scene >= b->S) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u >= %u", scene, b->S);
    int rc = validate_params(*params);
    if (rc != MP_OK) return rc;
    if (params->solver_iterations != b->iterations)
        return fail(MP_ERR_INVALID_ARGUMENT, "all scenes must use the same solver_iterations");
    GridDev g0, g1;
    make_grid(b->params[scene], g0);
    rc = make_grid(*params, g1);
    if (rc != MP_OK) return rc;
    if (g0.dgx != g1.dgx || g0.dgy != g1.dgy || g0.dgz != g1.dgz || g0.ox != g1.ox || g0.oy != g1.oy ||
        g0.oz != g1.oz || g0.cs != g1.cs)
        return fail(MP_ERR_INVALID_ARGUMENT, "the hash grid (box, cell size) cannot change without a reset");
    DeviceGuard g(b->device);
    b->roll_valid = false;
    MP_CUDA(cudaDeviceSynchronize());
    SceneDev cur;
    MP_CUDA(cudaMemcpy(&cur, &b->scenes[scene], sizeof(SceneDev), cudaMemcpyDeviceToHost));
    cur.c = make_consts(*params, g1, b->counts[scene], b->dts[scene],
                        b->scene_ids[scene] == MP_SCENE_SPHERE_DROP);
    MP_CUDA(cudaMemcpy(&b->scenes[scene], &cur, sizeof(SceneDev), cudaMemcpyHostToDevice));
    b->params[scene] = *params;
    b->a.scorr4 = 1;
    for (const mp_pbf_params& q : b->params)
        if (q.scorr_n != 4) b->a.scorr4 = 0;
    b->host_scenes[scene].c = cur.c;
    b->drop_graph();
    return MP_OK;
}

int mp_batch_get_params(const mp_batch* b, uint32_t scene, mp_pbf_params* params) {
    if (!b || !params) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (scene >= b->S) return fail(MP_ERR_INVALID_ARGUMENT, "scene %u >= %u", scene, b->S);
    *params = b->params[scene];
    return MP_OK;
}

int mp_batch_rollout_forward(mp_batch* b, uint32_t steps, uint32_t checkpoint_every, mp_stream stream) {
    if (!b || checkpoint_every == 0) return fail(MP_ERR_INVALID_ARGUMENT, "bad argument");
    for (uint32_t s = 0; s < b->S; ++s) {
        GridDev g0;
        make_grid(b->params[s], g0);
        if (g0.dgx > 2048 || g0.dgy > 2048 || g0.dgz > 1024)
            return fail(MP_ERR_UNSUPPORTED, "scene %u: the adjoint needs a hash grid of at most "
                        "2048 x 2048 x 1024 cells", s);
    }
    DeviceGuard g(b->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    b->roll_valid = false;
    const uint32_t nck = (steps + checkpoint_every - 1) / checkpoint_every;
    int rc = b->ensure_ckpts(nck + 1);  // + the final state, saved by the backward pass
    for (uint32_t t = 0; rc == MP_OK && t < steps; ++t) {
        if (t % checkpoint_every == 0) rc = b->save(b->ckpts[t / checkpoint_every], st);
        if (rc == MP_OK) rc = b->step(st);
    }
    if (rc != MP_OK) return rc;
    b->roll_steps = steps;
    b->roll_every = checkpoint_every;
    b->roll_valid = true;
    return MP_OK;
}

int mp_batch_rollout_backward(mp_batch* b, const float* dpos, const float* dvel, float* dpos0, float* dvel0,
                              double* dscene, mp_stream stream) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    if (!b->roll_valid)
        return fail(MP_ERR_INVALID_ARGUMENT, "no rollout recorded since the state last changed");
    DeviceGuard g(b->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t steps = b->roll_steps, every = b->roll_every;
    const uint32_t nck = (steps + every - 1) / every;
    int rc = b->ensure_tape(std::min(steps, every));
    if (rc == MP_OK) rc = b->ensure_adjoint();
    if (rc != MP_OK) return rc;
    const size_t v4 = size_t(b->N) * 16;
    AdjArgs& ad = b->adj;
    if (dpos) MP_CUDA(cudaMemcpyAsync(ad.xbar, dpos, v4, cudaMemcpyDeviceToDevice, st));
    else MP_CUDA(cudaMemsetAsync(ad.xbar, 0, v4, st));
    if (dvel) MP_CUDA(cudaMemcpyAsync(ad.vbar, dvel, v4, cudaMemcpyDeviceToDevice, st));
    else MP_CUDA(cudaMemsetAsync(ad.vbar, 0, v4, st));
    MP_CUDA(cudaMemsetAsync(ad.grads, 0, sizeof(double) * kGradStride * b->S, st));
    MP_CUDA(cudaMemsetAsync(ad.kacc, 0, sizeof(double) * b->N, st));
    MP_CUDA(cudaMemsetAsync(ad.sacc, 0, sizeof(double4) * b->N, st));
    MP_CUDA(cudaMemsetAsync(ad.inbox_count, 0, sizeof(uint32_t) * b->N, st));
    MP_CUDA(cudaMemsetAsync(ad.ovf_head, 0xff, sizeof(uint32_t) * b->N, st));
    const mp_batch::Saved& fin = b->ckpts[nck];
    rc = b->save(fin, st);
    for (uint32_t seg = nck; rc == MP_OK && seg-- > 0;) {
        const uint32_t t0 = seg * every, t1 = std::min(steps, t0 + every);
        rc = b->restore(b->ckpts[seg], st);
        for (uint32_t t = t0; rc == MP_OK && t < t1; ++t) rc = b->enqueue_recorded(t - t0, st);
        for (uint32_t t = t1; rc == MP_OK && t-- > t0;) {
            const float4* x1 = t + 1 == t1 ? b->a.pos : b->slots[t + 1 - t0].x0;
            rc = b->enqueue_adjoint(t - t0, x1, st);
        }
    }
    if (rc == MP_OK) {  // dL/dk of every scene from the per-slot shares
        AdjArgs fa = ad;
        fa.t.scenes = b->slots[0].rec.scenes;
        const cudaError_t e = launch_adjoint_finish(fa, st);
        if (e != cudaSuccess) rc = fail(MP_ERR_CUDA, "adjoint finish launch: %s", cudaGetErrorString(e));
    }
    if (rc == MP_OK) rc = b->restore(fin, st);
    if (rc != MP_OK) return rc;
    if (dpos0) MP_CUDA(cudaMemcpyAsync(dpos0, ad.xbar, v4, cudaMemcpyDeviceToDevice, st));
    if (dvel0) MP_CUDA(cudaMemcpyAsync(dvel0, ad.vbar, v4, cudaMemcpyDeviceToDevice, st));
    if (dscene)
        MP_CUDA(cudaMemcpyAsync(dscene, ad.grads, sizeof(double) * kGradStride * b->S,
                                cudaMemcpyDeviceToDevice, st));
    return MP_OK;
}

uint32_t mp_batch_rollout_launch_count(const mp_batch* b, uint32_t steps) {
    if (!b || b->N == 0) return 0;
    return steps * (1u + adjoint_launch_count(b->iterations)) + (steps ? 1u : 0u);
}

size_t mp_batch_snapshot_size(const mp_batch* b) {
    return b ? mpb::snapshot_bytes(b->S, b->N) : 0;
}

int mp_batch_snapshot(mp_batch* b, void* host, size_t bytes) {
    if (!b || !host) return fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t need = mpb::snapshot_bytes(b->S, b->N);
    if (bytes < need) return fail(MP_ERR_INVALID_ARGUMENT, "snapshot needs %zu bytes, got %zu", need, bytes);
    DeviceGuard g(b->device);
    MP_CUDA(cudaDeviceSynchronize());
    char* out = static_cast<char*>(host);
    mpb::SnapshotHeader h;
    mpb::snapshot_header(h, mpb::kSnapshotBatch, b->S, b->N);
    std::memcpy(out, &h, sizeof(h));
    std::vector<SceneDev> cur(b->S);
    if (b->S) MP_CUDA(cudaMemcpy(cur.data(), b->scenes, sizeof(SceneDev) * b->S, cudaMemcpyDeviceToHost));
    for (uint32_t s = 0; s < b->S; ++s) {
        mpb::SnapshotScene sc;
        std::memset(&sc, 0, sizeof(sc));
        sc.params = b->params[s];
        sc.desc = b->descs[s];
        sc.scene_id = b->scene_ids[s];
        sc.count = b->counts[s];
        sc.dt = b->dts[s];
        for (int a = 0; a < 3; ++a) {
            sc.sphere[a] = cur[s].sphere.c[a];
            sc.sphere[3 + a] = cur[s].sphere.v[a];
        }
        sc.sphere[6] = cur[s].sphere.r;
        std::memcpy(out + sizeof(h) + s * sizeof(sc), &sc, sizeof(sc));
    }
    char* arrays = out + sizeof(h) + size_t(b->S) * sizeof(mpb::SnapshotScene);
    if (b->N) {
        MP_CUDA(cudaMemcpy(arrays, b->a.pos, 16 * size_t(b->N), cudaMemcpyDeviceToHost));
        MP_CUDA(cudaMemcpy(arrays + 16 * size_t(b->N), b->a.vel, 16 * size_t(b->N), cudaMemcpyDeviceToHost));
    }
    return MP_OK;
}

int mp_batch_restore(mp_batch* b, const void* host, size_t bytes) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    if (const char* why = mpb::snapshot_check(host, bytes, mpb::kSnapshotBatch))
        return fail(MP_ERR_INVALID_ARGUMENT, "%s", why);
    const char* in = static_cast<const char*>(host);
    mpb::SnapshotHeader h;
    std::memcpy(&h, in, sizeof(h));
    std::vector<mpb::SnapshotScene> sc(h.nscenes);
    uint64_t total = 0;
    for (uint32_t s = 0; s < h.nscenes; ++s) {
        std::memcpy(&sc[s], in + sizeof(h) + s * sizeof(mpb::SnapshotScene), sizeof(mpb::SnapshotScene));
        total += sc[s].count;
    }
    if (total != h.particles) return fail(MP_ERR_INVALID_ARGUMENT, "snapshot particle counts disagree");
    std::vector<uint32_t> counts(h.nscenes), ids(h.nscenes);
    std::vector<mp_pbf_params> params(h.nscenes);
    std::vector<mp_scene_desc> descs(h.nscenes);
    std::vector<float> dts(h.nscenes);
    for (uint32_t s = 0; s < h.nscenes; ++s) {
        counts[s] = sc[s].count;
        ids[s] = sc[s].scene_id;
        params[s] = sc[s].params;
        descs[s] = sc[s].desc;
        dts[s] = sc[s].dt;
    }
    int rc = mp_batch_reset(b, h.nscenes, counts.data(), ids.data(), params.data(), descs.data(), dts.data());
    if (rc != MP_OK) return rc;
    DeviceGuard g(b->device);
    const char* arrays = in + sizeof(h) + size_t(h.nscenes) * sizeof(mpb::SnapshotScene);
    if (b->N) {
        MP_CUDA(cudaMemcpy(b->a.pos, arrays, 16 * size_t(b->N), cudaMemcpyHostToDevice));
        MP_CUDA(cudaMemcpy(b->a.vel, arrays + 16 * size_t(b->N), 16 * size_t(b->N), cudaMemcpyHostToDevice));
    }
    for (uint32_t s = 0; s < h.nscenes && rc == MP_OK; ++s)
        rc = mp_batch_set_sphere(b, s, sc[s].sphere, sc[s].sphere + 3, sc[s].sphere[6]);
    return rc;
}

int mp_batch_check_errors(mp_batch* b, uint32_t* bits) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    DeviceGuard g(b->device);
    MP_CUDA(cudaDeviceSynchronize());
    uint32_t w = 0;
    if (b->a.err) {
        MP_CUDA(cudaMemcpy(&w, b->a.err, 4, cudaMemcpyDeviceToHost));
        MP_CUDA(cudaMemset(b->a.err, 0, 4));
        if (w & kDevErrSpin) {
            // a barrier wait gave up: the launch left the barrier counter
            // mid-count and the abort flag set; re-arm both
            MP_CUDA(cudaMemset(b->a.bar_count, 0, sizeof(unsigned)));
            MP_CUDA(cudaMemset(b->a.abort, 0, sizeof(uint32_t)));
        }
    }
    if (bits) *bits = w;
    if (w & kDevErrSpin) return fail(MP_ERR_SPIN_LIMIT, "a bounded device wait gave up (bits 0x%x)", w);
    if (w) return fail(MP_ERR_DEVICE, "device error word 0x%x", w);
    return MP_OK;
}

int mp_batch_debug_barrier_extra(mp_batch* b, uint32_t extra) {
    if (!b) return fail(MP_ERR_INVALID_ARGUMENT, "NULL batch");
    if (extra > 1024) return fail(MP_ERR_INVALID_ARGUMENT, "extra = %u > 1024", extra);
    b->bar_extra = extra;
    b->drop_graph();
    return MP_OK;
}

}  // extern "C"
