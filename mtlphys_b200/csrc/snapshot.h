// snapshot.h — binary layout of engine and batch state snapshots
// (mp_engine_snapshot / mp_batch_snapshot; no reference counterpart: the
// reference keeps its state only in its Metal buffers).
//
// Little-endian, packed as the structs below:
//   SnapshotHeader
//   nscenes x SnapshotScene
//   particles x float4 positions, particles x float4 velocities
// (original particle order; a batch's scenes back to back).
// mtlphys_b200/snapshot.py reads and writes the same layout.
#pragma once

#include <cstdint>
#include <cstring>

#include "../../include/mtlphys_b200.h"

namespace mpb {

constexpr char kSnapshotMagic[8] = {'M', 'T', 'L', 'P', 'S', 'N', 'A', 'P'};
constexpr uint32_t kSnapshotVersion = 1;
constexpr uint32_t kSnapshotEngine = 0, kSnapshotBatch = 1;

struct SnapshotHeader {
    char magic[8];
    uint32_t version;
    uint32_t kind;         // kSnapshotEngine or kSnapshotBatch
    uint32_t nscenes;
    uint32_t particles;
    uint32_t params_size;  // sizeof(mp_pbf_params)
    uint32_t scene_size;   // sizeof(SnapshotScene)
    uint32_t desc_size;    // sizeof(mp_scene_desc)
    uint32_t reserved[7];
};
static_assert(sizeof(SnapshotHeader) == 64, "snapshot header layout");

struct SnapshotScene {
    mp_pbf_params params;
    mp_scene_desc desc;    // how the scene was seeded
    uint32_t scene_id;     // MP_SCENE_*
    uint32_t count;        // particles of the scene
    float dt;              // a batch scene's time step; 0 for an engine
    float sphere[7];       // sphere center, velocity, radius at snapshot time
};

inline size_t snapshot_bytes(uint32_t nscenes, uint32_t particles) {
    return sizeof(SnapshotHeader) + size_t(nscenes) * sizeof(SnapshotScene) + 32 * size_t(particles);
}

inline void snapshot_header(SnapshotHeader& h, uint32_t kind, uint32_t nscenes, uint32_t particles) {
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kSnapshotMagic, 8);
    h.version = kSnapshotVersion;
    h.kind = kind;
    h.nscenes = nscenes;
    h.particles = particles;
    h.params_size = sizeof(mp_pbf_params);
    h.scene_size = sizeof(SnapshotScene);
    h.desc_size = sizeof(mp_scene_desc);
}

// Checks a snapshot of `bytes` bytes: magic, version, kind, struct sizes and
// total size.  Returns nullptr if it is valid, else the reason.
inline const char* snapshot_check(const void* data, size_t bytes, uint32_t kind) {
    if (!data) return "snapshot is NULL";
    if (bytes < sizeof(SnapshotHeader)) return "snapshot shorter than its header";
    SnapshotHeader h;
    std::memcpy(&h, data, sizeof(h));
    if (std::memcmp(h.magic, kSnapshotMagic, 8) != 0) return "not a snapshot (bad magic)";
    if (h.version != kSnapshotVersion) return "unsupported snapshot version";
    if (h.kind != kind) return kind == kSnapshotEngine ? "not an engine snapshot" : "not a batch snapshot";
    if (h.params_size != sizeof(mp_pbf_params) || h.scene_size != sizeof(SnapshotScene) ||
        h.desc_size != sizeof(mp_scene_desc))
        return "snapshot written by an incompatible build (struct sizes differ)";
    if (h.nscenes > (1u << 24) || h.particles >= (1u << 31)) return "snapshot counts out of range";
    if (bytes < snapshot_bytes(h.nscenes, h.particles)) return "snapshot truncated";
    return nullptr;
}

}  // namespace mpb
