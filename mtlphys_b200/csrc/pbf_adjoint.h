// pbf_adjoint.h — the adjoint (reverse-mode derivative) of one recorded PBF
// step of a batch of scenes.  No reference counterpart: the reference engine
// is not differentiable.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_batch.h"

namespace mpb {

// Per-scene gradient accumulators (FP64): d/d s_corr k, the sphere's center
// (3), velocity (3) and radius.  During the reverse sweep the sphere entries
// hold the adjoint of the sphere state at the current step.
constexpr uint32_t kGradStride = 8;
constexpr uint32_t kGradK = 0, kGradCenter = 1, kGradVel = 4, kGradRadius = 7;

// One recorded step, as the forward step kept it (pbf_batch.h BatchRecord
// plus the per-step arrays the record owns).
struct AdjStep {
    const SceneDev* scenes;       // scene table: sub-grids and sphere of the step
    const SphereState* sphere0;   // spheres before the step's kinematic advance
    const float4* x0;             // positions at the start of the step (original order)
    const float4* x1;             // positions at the end of the step (original order)
    const uint32_t* sidx;         // slot -> particle
    const uint32_t* scell;        // slot -> hash cell (sub-grid local id)
    const uint32_t* cstart;       // cell starts of the step's grids
    const float4* lam;            // iterations x stride: (l, lambda)
    const float4* delta;          // iterations x stride: unclamped corrections
    const uint32_t* masks;        // iterations x 9 x mask_stride row masks
    const uint32_t* overflow;     // iterations x mask_stride: bit r set for a long row r
};

// Pair terms that a particle's sweep owes another particle whose own sweep
// does not see the pair (one-way pairs) are posted to the receiver's inbox:
// kInbox slots per receiver, then a shared pool of overflow entries linked
// into a list per receiver.  A delivery kernel then adds each receiver's
// posts in ascending order of the sender's slot, so the sums do not depend
// on the order the posts arrived in (no float atomics: two backward passes
// give the same bytes).
constexpr uint32_t kInbox = 4;
constexpr uint32_t kInboxOverflow = 1u << 18;  // pooled entries beyond kInbox, all receivers together
constexpr uint32_t kNoPost = 0xffffffffu;      // end of a receiver's overflow list
// The per-scene sums of the sphere gradient run over chunks of this many slots.
constexpr uint32_t kSumChunk = 2048;

struct AdjArgs {
    AdjStep t;
    const uint32_t* scene_of;     // scene of every particle / slot
    uint32_t n, nscenes, iterations, stride, mask_stride;
    float4* xbar;                 // in: dL/dx(t+1), out: dL/dx(t) (original order)
    float4* vbar;                 // in: dL/dv(t+1), out: dL/dv(t)
    // per-slot scratch (sorted order)
    float4 *pbar, *qbar, *dbar, *lbar, *gd, *p_extra;
    float *qsc, *lam_part, *lam_extra;
    uint32_t *ccur, *cpred;
    // one-way pair posts: per receiver slot a count and kInbox (sender,
    // value) entries (entry e of receiver j at e * stride + j); further posts
    // take pooled entries (sender, value, next) linked from ovf_head[j]
    uint32_t *inbox_count, *inbox_src;
    float4* inbox_val;
    uint32_t *ovf_head, *ovf_count, *ovf_src, *ovf_next;
    float4* ovf_val;
    // per-slot FP64 accumulators of the scene gradients, reduced per scene in
    // a fixed order: dL/dk (over the whole backward pass) and the sphere's
    // center (xyz) and radius (w) (over one step, summed per chunk of
    // kSumChunk slots into spart[scene * sum_chunks + chunk])
    double* kacc;
    double4 *sacc, *spart;
    uint32_t sum_chunks;
    uint32_t* err;                // device error word (kDevErrIndex: a post was dropped)
    double* grads;                // nscenes x kGradStride
};

// Enqueue the reverse of one step: finalize, every solver iteration in
// reverse order, predict, and the sphere kinematics.  p_extra, lam_extra,
// inbox_count and sacc must be zero and ovf_head kNoPost on entry (they are
// left so); kacc accumulates.
cudaError_t launch_adjoint_step(const AdjArgs& a, cudaStream_t s);
// grads[scene][kGradK] = the sum of kacc over the scene's slots (fixed order);
// kacc is cleared.
cudaError_t launch_adjoint_finish(const AdjArgs& a, cudaStream_t s);

// Kernel launches per reversed step.
uint32_t adjoint_launch_count(uint32_t iterations);

}  // namespace mpb
