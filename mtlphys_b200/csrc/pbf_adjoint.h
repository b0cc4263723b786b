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
    double* grads;                // nscenes x kGradStride
};

// Enqueue the reverse of one step: finalize, every solver iteration in
// reverse order, predict, and the sphere kinematics.  p_extra and lam_extra
// must be zero on entry (they are left zero).
cudaError_t launch_adjoint_step(const AdjArgs& a, cudaStream_t s);

// Kernel launches per reversed step.
uint32_t adjoint_launch_count(uint32_t iterations);

}  // namespace mpb
