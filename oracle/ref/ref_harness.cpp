// ref_harness.cpp — host-side dispatch order of the reference Engine
// (engine/src/Engine.cpp:551-572 parameters, :601-679 buildSpatialHash,
// :685-811 step), driving the reference's shader code compiled as C++.
//
// TEST INFRASTRUCTURE ONLY.
#include "ref_harness.h"

#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
int g_threads = 1;
constexpr float kPi = 3.14159265358979323846f;

struct Grid {
    uint32_t dims[3];
    uint32_t cells;
};

Grid make_grid(const ref_config* c) {
    Grid g{};
    g.cells = ref_grid(c, g.dims);
    return g;
}

std::vector<unsigned char> spatial_params(const ref_config* c, const Grid& g, uint32_t n) {
    std::vector<unsigned char> sp(ref_sizeof_spatial_params());
    ref_fill_spatial_params(sp.data(), c->bounds_min, c->cell, 1.0f / c->cell, c->h * c->h, n,
                            g.cells, g.dims, c->max_neighbors);
    return sp;
}

// Engine::writePBFParams (Engine.cpp:551-572) with the gravity, density,
// epsilon and damping taken from the config instead of the constexprs.
std::vector<unsigned char> pbf_params(const ref_config* c, float dt, uint32_t n) {
    const float h = c->h;
    const float h2 = h * h;
    const float h3 = h2 * h;
    const float h6 = h3 * h3;
    const float h9 = h6 * h3;
    std::vector<unsigned char> pp(ref_sizeof_pbf_params());
    ref_fill_pbf_params(pp.data(), c->gravity, dt, c->bounds_min, c->bounds_max, h, h2,
                        315.0f / (64.0f * kPi * h9), 45.0f / (kPi * h6), c->rest_density,
                        c->epsilon, c->damping, n);
    return pp;
}

void hash_pass(const ref_config* c, const Grid& g, const void* sp, uint32_t n, const float* pos4,
               uint32_t* hashes, uint32_t* cell_start, uint32_t* sorted_index, float* sorted4,
               uint32_t* ncount) {
    std::vector<uint32_t> counts(size_t(g.cells) + 1, 0), cursor(g.cells, 0);
    ref_k_hash_cells(pos4, hashes, sp, n);
    ref_k_count_cells(hashes, counts.data(), sp, n);
    // runExclusiveScan over cells+1 entries: the reference's CPU form
    // (tests/TestUtils.hpp:52-61).
    uint32_t run = 0;
    for (size_t i = 0; i <= g.cells; ++i) {
        const uint32_t v = counts[i];
        cell_start[i] = run;
        run += v;
    }
    ref_k_scatter_particles(hashes, cell_start, cursor.data(), sorted_index, sp, n);
    ref_k_gather_positions(pos4, sorted_index, sorted4, sp, n);
    ref_k_count_neighbors(pos4, cell_start, sorted_index, ncount, sp, sorted4, n);
    (void)c;
}
}  // namespace

extern "C" {

void ref_set_threads(int n) {
    g_threads = n < 1 ? 1 : n;
#ifdef _OPENMP
    omp_set_num_threads(g_threads);
#endif
}
int ref_parallel(void) { return g_threads > 1; }
int ref_threads(void) { return g_threads; }

uint32_t ref_grid(const ref_config* c, uint32_t dims[3]) {
    // buildSpatialBuffers (Engine.cpp:399-403).
    for (int a = 0; a < 3; ++a) {
        const float extent = c->bounds_max[a] - c->bounds_min[a];
        dims[a] = uint32_t(std::ceil(extent / c->cell));
    }
    return dims[0] * dims[1] * dims[2];
}

void ref_build_spatial_hash(const ref_config* c, uint32_t n, const float* pos4, uint32_t* hashes,
                            uint32_t* cell_start, uint32_t* sorted_index, float* sorted4,
                            uint32_t* ncount) {
    const Grid g = make_grid(c);
    const auto sp = spatial_params(c, g, n);
    hash_pass(c, g, sp.data(), n, pos4, hashes, cell_start, sorted_index, sorted4, ncount);
}

void ref_step(ref_config* c, float dt, uint32_t n, float* pos4, float* vel4, float* prev4_out,
              float* lambdas_out, uint32_t* ncount_out, float* foam_out, uint32_t* hashes_out,
              uint32_t* cell_start_out, uint32_t* sorted_index_out) {
    if (dt <= 0) return;  // Engine.cpp:686
    const Grid g = make_grid(c);
    const auto sp = spatial_params(c, g, n);
    const auto pp = pbf_params(c, dt, n);

    if (c->sphere) {  // Engine.cpp:693-712 (host-side sphere kinematics)
        float* ctr = c->sphere_center;
        float* vel = c->sphere_velocity;
        vel[1] += -9.81f * dt;
        vel[0] *= 0.998f;
        vel[1] *= 0.998f;
        vel[2] *= 0.998f;
        ctr[0] += vel[0] * dt;
        ctr[1] += vel[1] * dt;
        ctr[2] += vel[2] * dt;
        const float r = c->sphere_radius;
        for (int a = 0; a < 3; ++a) {
            if (ctr[a] - r < c->bounds_min[a]) { ctr[a] = c->bounds_min[a] + r; vel[a] = -vel[a] * 0.4f; }
            if (ctr[a] + r > c->bounds_max[a]) { ctr[a] = c->bounds_max[a] - r; vel[a] = -vel[a] * 0.4f; }
        }
    }

    std::vector<float> prev(4 * size_t(n)), sortedA(4 * size_t(n)), sortedB(4 * size_t(n));
    std::vector<float> sorted_lambda(n), lambdas(n), foam(n);
    std::vector<uint32_t> hashes(n), cell_start(size_t(g.cells) + 1), sorted_index(n), ncount(n);

    ref_k_predict(pos4, vel4, prev.data(), pp.data(), n);
    hash_pass(c, g, sp.data(), n, pos4, hashes.data(), cell_start.data(), sorted_index.data(),
              sortedA.data(), ncount.data());

    float* cur = sortedA.data();
    float* nxt = sortedB.data();
    for (uint32_t it = 0; it < c->iterations; ++it) {
        ref_k_density_lambda(cur, cell_start.data(), sorted_index.data(), sorted_lambda.data(),
                             lambdas.data(), sp.data(), pp.data(), n);
        ref_k_apply_delta(cur, cell_start.data(), sorted_lambda.data(), nxt, sp.data(), pp.data(), n);
        if (c->sphere) ref_k_sphere_collision(nxt, sp.data(), c->sphere_center, c->sphere_radius, n);
        std::swap(cur, nxt);
    }
    ref_k_scatter_to_original(cur, sorted_index.data(), pos4, sp.data(), n);
    ref_k_finalize(pos4, vel4, prev.data(), pp.data(), n);
    ref_k_compute_foam(vel4, ncount.data(), foam.data(), n, float(c->max_neighbors), n);

    if (prev4_out) std::memcpy(prev4_out, prev.data(), 16 * size_t(n));
    if (lambdas_out) std::memcpy(lambdas_out, lambdas.data(), 4 * size_t(n));
    if (ncount_out) std::memcpy(ncount_out, ncount.data(), 4 * size_t(n));
    if (foam_out) std::memcpy(foam_out, foam.data(), 4 * size_t(n));
    if (hashes_out) std::memcpy(hashes_out, hashes.data(), 4 * size_t(n));
    if (cell_start_out) std::memcpy(cell_start_out, cell_start.data(), 4 * (size_t(g.cells) + 1));
    if (sorted_index_out) std::memcpy(sorted_index_out, sorted_index.data(), 4 * size_t(n));
}

}  // extern "C"
