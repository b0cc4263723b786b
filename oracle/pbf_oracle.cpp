// pbf_oracle.cpp — CPU oracle of the PBF simulation step.
//
// TEST INFRASTRUCTURE ONLY: loaded by the tests, the smoke check and the
// benchmark's CPU-baseline leg as the checker; never by the product path.
//
// FP64 restatement of the reference step, written from
//   engine/shaders/Constraints.metal (predict :54-66, poly6/spikyGrad :29-39,
//     densityLambdaSorted :82-131, applyDeltaSorted :140-199,
//     scatterPositionsToOriginal :205-213, sphereCollision :262-277,
//     computeFoam :287-299, finalizeStep :305-353),
//   engine/shaders/Spatial.metal (cellCoordOf/cellHashOf :35-43, hashCells
//     :49-57, countCells :63-70, scan :82-161, scatterParticles :169-180,
//     gatherPositions :190-198, countNeighbors :207-243),
//   engine/src/Engine.cpp (grid :398-452, seeding :454-549, parameters
//     :551-572, hash dispatch order :601-679, step :685-811).
// Integer outputs use FP32 with the CUDA path's exact rounding so they can be
// compared bit for bit; the solver arithmetic is FP64.

#include "pbf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Saturating float -> int conversion of an already floored value, the
// semantics of the GPU's cvt.rmi.s32.f32 (NaN -> 0).
inline int floor_to_int_sat(float q) {
    if (std::isnan(q)) return 0;
    const float f = std::floor(q);
    if (f >= 2147483648.0f) return 2147483647;
    if (f < -2147483648.0f) return (-2147483647 - 1);
    return int(f);
}
inline int floor_to_int_sat(double q) {
    if (std::isnan(q)) return 0;
    const double f = std::floor(q);
    if (f >= 2147483648.0) return 2147483647;
    if (f < -2147483648.0) return (-2147483647 - 1);
    return int(f);
}
inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// cellCoordOf (Spatial.metal:35-39) in FP32: q = (p - origin) * invCellSize.
inline void cell_coord_f32(const or_grid& g, float px, float py, float pz, int c[3]) {
    const float p[3] = {px, py, pz};
    for (int a = 0; a < 3; ++a) {
        volatile float d = p[a] - g.origin[a];  // one rounding per op, no contraction
        volatile float q = d * g.inv_cell;
        c[a] = clampi(floor_to_int_sat(float(q)), 0, int(g.dims[a]) - 1);
    }
}
// cellHashOf (Spatial.metal:41-43): x + y*gx + z*gx*gy.
inline uint32_t cell_hash(const or_grid& g, int x, int y, int z) {
    return uint32_t(x) + uint32_t(y) * g.dims[0] + uint32_t(z) * g.dims[0] * g.dims[1];
}

// FP32 squared distance in the product's order: fma(dz,dz, fma(dy,dy, dx*dx)).
inline float r2_f32(float dx, float dy, float dz) {
    return std::fmaf(dz, dz, std::fmaf(dy, dy, dx * dx));
}

struct Consts {
    double h, h2, poly6, spiky, inv_rho0, eps, damping;
    double g[3], bmin[3], bmax[3];
    double scorr_k, inv_wq, max_step;
    uint32_t scorr_n, iters;
    double wall_eps, floor_fric, wall_fric, foam_maxn, foam_lo, foam_hi;
    double dt, inv_dt, vmax;
    double sph_gravity, sph_drag, sph_rest;
    // FP64 copy of the grid for the solver's stencil (current iterate)
    double origin[3], inv_cell;
    int dims[3];
};

inline double poly6(double r2, const Consts& c) {
    if (r2 >= c.h2) return 0.0;
    const double d = c.h2 - r2;
    return c.poly6 * d * d * d;
}
inline V3 spiky_grad(V3 r, double rl, const Consts& c) {
    if (rl <= double(1e-6f) || rl >= c.h) return {0, 0, 0};
    const double d = c.h - rl;
    return (-c.spiky * d * d / rl) * r;
}

Consts make_consts(const mp_pbf_params* p, const or_grid& g, double dt) {
    Consts c{};
    c.h = p->h;
    c.h2 = c.h * c.h;
    c.poly6 = 315.0 / (64.0 * kPi * std::pow(c.h, 9));
    c.spiky = 45.0 / (kPi * std::pow(c.h, 6));
    c.inv_rho0 = 1.0 / double(p->rest_density);
    c.eps = p->epsilon;
    c.damping = p->damping;
    for (int a = 0; a < 3; ++a) {
        c.g[a] = p->gravity[a];
        c.bmin[a] = p->bounds_min[a];
        c.bmax[a] = p->bounds_max[a];
        c.origin[a] = g.origin[a];
        c.dims[a] = int(g.dims[a]);
    }
    c.inv_cell = g.inv_cell;
    c.scorr_k = p->scorr_k;
    c.scorr_n = p->scorr_n;
    const double dq = double(p->scorr_dq) * c.h;
    const double wq = poly6(dq * dq, c);
    c.inv_wq = wq > 0 ? 1.0 / wq : 0.0;
    c.max_step = double(p->max_delta) * c.h;
    c.iters = p->solver_iterations;
    c.wall_eps = p->wall_eps;
    c.floor_fric = p->floor_friction;
    c.wall_fric = p->wall_friction;
    c.foam_maxn = p->foam_max_neighbors;
    c.foam_lo = p->foam_speed_lo;
    c.foam_hi = p->foam_speed_hi;
    c.dt = dt;
    c.inv_dt = 1.0 / dt;
    c.vmax = double(p->vmax) * c.h * c.inv_dt;
    c.sph_gravity = p->sphere_gravity;
    c.sph_drag = p->sphere_drag;
    c.sph_rest = p->sphere_restitution;
    return c;
}

// Stencil cell of the current iterate: the reference derives it from its
// FP32 position with cellCoordOf (Constraints.metal:94, 152), so the FP64
// iterate is rounded to FP32 and put through the same FP32 formula.  (A plain
// FP64 floor would disagree with the reference exactly at cell faces, where
// the stencil, and so the result, is discontinuous.)
inline void cell_coord_iter(const or_grid& g, V3 p, int out[3]) {
    cell_coord_f32(g, float(p.x), float(p.y), float(p.z), out);
}

// Visit the 27-cell stencil around `cc` as 9 contiguous slot ranges, in the
// reference's z, y, x order (Constraints.metal:104-110).
template <class F>
inline void for_stencil(const or_grid& g, const int cc[3], const uint32_t* cell_start, F&& f) {
    const int zLo = std::max(cc[2] - 1, 0), zHi = std::min(cc[2] + 1, int(g.dims[2]) - 1);
    const int yLo = std::max(cc[1] - 1, 0), yHi = std::min(cc[1] + 1, int(g.dims[1]) - 1);
    const int xLo = std::max(cc[0] - 1, 0), xHi = std::min(cc[0] + 1, int(g.dims[0]) - 1);
    for (int z = zLo; z <= zHi; ++z)
        for (int y = yLo; y <= yHi; ++y) {
            const uint32_t s = cell_start[cell_hash(g, xLo, y, z)];
            const uint32_t e = cell_start[cell_hash(g, xHi, y, z) + 1];
            for (uint32_t k = s; k < e; ++k) f(k);
        }
}

double smoothstep(double e0, double e1, double x) {
    double t = (x - e0) / (e1 - e0);
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    return t * t * (3.0 - 2.0 * t);
}

void sphere_advance(const Consts& c, double dt, double* s) {
    // Engine.cpp:694-707, in FP64.
    s[4] += c.sph_gravity * dt;
    s[3] *= c.sph_drag;
    s[4] *= c.sph_drag;
    s[5] *= c.sph_drag;
    s[0] += s[3] * dt;
    s[1] += s[4] * dt;
    s[2] += s[5] * dt;
    const double r = s[6];
    for (int a = 0; a < 3; ++a) {
        if (s[a] - r < c.bmin[a]) { s[a] = c.bmin[a] + r; s[3 + a] = -s[3 + a] * c.sph_rest; }
        if (s[a] + r > c.bmax[a]) { s[a] = c.bmax[a] - r; s[3 + a] = -s[3 + a] * c.sph_rest; }
    }
}

// A deliberate mistake the tests plant here, on the CPU, to show that the
// parity checks catch it (or_plant_fault); 0 = none.
int g_planted_fault = 0;

// Metal's clamp(x, lo, hi) = fmin(fmax(x, lo), hi): a NaN coordinate goes to
// the lower bound.
inline double clampd(double x, double lo, double hi) { return std::fmin(std::fmax(x, lo), hi); }

// The shared FP64 step.  `pos`/`vel` are the state at the start of the step
// (FP64, original order), `pred32` the FP32 predicted positions the hash is
// built on.  solve_from_pred32: the solver starts from those FP32 predicted
// positions (the reference's own predict arithmetic, bit-exact with the
// product) instead of the FP64 prediction.  Writes every non-NULL output.
int step_core(const mp_pbf_params* p, double dt, uint32_t n, const V3* pos, const V3* vel,
              const float* pred32, bool solve_from_pred32, double* sphere, V3* pos_out,
              V3* vel_out, or_step_out* out) {
    or_grid g;
    if (or_make_grid(p, &g) != 0) return MP_ERR_INVALID_ARGUMENT;
    const Consts c = make_consts(p, g, dt);

    double sph[7] = {0, 0, 0, 0, 0, 0, 0};
    if (sphere) {
        sphere_advance(c, dt, sphere);
        std::memcpy(sph, sphere, sizeof(sph));
    }

    // 1. predict (FP64 solver copy).  prev = pos.
    std::vector<V3> pred(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) {
        if (solve_from_pred32) {
            pred[i] = {pred32[4 * i], pred32[4 * i + 1], pred32[4 * i + 2]};
        } else {
            const V3 vn = {vel[i].x + c.g[0] * dt, vel[i].y + c.g[1] * dt, vel[i].z + c.g[2] * dt};
            pred[i] = pos[i] + dt * vn;
        }
    }

    // 2. spatial hash on the FP32 predicted positions.
    std::vector<uint32_t> hashes(n), cell_start(size_t(g.cells) + 1), sorted(n), ncount(n);
    or_hash_f32(pred32, n, &g, hashes.data());
    or_counting_sort(hashes.data(), n, g.cells, cell_start.data(), sorted.data());
    const float h2f = p->h * p->h;
    or_count_neighbors_f32(pred32, n, &g, h2f, cell_start.data(), sorted.data(), ncount.data());

    // gather: sorted FP64 positions
    std::vector<V3> cur(n), nxt(n);
    std::vector<double> lam(n, 0.0);
    for (uint32_t s = 0; s < n; ++s) cur[s] = pred[sorted[s]];

    const double rr = sph[6] * sph[6];
    for (uint32_t it = 0; it < c.iters; ++it) {
        // 3a. densityLambdaSorted
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t s = 0; s < int64_t(n); ++s) {
            const V3 pi = cur[s];
            int cc[3];
            cell_coord_iter(g, pi, cc);
            // planted fault 1: the self term W(0) only when the particle's own
            // slot lies in the stencil of its current cell
            const bool self_in_stencil_only = g_planted_fault == 1;
            double dens = self_in_stencil_only ? 0.0 : poly6(0.0, c), gsq = 0.0;
            V3 gs = {0, 0, 0};
            for_stencil(g, cc, cell_start.data(), [&](uint32_t k) {
                if (k == uint32_t(s)) {
                    if (self_in_stencil_only) dens += poly6(0.0, c);
                    return;
                }
                const V3 r = pi - cur[k];
                const double r2 = dot(r, r);
                if (r2 >= c.h2) return;
                dens += poly6(r2, c);
                const V3 gr = spiky_grad(r, std::sqrt(r2), c);
                gs = gs + gr;
                gsq += dot(gr, gr);
            });
            const double C = dens * c.inv_rho0 - 1.0;
            const double denom = c.inv_rho0 * c.inv_rho0 * (dot(gs, gs) + gsq) + c.eps;
            lam[s] = -C / denom;
        }
        // 3b. applyDeltaSorted (+ 3c sphereCollision on the result)
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t s = 0; s < int64_t(n); ++s) {
            const V3 pi = cur[s];
            const double li = lam[s];
            int cc[3];
            cell_coord_iter(g, pi, cc);
            V3 d = {0, 0, 0};
            for_stencil(g, cc, cell_start.data(), [&](uint32_t k) {
                if (k == uint32_t(s)) return;
                const V3 r = pi - cur[k];
                const double r2 = dot(r, r);
                if (r2 >= c.h2) return;
                const V3 gr = spiky_grad(r, std::sqrt(r2), c);
                const double ratio = poly6(r2, c) * c.inv_wq;
                double rn = 1.0;
                for (uint32_t e = 0; e < c.scorr_n; ++e) rn *= ratio;
                const double scorr = -c.scorr_k * rn;
                d = d + (li + lam[k] + scorr) * gr;
            });
            d = c.inv_rho0 * d;
            const double dl = std::sqrt(dot(d, d));
            if (dl > c.max_step) d = (c.max_step / dl) * d;
            V3 np = pi + d;
            np.x = clampd(np.x, c.bmin[0], c.bmax[0]);
            np.y = clampd(np.y, c.bmin[1], c.bmax[1]);
            np.z = clampd(np.z, c.bmin[2], c.bmax[2]);
            if (sphere) {
                const V3 ctr = {sph[0], sph[1], sph[2]};
                const V3 dd = np - ctr;
                const double r2 = dot(dd, dd);
                if (r2 < rr) {
                    const double r = std::sqrt(std::fmax(r2, double(1e-8f)));
                    np = ctr + (sph[6] / r) * dd;
                }
            }
            nxt[s] = np;
        }
        std::swap(cur, nxt);
    }

    // 4-6. scatter back, finalize, foam (original order)
    std::vector<V3> pfin(n), vfin(n);
    std::vector<double> foam(n), lam_orig(n);
    for (uint32_t s = 0; s < n; ++s) {
        pfin[sorted[s]] = cur[s];
        lam_orig[sorted[s]] = lam[s];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) {
        V3 q = pfin[i];
        q.x = clampd(q.x, c.bmin[0], c.bmax[0]);
        q.y = clampd(q.y, c.bmin[1], c.bmax[1]);
        q.z = clampd(q.z, c.bmin[2], c.bmax[2]);
        V3 v = {(q.x - pos[i].x) * c.inv_dt * c.damping, (q.y - pos[i].y) * c.inv_dt * c.damping,
                (q.z - pos[i].z) * c.inv_dt * c.damping};
        const bool xMin = q.x <= c.bmin[0] + c.wall_eps;
        const bool xMax = q.x >= c.bmax[0] - c.wall_eps;
        const bool yMin = q.y <= c.bmin[1] + c.wall_eps;
        const bool yMax = q.y >= c.bmax[1] - c.wall_eps;
        const bool zMin = q.z <= c.bmin[2] + c.wall_eps;
        const bool zMax = q.z >= c.bmax[2] - c.wall_eps;
        if (xMin) v.x = std::fmax(v.x, 0.0);
        if (xMax) v.x = std::fmin(v.x, 0.0);
        if (yMin) v.y = std::fmax(v.y, 0.0);
        if (yMax) v.y = std::fmin(v.y, 0.0);
        if (zMin) v.z = std::fmax(v.z, 0.0);
        if (zMax) v.z = std::fmin(v.z, 0.0);
        if (yMin) {
            v.x *= c.floor_fric;
            v.z *= c.floor_fric;
        } else if (xMin || xMax || zMin || zMax) {
            v = c.wall_fric * v;
        }
        const double vl = std::sqrt(dot(v, v));
        if (vl > c.vmax) v = (c.vmax / vl) * v;
        pfin[i] = q;
        vfin[i] = v;
        const double surface =
            1.0 - clampd(double(ncount[i]) / c.foam_maxn, 0.0, 1.0);
        foam[i] = surface * smoothstep(c.foam_lo, c.foam_hi, std::sqrt(dot(v, v)));
    }

    if (pos_out) std::memcpy(pos_out, pfin.data(), sizeof(V3) * n);
    if (vel_out) std::memcpy(vel_out, vfin.data(), sizeof(V3) * n);
    if (out) {
        if (out->pos3) std::memcpy(out->pos3, pfin.data(), sizeof(V3) * n);
        if (out->vel3) std::memcpy(out->vel3, vfin.data(), sizeof(V3) * n);
        if (out->lambda) std::memcpy(out->lambda, lam_orig.data(), sizeof(double) * n);
        if (out->foam) std::memcpy(out->foam, foam.data(), sizeof(double) * n);
        if (out->neighbor_counts) std::memcpy(out->neighbor_counts, ncount.data(), 4 * size_t(n));
        if (out->hashes) std::memcpy(out->hashes, hashes.data(), 4 * size_t(n));
        if (out->cell_start)
            std::memcpy(out->cell_start, cell_start.data(), 4 * (size_t(g.cells) + 1));
        if (out->sorted_index) std::memcpy(out->sorted_index, sorted.data(), 4 * size_t(n));
        if (out->pred4) std::memcpy(out->pred4, pred32, 16 * size_t(n));
    }
    return 0;
}

}  // namespace

extern "C" {

int or_make_grid(const mp_pbf_params* p, or_grid* g) {
    if (!p || !g || !(p->cell_size > 0.0f)) return MP_ERR_INVALID_ARGUMENT;
    uint64_t cells = 1;
    for (int a = 0; a < 3; ++a) {
        const float ext = p->bounds_max[a] - p->bounds_min[a];
        const float d = std::ceil(ext / p->cell_size);
        if (!(d >= 1.0f) || d > 65536.0f) return MP_ERR_INVALID_ARGUMENT;
        g->dims[a] = uint32_t(d);
        g->origin[a] = p->bounds_min[a];
        cells *= g->dims[a];
    }
    if (cells >= (1ull << 31)) return MP_ERR_INVALID_ARGUMENT;
    g->cell = p->cell_size;
    g->inv_cell = 1.0f / p->cell_size;
    g->cells = uint32_t(cells);
    return 0;
}

void or_hash_f32(const float* pos4, uint32_t n, const or_grid* g, uint32_t* hashes) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) {
        int c[3];
        cell_coord_f32(*g, pos4[4 * i + 0], pos4[4 * i + 1], pos4[4 * i + 2], c);
        hashes[i] = cell_hash(*g, c[0], c[1], c[2]);
    }
}

void or_exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n) {
    uint32_t run = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t v = in[i];
        out[i] = run;
        run += v;
    }
}

void or_counting_sort(const uint32_t* hashes, uint32_t n, uint32_t cells, uint32_t* cell_start,
                      uint32_t* sorted_index) {
    std::vector<uint32_t> counts(size_t(cells) + 1, 0), cursor(size_t(cells) + 1, 0);
    for (uint32_t i = 0; i < n; ++i) counts[hashes[i]]++;
    or_exclusive_scan_u32(counts.data(), cell_start, cells + 1);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t c = hashes[i];
        sorted_index[cell_start[c] + cursor[c]++] = i;  // ascending i within a cell
    }
}

void or_count_neighbors_f32(const float* pos4, uint32_t n, const or_grid* g, float r2max,
                            const uint32_t* cell_start, const uint32_t* sorted_index,
                            uint32_t* counts) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < int64_t(n); ++i) {
        const float px = pos4[4 * i], py = pos4[4 * i + 1], pz = pos4[4 * i + 2];
        int cc[3];
        cell_coord_f32(*g, px, py, pz, cc);
        uint32_t cnt = 0;
        for_stencil(*g, cc, cell_start, [&](uint32_t k) {
            const uint32_t j = sorted_index[k];
            if (j == uint32_t(i)) return;
            const float dx = pos4[4 * j] - px, dy = pos4[4 * j + 1] - py, dz = pos4[4 * j + 2] - pz;
            if (r2_f32(dx, dy, dz) < r2max) ++cnt;
        });
        counts[i] = cnt;
    }
}

void or_predict_f32(const float* pos4, const float* vel4, uint32_t n, const float g[3], float dt,
                    float* pred4) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) {
        for (int a = 0; a < 3; ++a) {
            const float vn = std::fmaf(g[a], dt, vel4[4 * i + a]);
            pred4[4 * i + a] = std::fmaf(vn, dt, pos4[4 * i + a]);
        }
        pred4[4 * i + 3] = pos4[4 * i + 3];
    }
}

int or_seed_scene(const mp_pbf_params* p, uint32_t scene, const mp_scene_desc* d, uint32_t n,
                  float* pos4) {
    if (!p || (!pos4 && n)) return MP_ERR_INVALID_ARGUMENT;
    std::memset(pos4, 0, 16 * size_t(n));
    const float spacing_ref = p->h * 0.5f;  // Engine.cpp:457
    uint32_t i = 0;
    if (d && d->lattice) {
        const double sp = d->spacing > 0.0f ? double(d->spacing) : double(spacing_ref);
        const uint64_t cap = uint64_t(d->dims[0]) * d->dims[1] * d->dims[2];
        if (cap < n) return MP_ERR_INVALID_ARGUMENT;
        std::mt19937_64 rng(d->seed);
        auto jit = [&]() {
            const double u = double(rng() >> 11) * 0x1.0p-53;
            return (2.0 * u - 1.0) * double(d->jitter);
        };
        for (uint32_t y = 0; y < d->dims[1] && i < n; ++y)
            for (uint32_t z = 0; z < d->dims[2] && i < n; ++z)
                for (uint32_t x = 0; x < d->dims[0] && i < n; ++x, ++i) {
                    const double jx = jit(), jy = jit(), jz = jit();
                    pos4[4 * i + 0] = float(double(d->origin[0]) + double(x) * sp + jx);
                    pos4[4 * i + 1] = float(double(d->origin[1]) + double(y) * sp + jy);
                    pos4[4 * i + 2] = float(double(d->origin[2]) + double(z) * sp + jz);
                    pos4[4 * i + 3] = 1.0f;
                }
        return 0;
    }
    const float spacing = spacing_ref;
    const float* bmin = p->bounds_min;
    const float* bmax = p->bounds_max;
    const float cx = 0.5f * (bmin[0] + bmax[0]);
    const float cz = 0.5f * (bmin[2] + bmax[2]);
    if (scene == MP_SCENE_DAM_BREAK) {  // Engine.cpp:463-491
        const float kMaxHeightM = 5.5f;
        const uint32_t nLayers = uint32_t(kMaxHeightM / spacing);
        if (nLayers == 0) return MP_ERR_INVALID_ARGUMENT;
        const uint32_t perLayer = (n + nLayers - 1) / nLayers;
        const uint32_t side = uint32_t(std::ceil(std::sqrt(double(perLayer))));
        const float baseExtent = float(side - 1) * spacing;
        const float xMin = bmin[0] + 0.05f;
        const float yMin = bmin[1] + 0.05f;
        const float zStart = cz - baseExtent * 0.5f;
        for (uint32_t y = 0; y < nLayers && i < n; ++y)
            for (uint32_t z = 0; z < side && i < n; ++z)
                for (uint32_t x = 0; x < side && i < n; ++x, ++i) {
                    pos4[4 * i + 0] = xMin + float(x) * spacing;
                    pos4[4 * i + 1] = yMin + float(y) * spacing;
                    pos4[4 * i + 2] = zStart + float(z) * spacing;
                    pos4[4 * i + 3] = 1.0f;
                }
        return 0;
    }
    if (scene == MP_SCENE_SPHERE_DROP) {  // Engine.cpp:494-527
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
                    pos4[4 * i + 0] = xMin + float(x) * spacing;
                    pos4[4 * i + 1] = yPos;
                    pos4[4 * i + 2] = zMin + float(z) * spacing;
                    pos4[4 * i + 3] = 1.0f;
                }
            if (nx == 0 || nz == 0) break;
        }
        return 0;
    }
    if (scene != MP_SCENE_CUBE_DROP) return MP_ERR_INVALID_ARGUMENT;
    // Cube drop: Engine.cpp:530-548.
    const uint32_t side = uint32_t(std::ceil(std::cbrt(double(n))));
    const float halfBlk = 0.5f * float(side - 1) * spacing;
    const float topY = 2.0f;
    for (uint32_t y = 0; y < side && i < n; ++y)
        for (uint32_t z = 0; z < side && i < n; ++z)
            for (uint32_t x = 0; x < side && i < n; ++x, ++i) {
                pos4[4 * i + 0] = cx - halfBlk + float(x) * spacing;
                pos4[4 * i + 1] = topY - float(y) * spacing;
                pos4[4 * i + 2] = cz - halfBlk + float(z) * spacing;
                pos4[4 * i + 3] = 1.0f;
            }
    return 0;
}

// Legacy integrator: kernel integrate (engine/shaders/Integrate.metal:11-42)
// as Engine::integrate dispatches it (Engine.cpp:578-596), in FP32 with one
// rounding per operation in the shader's order.
void or_integrate_f32(const mp_pbf_params* p, float dt, uint32_t n, float* pos4, float* vel4) {
    const float rest = p->integrate_restitution, damp = p->integrate_damping;
    for (uint32_t i = 0; i < n; ++i) {
        float* q = pos4 + 4 * size_t(i);
        float* v = vel4 + 4 * size_t(i);
        for (int a = 0; a < 3; ++a) {
            volatile float gdt = p->gravity[a] * dt;
            volatile float va = v[a] + gdt;
            v[a] = va * damp;
            volatile float step = v[a] * dt;
            q[a] = q[a] + step;
        }
        for (int a = 0; a < 3; ++a)
            if (q[a] < p->bounds_min[a]) { q[a] = p->bounds_min[a]; v[a] = -v[a] * rest; }
        for (int a = 0; a < 3; ++a)
            if (q[a] > p->bounds_max[a]) { q[a] = p->bounds_max[a]; v[a] = -v[a] * rest; }
        q[3] = 1.0f;
        v[3] = 0.0f;
    }
}

// kernel applyMousePulse (Constraints.metal:231-253) in FP32, dot products
// summed x + y, then + z.
void or_mouse_pulse_f32(const mp_pbf_params* p, const float origin[3], const float dir[3],
                        const float force[3], float radius, uint32_t n, const float* pos4,
                        float* vel4) {
    auto dot = [](const float* a, const float* b) {
        volatile float xy = a[0] * b[0] + a[1] * b[1];
        return xy + a[2] * b[2];
    };
    const float R2 = radius * radius;
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = pos4 + 4 * size_t(i);
        float toP[3];
        for (int a = 0; a < 3; ++a) toP[a] = q[a] - origin[a];
        const float t = dot(toP, dir);
        if (t <= 0.0f) continue;
        float d[3];
        for (int a = 0; a < 3; ++a) {
            volatile float c = origin[a] + dir[a] * t;
            d[a] = q[a] - c;
        }
        const float r2 = dot(d, d);
        if (r2 < R2) {
            volatile float den = R2 * p->mouse_falloff;
            const float intensity = std::exp(-r2 / den);
            float* v = vel4 + 4 * size_t(i);
            for (int a = 0; a < 3; ++a) v[a] = v[a] + force[a] * intensity;
            v[3] = 0.0f;
        }
    }
}

void or_sphere_advance(const mp_pbf_params* p, double dt, double* s) {
    or_grid g;
    if (or_make_grid(p, &g) != 0) return;
    const Consts c = make_consts(p, g, dt);
    sphere_advance(c, dt, s);
}

int or_step(const mp_pbf_params* p, float dt, uint32_t n, const float* pos4, const float* vel4,
            double* sphere, or_step_out* out) {
    if (!p || (n && (!pos4 || !vel4))) return MP_ERR_INVALID_ARGUMENT;
    if (!(dt > 0.0f)) return 0;  // Engine.cpp:686
    std::vector<V3> pos(n), vel(n);
    for (uint32_t i = 0; i < n; ++i) {
        pos[i] = {pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]};
        vel[i] = {vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2]};
    }
    std::vector<float> pred32(4 * size_t(n));
    or_predict_f32(pos4, vel4, n, p->gravity, dt, pred32.data());
    return step_core(p, double(dt), n, pos.data(), vel.data(), pred32.data(), true, sphere,
                     nullptr, nullptr, out);
}

int or_step_f64(const mp_pbf_params* p, double dt, uint32_t n, double* pos3, double* vel3,
                double* sphere) {
    if (!p || (n && (!pos3 || !vel3))) return MP_ERR_INVALID_ARGUMENT;
    if (!(dt > 0.0)) return 0;
    std::vector<float> pred32(4 * size_t(n));
    for (uint32_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            pred32[4 * i + a] =
                float(pos3[3 * i + a] + dt * (vel3[3 * i + a] + double(p->gravity[a]) * dt));
    const V3* pos = reinterpret_cast<const V3*>(pos3);
    const V3* vel = reinterpret_cast<const V3*>(vel3);
    std::vector<V3> po(n), vo(n);
    const int rc =
        step_core(p, dt, n, pos, vel, pred32.data(), false, sphere, po.data(), vo.data(), nullptr);
    if (rc) return rc;
    std::memcpy(pos3, po.data(), sizeof(V3) * n);
    std::memcpy(vel3, vo.data(), sizeof(V3) * n);
    return 0;
}

void or_plant_fault(int which) { g_planted_fault = which; }

void or_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
