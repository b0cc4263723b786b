/*
 * c_consumer.c — a plain C program that uses the engine the way the
 * reference's C++ callers use mtlphys::Engine (tests/test_pbf.cpp:36-65,
 * app/bridge/EngineBridge.mm:12-72): include the header, link the library,
 * create -> reset -> step -> download, with no CUDA headers (the stream is a
 * void*).  The tests compile it with gcc against include/mtlphys_b200.h and
 * mtlphys_b200/libmtlphys_b200.so.
 *
 *   c_consumer abi   host-only calls (no GPU needed): version, defaults
 *   c_consumer run   the GPU checks below; prints "ok" lines, exits non-zero
 *                    on the first failure
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mtlphys_b200.h"

#define CHECK(call)                                                                  \
    do {                                                                             \
        int rc_ = (call);                                                            \
        if (rc_ != MP_OK) {                                                          \
            fprintf(stderr, "%s -> %d: %s\n", #call, rc_, mp_last_error());          \
            return 1;                                                                \
        }                                                                            \
    } while (0)

#define EXPECT(cond, ...)                                                            \
    do {                                                                             \
        if (!(cond)) {                                                               \
            fprintf(stderr, "expectation failed: %s: ", #cond);                      \
            fprintf(stderr, __VA_ARGS__);                                            \
            fprintf(stderr, "\n");                                                   \
            return 1;                                                                \
        }                                                                            \
    } while (0)

static int abi_checks(void) {
    mp_pbf_params p;
    mp_scene_desc d;
    EXPECT(mp_abi_version() >= 1, "abi version %u", mp_abi_version());
    CHECK(mp_default_params(&p));
    CHECK(mp_default_scene_desc(&d));
    EXPECT(p.size == sizeof(mp_pbf_params), "params size %u", p.size);
    EXPECT(p.solver_iterations == 5 && p.rest_density == 8000.0f && p.epsilon == 800.0f,
           "reference tunables (Engine.cpp:32-39)");
    EXPECT(d.size == sizeof(mp_scene_desc) && d.lattice == 0, "scene desc defaults");
    EXPECT(mp_default_params(NULL) == MP_ERR_INVALID_ARGUMENT, "NULL rejected");
    EXPECT(fabs(mp_lattice_rest_density(0.1, 0.05) - 8078.2013) < 1e-3, "rest density");
    printf("ok abi\n");
    return 0;
}

/* test_pbf.cpp:47-65: one isolated particle falls under gravity for one step. */
static int isolated_particle(mp_engine* e) {
    mp_pbf_params p;
    float pos[4] = {0.0f, 1.0f, 0.0f, 1.0f}, vel[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    CHECK(mp_default_params(&p));
    CHECK(mp_engine_set_params(e, &p));
    CHECK(mp_engine_reset(e, 1));
    CHECK(mp_engine_upload(e, MP_BUF_POSITIONS, pos, 1, NULL));
    CHECK(mp_engine_upload(e, MP_BUF_VELOCITIES, vel, 1, NULL));
    CHECK(mp_engine_step(e, 0.01f, NULL));
    CHECK(mp_engine_download(e, MP_BUF_POSITIONS, pos, 1, NULL));
    CHECK(mp_engine_download(e, MP_BUF_VELOCITIES, vel, 1, NULL));
    CHECK(mp_engine_check_errors(e, NULL));
    EXPECT(fabsf(pos[1] - 0.99902f) < 1e-3f && vel[1] < 0.0f, "y = %g, vy = %g", pos[1], vel[1]);
    printf("ok isolated y=%.6f vy=%.6f\n", pos[1], vel[1]);
    return 0;
}

/* A 1000-particle cube drop (Engine.cpp:531-548), 50 steps at dt = 1/240
 * (test_pbf.cpp:109-130): finite and inside the box; the hash invariants. */
static int cube_drop(mp_engine* e) {
    const uint32_t n = 1000;
    mp_pbf_params p;
    float* pos = (float*)malloc(16 * n);
    uint32_t* cs;
    size_t bytes = 0;
    void* dptr = NULL;
    uint32_t i, cells;
    CHECK(mp_default_params(&p));
    CHECK(mp_engine_set_params(e, &p));
    CHECK(mp_engine_reset_scene(e, n, MP_SCENE_CUBE_DROP, NULL));
    EXPECT(mp_engine_particle_count(e) == n && mp_engine_current_scene(e) == MP_SCENE_CUBE_DROP,
           "count / scene");
    CHECK(mp_engine_set_graph_mode(e, 1));
    for (i = 0; i < 50; ++i) CHECK(mp_engine_step(e, 1.0f / 240.0f, NULL));
    CHECK(mp_engine_check_errors(e, NULL));
    CHECK(mp_engine_download(e, MP_BUF_POSITIONS, pos, n, NULL));
    for (i = 0; i < n; ++i) {
        const float* q = pos + 4 * i;
        EXPECT(isfinite(q[0]) && isfinite(q[1]) && isfinite(q[2]), "particle %u not finite", i);
        EXPECT(q[0] >= -3.0f && q[0] <= 3.0f && q[1] >= -3.0f && q[1] <= 6.0f && q[2] >= -3.0f &&
                   q[2] <= 3.0f,
               "particle %u outside the box", i);
    }
    CHECK(mp_engine_build_spatial_hash(e, NULL));
    CHECK(mp_engine_buffer(e, MP_BUF_CELL_START, &dptr, &bytes));
    cells = mp_engine_total_cells(e);
    EXPECT(bytes == 4 * ((size_t)cells + 1), "cellStart holds cells + 1 entries");
    cs = (uint32_t*)malloc(bytes);
    CHECK(mp_engine_download(e, MP_BUF_CELL_START, cs, cells + 1, NULL));
    EXPECT(cs[0] == 0 && cs[cells] == n, "cellStart[0] = %u, cellStart[C] = %u", cs[0], cs[cells]);
    for (i = 0; i < cells; ++i) EXPECT(cs[i] <= cs[i + 1], "cellStart not monotonic at %u", i);
    free(cs);
    free(pos);
    printf("ok cube_drop %u particles, %u cells\n", n, cells);
    return 0;
}

/* runExclusiveScan (Engine.cpp:843-882) on device memory the engine owns:
 * the neighbour counts as input, the lambdas buffer as output and the
 * sorted positions as scratch (all borrowed device pointers). */
static int scan(mp_engine* e) {
    const uint32_t n = mp_engine_particle_count(e);
    void *in = NULL, *out = NULL, *scratch = NULL;
    size_t bytes = 0, sbytes = mp_exclusive_scan_scratch_bytes(n);
    uint32_t *h_in = (uint32_t*)malloc(4 * n), *h_out = (uint32_t*)malloc(4 * n), run = 0, i;
    CHECK(mp_engine_buffer(e, MP_BUF_NEIGHBOR_COUNTS, &in, &bytes));
    CHECK(mp_engine_buffer(e, MP_BUF_LAMBDAS, &out, &bytes));
    CHECK(mp_engine_buffer(e, MP_BUF_SORTED_POSITIONS, &scratch, &bytes));
    EXPECT(bytes >= sbytes, "scratch too small");
    CHECK(mp_engine_download(e, MP_BUF_NEIGHBOR_COUNTS, h_in, n, NULL));
    CHECK(mp_exclusive_scan((const uint32_t*)in, (uint32_t*)out, n, scratch, sbytes, NULL));
    CHECK(mp_exclusive_scan_status(scratch, NULL));
    CHECK(mp_engine_download(e, MP_BUF_LAMBDAS, h_out, n, NULL));
    for (i = 0; i < n; ++i) {
        EXPECT(h_out[i] == run, "scan[%u] = %u, expected %u", i, h_out[i], run);
        run += h_in[i];
    }
    free(h_in);
    free(h_out);
    printf("ok scan %u\n", n);
    return 0;
}

int main(int argc, char** argv) {
    mp_engine* e = NULL;
    int rc;
    if (argc < 2) return 2;
    if (abi_checks()) return 1;
    if (strcmp(argv[1], "abi") == 0) return 0;
    CHECK(mp_engine_create(0, &e));
    EXPECT(mp_engine_particle_count(e) == 200000, "Engine() seeds 200K particles (Engine.cpp:101)");
    rc = isolated_particle(e) || cube_drop(e) || scan(e);
    CHECK(mp_engine_destroy(e));
    if (rc == 0) printf("ok all\n");
    return rc;
}
