/*
 * hidem_oracle.c — CPU restatement of the HiDEM per-timestep hot path.
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py as the checker of the CUDA path; never by the product.
 * The precision-generic body lives in hidem_oracle_impl.h, instantiated here for
 * the mixed (float lp/ct) and the plain FP64 builds of the reference.
 */
#define _POSIX_C_SOURCE 199309L
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "hidem_oracle.h"

/* GlacierDem maps of the next runs (slot 0 bed height, 1 bed friction, 2..7 external
 * forces x y z u v w); the caller keeps the data alive. */
static hidem_map2d g_maps[8];
static int g_map_set[8];

void hidem_oracle_set_maps(const hidem_map2d *bed, const hidem_map2d *friction,
                           const hidem_map2d *ext) {
    memset(g_maps, 0, sizeof g_maps);
    memset(g_map_set, 0, sizeof g_map_set);
    if (bed) { g_maps[0] = *bed; g_map_set[0] = 1; }
    if (friction) { g_maps[1] = *friction; g_map_set[1] = 1; }
    if (ext)
        for (int k = 0; k < 6; ++k) { g_maps[2 + k] = ext[k]; g_map_set[2 + k] = 1; }
}

/* Link functor of the next runs: 0 the default (HiDEMDefLinkForceFunc), 1 the IceBlock
 * sample's own (HiDEM/IceBlock/MainIceBlock.cpp:173-262). */
static int g_link_variant;

void hidem_oracle_set_link_variant(int variant) { g_link_variant = variant; }

static int clampi_(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Collision mesh of the next runs (the caller keeps its arrays alive) and the face forces
 * of the last run with a mesh ([triangle][x y z], lp of that run). */
static hidem_mesh g_mesh;
static int g_mesh_set;
static void *g_mesh_face;
static int g_mesh_face_lp;

void hidem_oracle_set_mesh(const hidem_mesh *mesh) {
    memset(&g_mesh, 0, sizeof g_mesh);
    g_mesh_set = 0;
    if (mesh && mesh->triangles > 0) {
        g_mesh = *mesh;
        g_mesh_set = 1;
    }
}

/* Real3f arithmetic of the reference (PLiB/Util/Real3.h:142-258) */
typedef struct v3f {
    float x, y, z;
} v3f;
static v3f v3f_sub(v3f a, v3f b) { v3f r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3f v3f_mul(v3f a, v3f b) { v3f r = {a.x * b.x, a.y * b.y, a.z * b.z}; return r; }
static float v3f_dot(v3f a, v3f b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
static v3f v3f_cross(v3f a, v3f b) {
    v3f r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static float sign_f(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

#define LP float
#define LSQRT sqrtf
#define LABS fabsf
#define SFX(x) x##_mixed
#include "hidem_oracle_impl.h"
#undef LP
#undef LSQRT
#undef LABS
#undef SFX

#define LP double
#define LSQRT sqrt
#define LABS fabs
#define SFX(x) x##_fp64
#include "hidem_oracle_impl.h"
#undef LP
#undef LSQRT
#undef LABS
#undef SFX

int hidem_oracle_mesh_face_forces(void *x, void *y, void *z) {
    if (!g_mesh_face) return HIDEM_ERR_STATE;
    void *out[3] = {x, y, z};
    for (int k = 0; k < 3; ++k) {
        if (!out[k]) continue;
        for (int64_t t = 0; t < g_mesh.triangles; ++t) {
            if (g_mesh_face_lp == 4)
                ((float *)out[k])[t] = ((const float *)g_mesh_face)[3 * t + k];
            else
                ((double *)out[k])[t] = ((const double *)g_mesh_face)[3 * t + k];
        }
    }
    return 0;
}

int hidem_oracle_mesh_accel(int32_t precision, int32_t counts[3], double lower[3], double upper[3],
                            int32_t *sizes, int32_t *starts, int32_t *values, int64_t values_cap,
                            int64_t *values_count) {
    if (!g_mesh_set) return HIDEM_ERR_STATE;
    int64_t cells, nv;
    int c[3];
    double lo[3], hi[3];
    int32_t *sz, *st, *va;
    if (precision == HIDEM_PREC_MIXED) {
        mesh_accel_mixed A;
        mesh_build_mixed(&g_mesh, &A);
        c[0] = A.xCount; c[1] = A.yCount; c[2] = A.zCount;
        lo[0] = A.xLower; lo[1] = A.yLower; lo[2] = A.zLower;
        hi[0] = A.xUpper; hi[1] = A.yUpper; hi[2] = A.zUpper;
        cells = A.cells; nv = A.nvalues; sz = A.sizes; st = A.starts; va = A.values;
    } else {
        mesh_accel_fp64 A;
        mesh_build_fp64(&g_mesh, &A);
        c[0] = A.xCount; c[1] = A.yCount; c[2] = A.zCount;
        lo[0] = A.xLower; lo[1] = A.yLower; lo[2] = A.zLower;
        hi[0] = A.xUpper; hi[1] = A.yUpper; hi[2] = A.zUpper;
        cells = A.cells; nv = A.nvalues; sz = A.sizes; st = A.starts; va = A.values;
    }
    for (int k = 0; k < 3; ++k) {
        if (counts) counts[k] = c[k];
        if (lower) lower[k] = lo[k];
        if (upper) upper[k] = hi[k];
    }
    if (sizes) memcpy(sizes, sz, sizeof(int32_t) * (size_t)cells);
    if (starts) memcpy(starts, st, sizeof(int32_t) * (size_t)cells);
    if (values) memcpy(values, va, sizeof(int32_t) * (size_t)(nv < values_cap ? nv : values_cap));
    if (values_count) *values_count = nv;
    free(sz);
    free(st);
    free(va);
    return 0;
}

int hidem_oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int hidem_oracle_cells(const hidem_params *P, const hidem_particle_soa *p, int64_t n, int32_t *ix,
                       int32_t *iy, int32_t *iz, int64_t dims[3], double mins[3]) {
    if (!P || !p || n <= 0) return HIDEM_ERR_ARG;
    return P->precision == HIDEM_PREC_MIXED ? cells_mixed(P, p, n, ix, iy, iz, dims, mins)
                                            : cells_fp64(P, p, n, ix, iy, iz, dims, mins);
}

int hidem_oracle_neighbours(const hidem_params *P, const hidem_particle_soa *p, int64_t n,
                            int32_t *counts, int32_t *list, int64_t cap, int64_t *total) {
    if (!P || !p || n <= 0) return HIDEM_ERR_ARG;
    return P->precision == HIDEM_PREC_MIXED
               ? neighbours_mixed(P, p, n, counts, list, cap, total)
               : neighbours_fp64(P, p, n, counts, list, cap, total);
}

int hidem_oracle_run(const hidem_params *P, hidem_particle_soa *p, int64_t n, hidem_link_soa *l,
                     int64_t L, int64_t start_step, int32_t nsteps, void *force_out[6],
                     int64_t *ev_link, int64_t *ev_step, int64_t ev_cap, int64_t *ev_count,
                     int64_t *regen_steps, int64_t regen_cap, int64_t *regen_count,
                     double *seconds) {
    if (!P || !p || !l || n <= 0 || L < 0 || nsteps < 0) return HIDEM_ERR_ARG;
    return P->precision == HIDEM_PREC_MIXED
               ? run_mixed(P, p, n, l, L, start_step, nsteps, force_out, ev_link, ev_step, ev_cap,
                           ev_count, regen_steps, regen_cap, regen_count, seconds)
               : run_fp64(P, p, n, l, L, start_step, nsteps, force_out, ev_link, ev_step, ev_cap,
                          ev_count, regen_steps, regen_cap, regen_count, seconds);
}
