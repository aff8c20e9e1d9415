/*
 * hidem_oracle.c — CPU restatement of the HiDEM per-timestep hot path.
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py as the checker of the CUDA path; never by the product.
 * The precision-generic body lives in hidem_oracle_impl.h, instantiated here for
 * the mixed (float lp/ct) and the plain FP64 builds of the reference.
 */
#define _POSIX_C_SOURCE 199309L
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

static int clampi_(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

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
