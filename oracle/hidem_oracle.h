/*
 * hidem_oracle.h — CPU restatement of the HiDEM hot path. TEST INFRASTRUCTURE ONLY.
 *
 * Plain C, IEEE arithmetic (built with -fno-fast-math -ffp-contract=off), one
 * function per reference stage, each citing the reference file:line it restates.
 * Used only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg, as
 * the checker of the CUDA path. It is pinned against the reference's own CPU code
 * (oracle/_ref, built from the reference sources by oracle/Makefile) and against
 * the committed fixtures under tests/golden/.
 */
#ifndef HIDEM_ORACLE_H
#define HIDEM_ORACLE_H
#include <stdint.h>
#include "hidem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Cells of NeighbourGrid::generate (PLiB/NeighbourGrid.cpp:48-161). */
int hidem_oracle_cells(const hidem_params *P, const hidem_particle_soa *p, int64_t n,
                       int32_t *ix, int32_t *iy, int32_t *iz, int64_t dims[3], double mins[3]);

/* Contact list of NeighAccel::generateNeighbours (PLiB/Accel/NeighAccel.h:25-137),
 * rows packed in the reference order. */
int hidem_oracle_neighbours(const hidem_params *P, const hidem_particle_soa *p, int64_t n,
                            int32_t *counts, int32_t *list, int64_t cap, int64_t *total);

/* The sample-main timestep loop over [start_step, start_step + nsteps); same
 * contract as the reference harness's hidem_ref_run. */
int hidem_oracle_run(const hidem_params *P, hidem_particle_soa *p, int64_t n, hidem_link_soa *l,
                     int64_t L, int64_t start_step, int32_t nsteps, void *force_out[6],
                     int64_t *ev_link, int64_t *ev_step, int64_t ev_cap, int64_t *ev_count,
                     int64_t *regen_steps, int64_t regen_cap, int64_t *regen_count,
                     double *seconds);

int hidem_oracle_threads(void);

/* Bed / friction / external force maps used by the integrate step of the next runs
 * (NULL: none); the data must stay alive while they run. */
void hidem_oracle_set_maps(const hidem_map2d *bed, const hidem_map2d *friction,
                           const hidem_map2d *ext);

/* Collision mesh used by the integrate step of the next runs (NULL: none), as
 * HiDEM/MeshConstrainedDem/MainMeshDem.cpp:111-113, 220-235 uses it; the arrays must
 * stay alive while they run. */
void hidem_oracle_set_mesh(const hidem_mesh *mesh);
/* 0: HiDEMDefLinkForceFunc; 1: the IceBlock sample's link functor */
void hidem_oracle_set_link_variant(int variant);
/* Face forces accumulated over the last run with a mesh (summed in particle order),
 * lp [triangles] each. */
int hidem_oracle_mesh_face_forces(void *x, void *y, void *z);
/* The MeshAccel grid of the set mesh in the given precision (the contract of
 * hidem_get_mesh_accel). */
int hidem_oracle_mesh_accel(int32_t precision, int32_t counts[3], double lower[3], double upper[3],
                            int32_t *sizes, int32_t *starts, int32_t *values, int64_t values_cap,
                            int64_t *values_count);

#ifdef __cplusplus
}
#endif
#endif
