/*
 * hidem_b200.h — C ABI of the B200-native HiDEM per-timestep hot path.
 *
 * One context owns one particle set and one link set resident in device
 * memory of one GPU, one CUDA stream, and the neighbour / link acceleration
 * structures.  Host arrays passed in or out are caller-owned and copied.
 * Every entry point returns a hidem_status; none exits or raises signals
 * (the reference's getErrorDev/exit(1) convention, Iterators/DevCall.h:29-91,
 * becomes a status code plus hidem_last_error()).
 *
 * Layout contract (reference field order, HiDEMLib/HiDEMParticleData.h:45-51,
 * HiDEMLib/HiDEMLinkData.h:39-50):
 *   particles: xCord yCord zCord (f64) xTheta yTheta zTheta xDiff yDiff zDiff
 *              uDiff vDiff wDiff radius (lp) owners (i32) type (u8) globalKeys (i64)
 *   links:     owners (i32) state (u8) globalKeys globalKeyEndA globalKeyEndB (i64)
 *              initialLen (lp) particleLinkNum (i32)
 *   link sides: CT0..CT5 (ct), 2 values per link: [sideA(l0), sideB(l0), sideA(l1), ...]
 *              (the checkpoint order, PLiB/LinkDataHandler.h:373-380,443-446)
 * lp = ct = float in HIDEM_PREC_MIXED (the reference default build, FP64
 * positions, PLiB/Global.h.in:47-52 with SET_FP32/SET_CT_FP32) and double in
 * HIDEM_PREC_FP64 (the reference built with both flags off).
 */
#ifndef HIDEM_B200_H
#define HIDEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HIDEM_B200_ABI_VERSION 1

typedef enum hidem_status {
    HIDEM_OK = 0,
    HIDEM_ERR_ARG = 1,       /* null pointer, negative size, unknown enum value */
    HIDEM_ERR_CUDA = 2,      /* a CUDA runtime call failed; see hidem_last_error */
    HIDEM_ERR_STATE = 3,     /* call out of order (e.g. forces before particles) */
    HIDEM_ERR_CAPACITY = 4,  /* a size exceeds a fixed limit (int32 indices, per-particle width) */
    HIDEM_ERR_IO = 5,        /* checkpoint or run-config file error */
    HIDEM_ERR_DEVICE = 6,    /* a device-side check failed (index out of range) */
    HIDEM_ERR_NOT_FOUND = 7  /* a link end names a globalKey that is not a particle */
} hidem_status;

typedef enum hidem_precision {
    HIDEM_PREC_FP64 = 0,  /* lp = ct = double */
    HIDEM_PREC_MIXED = 1  /* lp = ct = float, positions double (reference default) */
} hidem_precision;

/* Bits of the particle `type` byte read by the integrate step (extensions of
 * the sample integrate lambdas; the low bits keep the reference's material
 * type used for link generation). */
#define HIDEM_TYPE_FIXED 0x40u /* held in place: position and rotation unchanged, diffs zero */
#define HIDEM_TYPE_FRONT 0x80u /* calving-front face: hydrostatic pressure below waterLevel */

/* Raw run-config values (TOML keys general.*, grid.*, distribution.*; defaults
 * from HiDEM/MeshBlock/MainMeshBlock.cpp:69-102 and HiDEMLib/HiDEMLib.h:714-750).
 * Derived constants (scaled drags, invDt, W2, W4, G, ...) are computed inside
 * the library in lp precision exactly as the sample main does. */
typedef struct hidem_params {
    double dt, scale, E, beamWidth, damping, dampingRotation;
    double attractDistance, attractScaleForce;
    double maxLoad, bendBreak, breakTime;
    double g, rhoIce, rhoWater, waterLevel;
    double airDrag, waterDrag, bedDrag, bedStiffness, bedInteract;
    double maxVel, maxRot;
    double lowerLimit[3], upperLimit[3];    /* simulation box for the boundary conditions */
    int32_t boundaryMin[3], boundaryMax[3]; /* general.{x,y,z}Boundary{Min,Max} */
    double searchDistanceScale;             /* grid.searchDistanceScale */
    int32_t gridRegenInterval;              /* grid.gridRegenInterval (-1: displacement rule) */
    int32_t firstBalanceTimestep;           /* distribution.firstBalanceTimestep (forces a rebuild) */
    double maxRadius;                       /* largest particle radius (geometry.maxRadius) */
    /* integrate extensions (off in the MeshBlock sample) */
    int32_t useBed;                         /* flat bed: GlacierDem bed drag + stiffness (HiDEM/GlacierDem/MainDem.cpp:176-207) */
    double bedHeight, bedFriction;
    int32_t useVelocityLimit;               /* HiDEMDefVelocityLimit */
    int32_t useBoundary;                    /* HiDEMDefBoundaryCondition */
    int32_t useFixed;                       /* honour HIDEM_TYPE_FIXED */
    int32_t useFrontPressure;               /* honour HIDEM_TYPE_FRONT */
    int32_t precision;                      /* hidem_precision */
} hidem_params;

/* Particle arrays, reference field order. lp fields point at float (mixed) or
 * double (fp64) arrays of n elements. Any pointer may be NULL on output calls
 * to skip that field. */
typedef struct hidem_particle_soa {
    double *xCord, *yCord, *zCord;
    void *xTheta, *yTheta, *zTheta;
    void *xDiff, *yDiff, *zDiff, *uDiff, *vDiff, *wDiff;
    void *radius;
    int32_t *owners;
    uint8_t *type;
    int64_t *globalKeys;
} hidem_particle_soa;

/* Link arrays (L elements) plus side data CT0..CT5 (2L elements each). */
typedef struct hidem_link_soa {
    int32_t *owners;
    uint8_t *state;
    int64_t *globalKeys, *globalKeyEndA, *globalKeyEndB;
    void *initialLen;
    int32_t *particleLinkNum;
    void *CT[6];
} hidem_link_soa;

typedef struct hidem_ctx hidem_ctx;

/* Counters of what the last calls did (for logs and tests). */
typedef struct hidem_stats {
    int64_t step;              /* current timestep (HiDEMLib::currentTimestep) */
    int64_t num_particles, num_links;
    int64_t num_neighbour_pairs;   /* directed pairs in the contact list */
    int64_t max_neighbours, max_links_per_particle;
    int64_t grid_dims[3];
    double grid_min[3];
    int64_t regen_count;       /* neighbour-structure rebuilds so far */
    int64_t last_regen_step;
    double accumulated_dist;   /* HiDEMLib::accumulatedDist */
    double search_distance, interact_distance;
    int64_t broken_links;      /* links with state == 0 */
    int64_t kernel_launches;   /* kernels launched by this context so far */
    int64_t grid_growth_events; /* rebuilds whose grid had more than 10x the previous one's
                                   cells (NeighbourGrid.cpp:89-92 prints a warning there) */
} hidem_stats;

/* ---- defaults -------------------------------------------------------- */

/* MeshBlock sample defaults (HiDEM/MeshBlock/MainMeshBlock.cpp:69-102,
 * HiDEMLib/HiDEMLib.h:714-750); extensions off; precision mixed. */
void hidem_params_default(hidem_params *p);

/* Run config from a TOML file plus command-line overrides — the keys the sample main
 * and HiDEMLib::setup read (MainMeshBlock.cpp:69-102, HiDEMLib.h:714-750, maxRadius =
 * lattice.particleRadius * general.scale as HiDEMGeometry.cpp:88-92) and ArgParser's
 * `--section.key=value` overrides (PLiB/Util/ArgParser.h:170-270). Keys that are absent
 * keep the hidem_params_default values; extension keys in [general]: useBed, bedHeight,
 * bedFriction, useVelocityLimit, useBoundary, useFixed, useFrontPressure, lowerLimit,
 * upperLimit, precision ("mixed" | "fp64"). path may be NULL (overrides only);
 * time_steps (may be NULL) receives iteration.timeSteps. Errors: HIDEM_ERR_IO with the
 * text in hidem_create_error(). */
hidem_status hidem_params_from_toml(const char *path, int32_t argc, const char *const *argv,
                                    hidem_params *out, int64_t *time_steps);

/* ---- context --------------------------------------------------------- */

/* Replaces HiDEMLib::setup (HiDEMLib/HiDEMLib.h:707-822) for the hot path:
 * selects `device`, creates the stream and the derived constants. */
hidem_status hidem_create(const hidem_params *params, int device, hidem_ctx **out);
void hidem_destroy(hidem_ctx *ctx);
const char *hidem_last_error(const hidem_ctx *ctx);
/* Per-thread text of the last failure of a call that has no context
 * (hidem_create, hidem_params_from_toml, hidem_read_particle_file, hidem_bin_cells_noalloc). */
const char *hidem_create_error(void);
int hidem_abi_version(void);

/* Replaces ParticleDataHandler::appendInitParticles / fromCheckpoint
 * (PLiB/ParticleDataHandler.h:215-267): copies n particles to the device.
 * The arrays of hidem_set_particles / hidem_set_links and of the readbacks
 * hidem_get_particles / hidem_get_links may be host memory (pageable or pinned) or device
 * memory of the context's GPU (the copies stay on the device); device arrays handed in must
 * be complete when the call is made (the caller has synchronised the work that wrote
 * them), and the readbacks' arrays are complete when the call returns. */
hidem_status hidem_set_particles(hidem_ctx *ctx, const hidem_particle_soa *p, int64_t n);
/* Replaces LinkDataHandler::appendInitLinks + LinkData::makeLocalPartEnds
 * (PLiB/LinkDataHandler.h:212-241, PLiB/LinkData.h:91-115): copies L links,
 * resolves their ends by globalKey, zeroes CT when `links->CT[0]` is NULL. */
hidem_status hidem_set_links(hidem_ctx *ctx, const hidem_link_soa *l, int64_t L);
/* Sets the timestep counter (restart: HiDEMLib::setFromRestart, HiDEMLib.h:840-846). */
hidem_status hidem_set_timestep(hidem_ctx *ctx, int64_t step);
/* Replaces the per-config params after creation (same precision). */
hidem_status hidem_set_params(hidem_ctx *ctx, const hidem_params *params);

/* ---- the per-timestep operator surface (HiDEMLib.h:256-530) ---------- */

/* HiDEMLib::gridService (HiDEMLib.h:533-628): displacement-accumulation rule,
 * then, when due, cell binning + reorder, contact list and link lists. */
hidem_status hidem_grid_service(hidem_ctx *ctx);
/* Forces a rebuild now (CombinedAccel::generateNeighbours + generateLinks). */
hidem_status hidem_regenerate(hidem_ctx *ctx);
/* HiDEMLib::computePartForce with HiDEMDefNeighForceFunc + HiDEMDefLinkForceFunc
 * (HiDEMLib.h:316-382, PLiB/Accel/CombinedAccel.h:122-197): writes the six
 * force arrays and advances CT. */
hidem_status hidem_compute_forces(hidem_ctx *ctx);
/* HiDEMLib::applyForce with the sample integrate lambda
 * (HiDEMLib.h:303-314, HiDEM/MeshBlock/MainMeshBlock.cpp:182-261). */
hidem_status hidem_integrate(hidem_ctx *ctx);
/* HiDEMLib::linkUpdate with HiDEMDefLinkBreakFunc (HiDEMLib.h:256-269,
 * PLiB/Accel/CombinedAccel.h:200-235). Always applies the functor; the
 * t*dt > breakTime gate of the sample main is the caller's (hidem_step applies it). */
hidem_status hidem_link_update(hidem_ctx *ctx);
/* HiDEMLib::finalizeTs (HiDEMLib.h:495-530): ++timestep. */
hidem_status hidem_finalize_ts(hidem_ctx *ctx);

/* ---- slab decomposition hooks (one context per rank) ------------------ */

/* The reference spreads one particle set over MPI ranks (HiDEMLib/HiDEMDistribution.h:
 * 99-234): each rank holds the particles it owns plus halo copies of its neighbours'
 * particles, computes the forces of its own, receives the forces of its halo particles
 * from their owners and integrates both (computePartForce, HiDEMLib.h:316-382, the
 * pForceComm exchange), and gridService reduces the displacement over ranks
 * (accumulateDist, HiDEMLib.h:463-474, MPI_Allreduce). These calls split the
 * rank-spanning steps so that the caller's transport (NCCL, or copies between
 * contexts of one process) does the exchange and the reductions:
 *
 *   gridService:  hidem_grid_service_local -> max over ranks -> hidem_grid_service_decide;
 *                 on regen: hidem_local_bounds -> min/max over ranks -> hidem_regenerate_frame
 *   forces:       hidem_compute_forces -> hidem_pack_halo_forces -> exchange ->
 *                 hidem_unpack_halo_forces -> hidem_integrate -> hidem_link_update ->
 *                 hidem_finalize_ts
 *
 * Indices are particle indices in the order of the last hidem_set_particles call. */

/* This rank's part of gridService's displacement rule at the current step: the maxima
 * over its particles of max(0, xDiff / yDiff / zDiff), as doubles (HiDEMLib.h:424-460).
 * *needs_reduce = 1 when the step reads them (the rule runs every 10 steps), else 0 and
 * diff_max is zeros. */
hidem_status hidem_grid_service_local(hidem_ctx *ctx, double diff_max[3], int32_t *needs_reduce);
/* The rest of gridService's decision from the maxima over all ranks (element-wise max of
 * every rank's hidem_grid_service_local): accumulated distance updated as
 * HiDEMLib.h:463-474 and 563-575 do, *regen = 1 when the neighbour structures must be
 * rebuilt now. Rebuilds nothing: the caller redistributes if it wants to, then calls
 * hidem_regenerate_frame. The reference reduces each rank's distance (the norm of its
 * own maxima); reducing the maxima makes every rank's decision that of one rank holding
 * all particles. */
hidem_status hidem_grid_service_decide(hidem_ctx *ctx, const double diff_max[3], int32_t *regen);
/* Bounding box of this rank's particles (ParticleData::getLimits, PLiB/ParticleData.h:
 * 47-59). Synchronises the context's stream. */
hidem_status hidem_local_bounds(hidem_ctx *ctx, double lower[3], double upper[3]);
/* hidem_regenerate with the grid spanning [lower, upper] (the element-wise min / max of
 * every rank's hidem_local_bounds) instead of this rank's own bounding box, so that cell
 * colours, and with them every contact list's order, are those of one rank holding all
 * particles. HIDEM_ERR_ARG if a particle of this rank lies outside the box. */
hidem_status hidem_regenerate_frame(hidem_ctx *ctx, const double lower[3], const double upper[3]);
/* The halo force lists: send_index[k] is a particle this rank owns whose force another
 * rank integrates (the k-th 6-value record of the packed buffer); recv_index[k] is a halo
 * particle whose force arrives as the k-th record. The caller orders the lists by
 * destination / source rank so that each peer's records are contiguous. Copied; the
 * indices stay valid across rebuilds. Either count may be 0. */
hidem_status hidem_set_halo_exchange(hidem_ctx *ctx, const int32_t *send_index, int64_t n_send,
                                     const int32_t *recv_index, int64_t n_recv);
/* Writes the forces of the send list, n_send x 6 lp values (x, y, z, u, v, w per
 * particle), from the last hidem_compute_forces to `device_out` (device memory), on the
 * context's stream (CommunicatorPacked::packAllCommData). */
hidem_status hidem_pack_halo_forces(hidem_ctx *ctx, void *device_out);
/* hidem_compute_forces followed by hidem_pack_halo_forces into `device_out`, with the send
 * records written by the force pass itself as it finishes each listed particle (the pack
 * fused into its epilogue; after the item and asynchronous-copy force kernels the pack
 * kernel runs instead). The same forces and records as the two calls. */
hidem_status hidem_compute_forces_packed(hidem_ctx *ctx, void *device_out);
/* Overwrites the forces of the receive list with n_recv x 6 lp values read from
 * `device_in` (device memory), on the context's stream; the caller has made the stream
 * wait for the data (CommunicatorPacked::unpackAllCommData). */
hidem_status hidem_unpack_halo_forces(hidem_ctx *ctx, const void *device_in);
/* n whole timesteps of the sample main loop (MainMeshBlock.cpp:274-323):
 * gridService, forces, integrate, gated link update, finalizeTs — each step as the
 * context's step kernel (hidem_set_step_kernel: one fused kernel, or the two-pass step's
 * force and integrate passes and break pass), launched back to back between the
 * gridService checks without host synchronisation. */
hidem_status hidem_step(hidem_ctx *ctx, int32_t nsteps);
/* The default functors as a caller's main constructs them (HiDEM/Common/
 * HiDEMDefaultFunctions.h): HiDEMDefNeighForceFunc(invDt, attractDistance,
 * attractScaleForce, damping, dampingRotation, scaleE) (21-87), HiDEMDefLinkForceFunc(invDt,
 * damping, dampingRotation, E, W2, W4, G) (90-204), HiDEMDefLinkBreakFunc(bendBreak,
 * maxLoad) (207-242). Values are lp (each double is rounded once to float in
 * HIDEM_PREC_MIXED). hidem_create / hidem_set_params derive them from the run config as the
 * MeshBlock sample does (MainMeshBlock.cpp:106-156); hidem_set_functor_params replaces them
 * (until the next hidem_set_params), hidem_get_functor_params reads the ones in use. The
 * integrate step keeps the run config's constants. */
typedef struct hidem_functor_params {
    double neigh_invDt, neigh_attractDistance, neigh_attractScaleForce;
    double neigh_damping, neigh_dampingRotation, neigh_scaleE;
    double link_invDt, link_damping, link_dampingRotation, link_E, link_W2, link_W4, link_G;
    double break_bendBreak, break_maxLoad;
} hidem_functor_params;
hidem_status hidem_set_functor_params(hidem_ctx *ctx, const hidem_functor_params *f);
hidem_status hidem_get_functor_params(hidem_ctx *ctx, hidem_functor_params *out);
/* Run-time checks beyond the reference's behaviour. The reference prints "grid 10x larger
 * than old, did something explode?" when a rebuild's grid has more than ten times the
 * cells of the previous one and carries on (PLiB/NeighbourGrid.cpp:89-92); the library
 * counts such rebuilds in hidem_stats.grid_growth_events, and with HIDEM_CHECK_GRID_GROWTH
 * set the rebuild fails with HIDEM_ERR_DEVICE instead. Always on, whatever the flags:
 * non-finite coordinates (NaN or infinite) fail a rebuild with HIDEM_ERR_DEVICE; a
 * neighbour-grid cell of more than 4096 particles fails it with HIDEM_ERR_CAPACITY; a link
 * end that names no particle fails hidem_set_links with HIDEM_ERR_NOT_FOUND
 * (LinkData::makeLocalPartEnds, PLiB/LinkData.h:102-108, exits there). */
#define HIDEM_CHECK_GRID_GROWTH 1
hidem_status hidem_set_checks(hidem_ctx *ctx, int32_t flags);
/* Blocks until the context's stream is idle; reports device-side check failures. */
hidem_status hidem_synchronize(hidem_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work
 * on it (e.g. CUDA events recorded on the same stream). */
void *hidem_get_stream(hidem_ctx *ctx);
/* Turns CUDA-event timing of each step's kernels (the fused kernel, or the two-pass
 * step's passes) on (1) or off (0) and clears the record; hidem_profile_read sums their
 * time over the steps since then and returns the number of steps timed. */
hidem_status hidem_profile(hidem_ctx *ctx, int32_t enable);
hidem_status hidem_profile_read(hidem_ctx *ctx, double *step_kernel_ms, int64_t *launches);

/* ---- device view (for the templated operator surface) ------------------ */

/* The context's device arrays as the templated CUDA header include/hidem_b200_iterate.cuh
 * reads them: the counterpart of the reference handing its ParticleData / LinkData objects
 * (managed memory, Iterators/Allocator.h:18-76) to Iterator::iterate and to the functors of
 * computePartForce / linkUpdate / applyForce (HiDEMLib.h:256-382). Particles are in storage
 * ("slot") order, the order the reference's own pInd indices follow after its
 * redistribution reorder: neighbour-grid cell, then input index.
 *   record of slot s at records + s * record_bytes: x y z (f64), xDiff yDiff zDiff uDiff
 *     vDiff wDiff (lp), radius (lp), xTheta yTheta zTheta (lp) [FP64: 3 doubles of padding]
 *   force: 6 lp arrays of n (xForce..wForce, slot order), what computePartForce writes and
 *     applyForce reads
 *   contact k of slot s at contacts[contact_offsets[s / 32] + 32 k + s % 32] (a partner slot),
 *     counts[s] & 0xffff contacts; link end k at end_offsets[s / 32] + 32 k + s % 32,
 *     counts[s] >> 16 ends in ascending link index: end_partner (partner slot, bit 31 set
 *     when this is end B of the link), end_ct[0..5] (CT0..CT5), end_state (the link's state
 *     as the force loop reads it), end_initial_length, end_link (input link index)
 *   per link (input order): link_state, link_slot_a / link_slot_b (the ends' slots),
 *     link_initial_length, link_end_index[2 l + e] (the end storage index of end e)
 * Taking the view builds the neighbour structures if none exist. It stays valid until the
 * next call that rebuilds them or swaps the particle records (hidem_grid_service,
 * hidem_regenerate, hidem_step, hidem_set_particles / hidem_set_links): take it again after
 * each. Work on it is ordered on `stream`, the context's stream. */
typedef struct hidem_device_view {
    int32_t precision;         /* hidem_precision: lp = float (mixed) or double (FP64) */
    int32_t record_bytes;      /* 64 (mixed) or 128 (FP64) */
    int64_t n, L, step;
    void *records;
    void *force;
    uint8_t *type;             /* per slot */
    const int32_t *input_index;/* slot -> input index */
    const int32_t *slot_of;    /* input index -> slot */
    const uint32_t *counts;
    const int64_t *contact_offsets;
    const int32_t *contacts;
    const int64_t *end_offsets;
    const uint32_t *end_partner;
    void *end_ct[6];
    uint8_t *end_state;
    void *end_initial_length;
    const int32_t *end_link;
    uint8_t *link_state;
    const int32_t *link_slot_a, *link_slot_b;
    void *link_initial_length;
    const int32_t *link_end_index;
    /* link-break events (input link index, timestep), the same list hidem_get_break_events
       reads: an event is added at events[atomicAdd(event_count, 1)] when below event_capacity */
    void *events;
    unsigned long long *event_count;
    int64_t event_capacity;
    void *stream;              /* cudaStream_t */
} hidem_device_view;
hidem_status hidem_get_device_view(hidem_ctx *ctx, hidem_device_view *out);

/* ---- readback (input order: index i is the i-th particle / link given) -- */

hidem_status hidem_get_particles(hidem_ctx *ctx, hidem_particle_soa *out);
hidem_status hidem_get_links(hidem_ctx *ctx, hidem_link_soa *out);
/* Six lp arrays (x,y,z,u,v,w) of the last hidem_compute_forces. */
hidem_status hidem_get_forces(hidem_ctx *ctx, void *force[6]);
/* Cell (ix,iy,iz) of each particle at the last rebuild, grid dims and minimum
 * corner (NeighbourGrid::getGridId / generateNeighbourGrid, PLiB/NeighbourGrid.cpp:31-114). */
hidem_status hidem_get_cells(hidem_ctx *ctx, int32_t *ix, int32_t *iy, int32_t *iz,
                             int64_t dims[3], double mins[3]);
/* Contact list of the last rebuild, in the reference's per-particle order
 * (NeighAccel::generateNeighbours, PLiB/Accel/NeighAccel.h:25-137):
 * counts[n] and, when `list` is not NULL, the neighbour input indices packed
 * row after row (sum(counts) entries, at most `cap`). */
hidem_status hidem_get_neighbours(hidem_ctx *ctx, int32_t *counts, int32_t *list, int64_t cap,
                                  int64_t *total);
/* Links broken since the last call: input link indices and the timestep at
 * which each broke (HiDEMDefLinkBreakFunc decisions), at most `cap`. */
hidem_status hidem_get_break_events(hidem_ctx *ctx, int64_t *link_index, int64_t *step,
                                    int64_t cap, int64_t *count);
hidem_status hidem_get_stats(hidem_ctx *ctx, hidem_stats *out);

/* ---- checkpoint (HDF5) ------------------------------------------------ */

/* Writes the context's state in the reference's checkpoint layout for one rank
 * (HiDEMLib/HiDEMH5Checkpoint.h:24-50, PLiB/H5IO/H5Checkpoint.h:42-111,
 * PLiB/ParticleDataHandler.h:215-230, PLiB/LinkDataHandler.h:356-395): root attribute
 * timeStep; groups Domains, Particles (field_0..15), Links (field_0..6), LinkSideData
 * (side_field_7..12, CT in [sideA, sideB] order), spann_sizes / spann_offsets; contiguous
 * datasets, lp fields float (mixed) or double (FP64). The file is written by the
 * library's own HDF5 encoder (superblock v2, compact groups). */
hidem_status hidem_checkpoint_write(hidem_ctx *ctx, const char *path);
/* Restarts from such a file (ParticleDataHandler::fromCheckpoint, LinkDataHandler::
 * fromCheckpoint, HiDEMLib::setFromRestart): timestep, particles, links, CT. The file's
 * lp type must match the context's precision. */
hidem_status hidem_checkpoint_read(hidem_ctx *ctx, const char *path);

/* ---- lattice generation (setup-side inputs for the workloads) --------- */

/* FCC lattice of nx*ny*nz unit cells, lattice constant a, radius r, origin o,
 * each coordinate jittered by U(-jitter, +jitter) from a seeded 64-bit
 * Mersenne Twister (std::mt19937_64). Sites in z, y, x, site order; globalKeys
 * 0..n-1; thetas, diffs zero. Arrays must hold 4*nx*ny*nz elements. `lp` fields
 * follow `precision`. */
hidem_status hidem_lattice_fcc(int32_t nx, int32_t ny, int32_t nz, double a, double radius,
                               const double origin[3], double jitter, uint64_t seed,
                               int32_t precision, hidem_particle_soa *out);
/* Distance-rule link generation (PLiB/Generators/LinkGenerator.h:60-110):
 * every pair i<j (by globalKey) with |x_i - x_j| <= scale*(r_i + r_j) gets a
 * link, ordered by (endA input index, endB input index), initialLen = |x_i-x_j|.
 * With out==NULL only *count is written. */
hidem_status hidem_links_by_distance(const hidem_particle_soa *p, int64_t n, int32_t precision,
                                     double scale, hidem_link_soa *out, int64_t cap,
                                     int64_t *count);

/* Replaces FileParticleGenerator::generate (PLiB/Generators/FileParticleGenerator.h:23-105)
 * on one rank: the HDF5 point file of the reference's File lattice (lattice.path; the
 * HiDEM/Benchmark/<size>/particles.h5 inputs of its MeshBlock benchmark, as libhdf5 writes
 * them: superblock 0, symbol-table groups, deflate-compressed chunks). Datasets x_name,
 * y_name, z_name, radius_name of the root group (lattice.xCords / yCords / zCords / radius;
 * NULL for "xCord", "yCord", "zCord", "radius"); each value is read as float, as the
 * reference reads them (readVectorSpann<float>), and stored in the particle fields
 * (positions as double); thetas and diffs zero, owners and type 0, globalKeys 0..n-1
 * (ParticleGenerator::setParticleKeys). The reference then keeps the particles that lie
 * inside their bounding geometry (createParticle, PLiB/Generators/ParticleGenerator.h:37-57);
 * that test is the caller's (the benchmark files hold only such points). With out == NULL
 * only *count is written. Errors: HIDEM_ERR_IO with the text in hidem_create_error(). */
hidem_status hidem_read_particle_file(const char *path, const char *x_name, const char *y_name,
                                      const char *z_name, const char *radius_name, int32_t precision,
                                      hidem_particle_soa *out, int64_t cap, int64_t *count);

/* ---- bed and external force maps ------------------------------------- */

/* A regular 2-D map in the reference's Map2d form (PLiB/Geometry/Map2d.h:23-60): values
 * (lp: float in HIDEM_PREC_MIXED, double in HIDEM_PREC_FP64) at x_points x y_points grid
 * points spanning [x_min, x_max] x [y_min, y_max], x fastest (data[ix + iy * x_points]).
 * Values between points are Map2d::interp's bilinear interpolation in float arithmetic
 * (Map2d.h:93-152), clamped to the grid outside it. */
typedef struct hidem_map2d {
    const void *data;
    int32_t x_points, y_points;
    float x_min, y_min, x_max, y_max;
} hidem_map2d;
/* The GlacierDem bed (InputBed, PLiB/Geometry/InputGeometry.h:54-78, used by
 * HiDEM/GlacierDem/MainDem.cpp:176-207): with params.useBed set, the bed height under a
 * particle is bed(x, y) instead of params.bedHeight, and the bed friction is
 * friction(x, y) instead of params.bedFriction. Either may be NULL (the constant). The
 * data is copied. */
hidem_status hidem_set_bed_maps(hidem_ctx *ctx, const hidem_map2d *bed, const hidem_map2d *friction);
/* External force maps (ExternalForces, PLiB/ExternalForces.h; MainDem.cpp:211-216): six
 * maps added to the x, y, z forces and u, v, w moments of every particle at its (x, y)
 * in the integrate step, after gravity, buoyancy and the bed force. maps: 6 maps, or NULL
 * to remove them. The data is copied. */
hidem_status hidem_set_external_force_maps(hidem_ctx *ctx, const hidem_map2d *maps);

/* ---- collision mesh ---------------------------------------------------- */

/* A triangle mesh the particles collide with, as the MeshConstrainedDem sample uses it
 * (HiDEM/MeshConstrainedDem/MainMeshDem.cpp:111-113, 220-235): the reference's
 * CollisionMesh (PLiB/Geometry/CollisionMesh.h, Mesh.h) with its MeshAccel grid
 * (PLiB/Geometry/MeshAccel.h). Vertex j of triangle t is (x_vertex[3t + j],
 * y_vertex[3t + j], z_vertex[3t + j]) and its normal (x_normal[t], ...), the MeshData
 * layout (PLiB/MeshData.h:21-27); all lp (float in HIDEM_PREC_MIXED, double in
 * HIDEM_PREC_FP64). */
typedef struct hidem_mesh {
    const void *x_vertex, *y_vertex, *z_vertex;  /* [3 * triangles] */
    const void *x_normal, *y_normal, *z_normal;  /* [triangles] */
    int32_t triangles;
    double cell_size;   /* MeshAccel cell size and search distance (the sample: 16 maxRadius) */
    double mesh_force;  /* general.meshForce (the sample's default 1e7) */
    double mesh_drag;   /* general.meshDrag (1000) */
} hidem_mesh;
/* Sets the collision mesh (NULL removes it) and builds its MeshAccel grid on the device
 * (MeshAccel::generateAccel, MeshAccel.h:57-165: cells of cell_size over the vertices'
 * bounding box grown by one cell, z fastest; each cell lists, in ascending order, the
 * triangles whose squared distance from the cell centre (MeshAccel::triSDF2, 329-372) is
 * below 3 cell_size^2 + cell_size). From then on the integrate step finds, for each
 * particle inside the grid, the closest triangle of its cell within bedInteract + radius
 * (Mesh::closestTriFun / MeshAccel::getClosestTriAccel, Mesh.h:69-83, MeshAccel.h:375-412)
 * and, when there is one, pushes the particle along minus the triangle's normal by
 * mesh_force * (bedInteract + radius - distance), sets the drag coefficient to
 * mesh_drag * (bedInteract + radius - distance) and adds the push to the triangle's face
 * force (MainMeshDem.cpp:220-235), after the bed force and before the external force maps.
 * Face forces start at zero. The data is copied. */
hidem_status hidem_set_collision_mesh(hidem_ctx *ctx, const hidem_mesh *mesh);
/* The face forces accumulated since the mesh was set or last zeroed (CollisionMesh
 * xFaceForce..zFaceForce, CollisionMesh.h:46-52): lp [triangles] each. The sum over a
 * face is formed with atomic additions, as in the reference, so its rounding depends on
 * the order the particles add in. */
hidem_status hidem_get_mesh_face_forces(hidem_ctx *ctx, void *x, void *y, void *z);
/* CollisionMesh::zeroForce (CollisionMesh.h:54-62) */
hidem_status hidem_zero_mesh_face_forces(hidem_ctx *ctx);
/* The MeshAccel grid: counts (x, y, z cells), lower and upper corners (lp values as
 * doubles), per cell (index (x * Y + y) * Z + z) the triangle count and start, and the
 * triangle lists (values_cap entries at most; *values_count receives the total). Any
 * array pointer may be NULL. */
hidem_status hidem_get_mesh_accel(hidem_ctx *ctx, int32_t counts[3], double lower[3], double upper[3],
                                  int32_t *sizes, int32_t *starts, int32_t *values,
                                  int64_t values_cap, int64_t *values_count);

/* ---- diagnostics ------------------------------------------------------ */

/* Kinetic energy of the current state, the convergence measure of settling runs (no
 * counterpart in the reference's step loop): translational and rotational energy summed
 * over the particles, with velocities diff / dt and the integrate step's mass rho d^3 and
 * moment of inertia m d^2 / 6 (MainMeshBlock.cpp:228-229); max_speed the largest particle
 * speed. Any output pointer may be NULL. Synchronises the context's stream. */
hidem_status hidem_kinetic_energy(hidem_ctx *ctx, double *translational, double *rotational,
                                  double *max_speed);
/* Momentum of the current state, with the velocities and masses of hidem_kinetic_energy:
 * linear sum m v and angular about the origin sum x (x) m v + I w, reduced in double
 * precision in a fixed order. Either pointer may be NULL. Synchronises the stream. */
hidem_status hidem_momentum(hidem_ctx *ctx, double linear[3], double angular[3]);

/* ---- step kernel choice ----------------------------------------------- */

/* No counterpart in the reference. The fused step has several kernels that give
 * bit-identical results and differ only in speed: one thread per (particle, contact) and
 * (particle, link end) item with the block's streams staged in shared memory (ITEMS), one
 * thread per particle with software-pipelined partner loads (THREAD), and the same with
 * registers capped for more CTAs per SM (THREAD_CAPPED: five in the mixed build, three in
 * FP64), and one thread per particle whose next two items' partner data travel by
 * asynchronous copies into shared memory (THREAD_ASYNC). TWO_PASS runs each timestep as
 * the THREAD_CAPPED force pass without the integrate tail, then the integrate pass over
 * the particles and the break pass over the links, as hidem_compute_forces /
 * hidem_integrate / hidem_link_update do. AUTO (the default) times each on the context's
 * own first steps (three rounds, the first discarded) and keeps the fastest; those steps
 * are ordinary timesteps. hidem_get_step_kernel returns the kernel in use (AUTO while
 * still timing). */
#define HIDEM_STEP_KERNEL_AUTO 0
#define HIDEM_STEP_KERNEL_ITEMS 1
#define HIDEM_STEP_KERNEL_THREAD 2
#define HIDEM_STEP_KERNEL_THREAD_CAPPED 3
#define HIDEM_STEP_KERNEL_THREAD_ASYNC 4
#define HIDEM_STEP_KERNEL_TWO_PASS 5
hidem_status hidem_set_step_kernel(hidem_ctx *ctx, int32_t kernel);
int32_t hidem_get_step_kernel(const hidem_ctx *ctx);

/* ---- batched contexts ------------------------------------------------- */

/* No counterpart in the reference (one HiDEMLib instance runs one particle set per
 * rank). Many independent contexts (ice blocks of uneven sizes) on one device and of one
 * precision advance together: every timestep is one launch (three for the two-pass
 * step: force, integrate and break passes) over all contexts that share their constants
 * apart from the break thresholds (maxLoad, bendBreak may differ per context; contexts
 * that differ in anything else form further launches), and the launches between two
 * gridService points (at most 10 steps) are replayed from a CUDA graph when
 * HIDEM_BATCH_GRAPHS is set. Each context's results are bit-identical to hidem_step on
 * that context alone: the batch runs the same gridService policy and the same step and
 * link update per context. The step kernel is the first context's
 * (hidem_set_step_kernel; AUTO or untimed means TWO_PASS, THREAD_ASYNC runs as
 * THREAD_CAPPED).
 * HIDEM_BATCH_PER_CONTEXT runs the single-context launch sequence context after context
 * instead (the same results, for comparison); rows too wide for the ITEMS kernel's shared
 * memory take that path too. During a batch call the contexts' work runs on the batch's
 * stream; the call returns after it finished. The contexts must outlive the batch and
 * must not be used from another thread during a batch call. On failure of
 * hidem_batch_create the text is in hidem_create_error(). */
typedef struct hidem_batch hidem_batch;
#define HIDEM_BATCH_GRAPHS 1
#define HIDEM_BATCH_PER_CONTEXT 2
hidem_status hidem_batch_create(hidem_ctx *const *ctxs, int32_t nctx, int32_t flags,
                                hidem_batch **out);
void hidem_batch_destroy(hidem_batch *b);
const char *hidem_batch_last_error(const hidem_batch *b);
hidem_status hidem_batch_step(hidem_batch *b, int32_t nsteps);
/* the cudaStream_t the batch's work runs on */
void *hidem_batch_get_stream(hidem_batch *b);
/* kernel launches of the batch so far, graph replays, entry uploads */
hidem_status hidem_batch_counts(const hidem_batch *b, int64_t *launches, int64_t *graph_launches,
                                int64_t *uploads);

/* ---- learned warm start (settling surrogate) -------------------------- */

/* No counterpart in the reference, which settles every geometry from rest. A coordinate
 * MLP predicts the gravity/buoyancy-settled displacement of each particle from
 * `inputs` normalised inputs per particle (the caller's choice: coordinates, the
 * geometry around the particle, its lattice neighbourhood): Fourier features (u_i for
 * all i, then sin(2^f pi u_i), cos(2^f pi u_i) for f < fourier_bands, f-major, zero-padded
 * to K_0 = the next multiple of 128 of inputs * (1 + 2 fourier_bands), at least 128),
 * hidden_layers x [Linear(width) + SiLU], Linear(3). Hidden layers are BF16 tensor-core
 * GEMMs (tcgen05, FP32 accumulation) written for this library; training is MSE with Adam
 * on FP32 master weights, `batch` rows per step drawn uniformly from the training set.
 * Parameters, flat, in this order: for each hidden layer l the weight [width][K_l]
 * (K_l = width for l > 0) then the bias [width]; the output weight [3][width], the output
 * bias [3]. Inputs are [n][inputs] and targets / outputs [n][3] FP32 host arrays,
 * row-major. On failure of hidem_surrogate_create the text is in hidem_create_error(). */
typedef struct hidem_surrogate hidem_surrogate;
typedef struct hidem_surrogate_config {
    int32_t hidden_layers;   /* 1..8 (4) */
    int32_t width;           /* 128 or 256 */
    int32_t fourier_bands;   /* 1..12 */
    int32_t batch;           /* rows per training step, a multiple of 128 (16384) */
    double learning_rate;    /* Adam step size (1e-3) */
    uint64_t seed;           /* weight initialisation and batch sampling */
    int32_t inputs;          /* normalised inputs per row, 1..128 (5) */
    int32_t cosine_decay;    /* 0: constant rate; 1: each hidem_surrogate_train call
                                decays it from learning_rate to 0 along a half cosine */
} hidem_surrogate_config;
void hidem_surrogate_config_default(hidem_surrogate_config *c);
hidem_status hidem_surrogate_create(const hidem_surrogate_config *c, int device, hidem_surrogate **out);
void hidem_surrogate_destroy(hidem_surrogate *s);
const char *hidem_surrogate_last_error(const hidem_surrogate *s);
int64_t hidem_surrogate_num_params(const hidem_surrogate *s);
hidem_status hidem_surrogate_get_params(hidem_surrogate *s, float *out);
hidem_status hidem_surrogate_set_params(hidem_surrogate *s, const float *in);
/* the training set (copied to the device) */
hidem_status hidem_surrogate_set_data(hidem_surrogate *s, const float *inputs, const float *targets,
                                      int64_t n);
/* `steps` Adam steps; *loss (may be NULL) receives the last step's batch loss */
hidem_status hidem_surrogate_train(hidem_surrogate *s, int32_t steps, double *loss);
hidem_status hidem_surrogate_predict(hidem_surrogate *s, const float *inputs, int64_t n, float *out);
/* hidem_surrogate_predict for inputs and outputs already in device memory of the
 * surrogate's GPU; the work runs on the surrogate's stream (hidem_surrogate_get_stream)
 * and the call returns when it has completed. */
hidem_status hidem_surrogate_predict_device(hidem_surrogate *s, const float *inputs, int64_t n, float *out);
void *hidem_surrogate_get_stream(hidem_surrogate *s);
/* The forward pass's kernel: AUTO (default) takes PINGPONG for width 256 and BLOCK for
 * width 128. BLOCK: one CTA per 128-row block runs the block through every layer.
 * PINGPONG (width 256 only): a persistent CTA per SM takes pairs of 128-row blocks and
 * alternates them, so one block's epilogue runs while the tensor cores compute the other
 * block's layer. Both give the same hidden layers bit for bit; the 3-wide output layer's
 * FP32 sums are added in a different order (BLOCK: one sum over all 256 columns;
 * PINGPONG: four sums of 64 columns, added in column order). */
#define HIDEM_SURROGATE_FORWARD_AUTO 0
#define HIDEM_SURROGATE_FORWARD_BLOCK 1
#define HIDEM_SURROGATE_FORWARD_PINGPONG 2
hidem_status hidem_surrogate_set_forward(hidem_surrogate *s, int32_t kind);
/* loss and gradient of all parameters (flat order above) on exactly these n rows, no
 * update; n a multiple of 128 and at most `batch` */
hidem_status hidem_surrogate_gradients(hidem_surrogate *s, const float *inputs, const float *targets,
                                       int64_t n, float *grads, double *loss);

/* ---- allocation-free binning ------------------------------------------ */

/* No counterpart in the reference. For callers that cannot let a library allocate
 * device memory: applications that place every device buffer themselves (an arena or
 * pool they size up front, or a host framework whose allocator must own all device
 * memory) and loops that cannot afford the device-wide synchronisation cudaMalloc and
 * cudaFree imply. Same binning as the rebuild (hidem_regenerate): bounds of x, y, z,
 * cell colour ix + iy*X + iz*X*Y of each particle (cell_of), and `order` = particle
 * indices sorted by (cell, index). x, y, z, cell_of, order are caller-owned device
 * arrays of n elements; dims and mins are host arrays; work is queued on `stream`
 * (a cudaStream_t, 0 for the default stream). The call waits on `stream` twice: for the
 * bounds, which size the grid, and at the end for the status of the per-cell sort, so it
 * returns with cell_of and order complete. Scratch is one fixed device array in the
 * library (about 4.1 MB, held on every GPU that loads the library until exit), so grids
 * of more than HIDEM_NOALLOC_MAX_CELLS cells, and cells of more than 4096 particles,
 * are refused with HIDEM_ERR_CAPACITY. Every call looks up that array's device address
 * (cudaGetSymbolAddress) with the caller's device current. A NaN or infinite coordinate
 * is refused with HIDEM_ERR_ARG. All calls share the array: calls that overlap on the
 * GPU race. On failure the text is in hidem_create_error(). */
#define HIDEM_NOALLOC_MAX_CELLS 262144
hidem_status hidem_bin_cells_noalloc(const double *x, const double *y, const double *z,
                                     int64_t n, double cell_size, int32_t *cell_of,
                                     int32_t *order, int64_t dims[3], double mins[3],
                                     void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HIDEM_B200_H */
