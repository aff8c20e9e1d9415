// Launch wrappers of the kernels in kernels.cu (all enqueue on the given stream).
#pragma once
#include "internal.h"

namespace hidem {

constexpr int kStepThreads = 128;
constexpr int kItemThreads = 256;
constexpr size_t kItemSmemLimit = 200 * 1024;
// Byte offsets of the item kernel's shared-memory regions (same for all CTAs of a launch):
// mbarrier, own records (AoS as copied, then SoA), contact indices, the link-end streams
// partner word / CT0..CT5 / state / initial length, then the force terms.
struct StageLayout {
    size_t own, soa, nbr, spw, sct, sst, sl0, terms, total;
};
inline __host__ __device__ size_t stage_align(size_t v) { return (v + 127) & ~size_t(127); }
inline __host__ __device__ StageLayout stage_layout(size_t rec, size_t lp, int maxContacts,
                                                    int maxEnds) {
    StageLayout L;
    const size_t ends = (size_t)maxEnds * 32;
    L.own = 128;
    L.soa = stage_align(L.own + 32 * rec);
    L.nbr = stage_align(L.soa + 96 * 8 + 320 * lp + 64 * 4);
    L.spw = stage_align(L.nbr + (size_t)maxContacts * 32 * 4);
    L.sct = stage_align(L.spw + ends * 4);
    L.sst = stage_align(L.sct + 6 * ends * lp);
    L.sl0 = stage_align(L.sst + ends);
    L.terms = stage_align(L.sl0 + ends * lp);
    L.total = stage_align(L.terms + (size_t)(maxContacts * 6 + maxEnds * 12) * 32 * lp);
    return L;
}

// One set of link-end ("side") arrays in the warp-blocked ELL layout.
template <class LP>
struct SideView {
    uint32_t *partner;  // partner slot | kSideIsB
    LP *ct[6];          // CT0..CT5
    uint8_t *state;     // per-side copy of the link state
    LP *L0;             // initial length of the link
    int32_t *link;      // link index (input order)
};

// Device pointers to the caller-order particle fields (positions f64, the rest lp).
template <class LP>
struct SoaIn {
    const double *x, *y, *z;
    const LP *d[6];
    const LP *r;
    const LP *th[3];
};

template <class LP>
void launch_pack_records(const SoaIn<LP> &s, int n, PRec<LP> *rec, cudaStream_t st);
template <class LP>
void launch_unpack_records(const PRec<LP> *rec, const int *orig, int n, const SoaIn<LP> &s,
                           cudaStream_t st);
template <class LP>
void launch_unpack_force(const LP *force, const int *orig, int n, LP *out, cudaStream_t st);
// pack: buf[6k + q] = force of particle index[k] (input order), component q;
// unpack: the reverse, overwriting those forces
template <class LP>
void launch_halo_forces(LP *force, const int *slotOf, const int *index, long long m, int n, LP *buf,
                        bool pack, cudaStream_t st);
// per-particle link-end lists (ascending link index) from the link ends A, B;
// deg and cursor hold n+1 zeros on entry; sums >= (n+1)/1024 + 1 elements
void launch_link_lists(const int *A, const int *B, long long L, int n, int *deg, int *start,
                       int *cursor, int *sums, int *plLink, uint8_t *plEnd, cudaStream_t st);
void launch_side_init(const uint8_t *linkState, long long L, int *sideSlot, uint8_t *sideState,
                      cudaStream_t st);
// link ends from particle keys that are the input indices 0..n-1: A, B; the lowest link
// index with an end outside [0, n) into *badMin, with A == B into *selfMin (both start at
// the largest value)
void launch_link_keys_identity(const long long *keyA, const long long *keyB, long long L,
                               long long n, int *A, int *B, unsigned long long *badMin,
                               unsigned long long *selfMin, cudaStream_t st);
// the same from particle keys in strictly ascending order (keys: n device words): each end
// found by binary search
void launch_link_keys_sorted(const long long *keys, long long n, const long long *keyA,
                             const long long *keyB, long long L, int *A, int *B,
                             unsigned long long *badMin, unsigned long long *selfMin, cudaStream_t st);
// out[i] = i (int64 / int32)
void launch_iota64(long long *out, long long count, cudaStream_t st);
void launch_iota32(int *out, int count, cudaStream_t st);
// *out = the IEEE bits of the largest particle radius, as a double (out zeroed first)
template <class LP>
void launch_max_radius(const PRec<LP> *rec, int n, unsigned long long *out, cudaStream_t st);
template <class LP>
void launch_gather_sides(const int *sideSlot, long long L, const LP *ct, LP *out,
                         const uint8_t *sState, uint8_t *linkState, cudaStream_t st);

template <class LP>
void launch_bounds(const PRec<LP> *rec, int n, double *partial, int nb, double *out, cudaStream_t s);
template <class LP>
void launch_cells(const PRec<LP> *rec, int n, const GridInfo &g, int *cellOf, int *cellCount,
                  int *errorFlag, cudaStream_t s);
// Exclusive scan of `in` (times scaleBy) into `out`; `sums` holds ceil(n/1024) elements;
// `total` (may be null) receives the grand total. Returns the number of launches.
template <class TI, class TO>
int launch_scan(const TI *in, long long n, TO scaleBy, TO *out, TO *sums, TO *total, cudaStream_t s);
void launch_scatter(const int *cellOf, int n, const int *cellStart, int *cursor, int *perm,
                    cudaStream_t s);
// pos[s] = position of slot s in the halo send list `index` (particle indices), else -1
void launch_send_pos(const int *slotOf, const int *index, long long m, int n, int *pos, cudaStream_t s);
// out[to[i]] = in[i] for i < n (slot-order bytes into caller order)
void launch_scatter_u8(const uint8_t *in, const int *to, int n, uint8_t *out, cudaStream_t s);
// Members of a neighbour-grid cell of at most kSmallCell are sorted by one thread; larger
// cells (listed in bigList, which holds n / kSmallCell + 1 entries) by one CTA each, up to
// kBigCellCap members: a larger cell sets errorCode in errorFlag. origOld == nullptr sorts
// by the member values themselves. Returns the number of kernel launches.
constexpr int kSmallCell = 32;
constexpr int kBigCellCap = 4096;
constexpr int kBigCellThreads = 512;
int launch_sort_cells(const int *cellStart, const int *cellCount, long long total,
                      const int *origOld, int *perm, int *bigList, int *bigCount, int *errorFlag,
                      int errorCode, int smCount, cudaStream_t s);
template <class LP>
void launch_permute(const int *perm, int n, const PRec<LP> *recOld, PRec<LP> *recNew,
                    const uint8_t *typeOld, uint8_t *typeNew, const int *origOld, int *origNew,
                    const int *cellOld, int *cellNew, int *slotOf, cudaStream_t s);
template <class LP>
void launch_nbr_count(const PRec<LP> *rec, int n, const int *cellOf, const GridInfo &g,
                      const int *cellStart, const int *cellCount, double interactDist,
                      uint32_t *counts, int *blockWidth, int *errorFlag, cudaStream_t s);
template <class LP>
void launch_nbr_fill(const PRec<LP> *rec, int n, const int *cellOf, const GridInfo &g,
                     const int *cellStart, const int *cellCount, double interactDist,
                     const long long *nOff, int32_t *nbr, cudaStream_t s);
// out[0..2] = total contacts, largest contact count, largest link-end count of the
// per-slot counts (out zeroed first)
void launch_count_stats(const uint32_t *counts, int n, long long *out, int smCount, cudaStream_t st);
void launch_side_count(const int *orig, int n, const int *plStart, uint32_t *counts,
                       int *blockWidth, int *errorFlag, cudaStream_t s);
template <class LP>
void launch_side_fill(const int *orig, int n, const int *slotOf, const int *plStart,
                      const int *plLink, const uint8_t *plEnd, const int *linkA, const int *linkB,
                      const LP *L0link, const int *sideSlotOld, const SideView<LP> &oldS,
                      const long long *sOff, const SideView<LP> &newS, int *sideSlotNew,
                      cudaStream_t s);
// One timestep's forces (fused: + previous link update, integrate, record swap) for
// rows of at most maxContacts contacts and maxEnds link ends, by the kernel `kernel`
// (HIDEM_STEP_KERNEL_*, not AUTO; the item kernel falls back to one thread per particle
// for rows too wide for its shared-memory buffers).
template <class LP>
void launch_step(const Consts<LP> &c, const StepArgs<LP> &a, bool fused, int maxContacts,
                 int maxEnds, int kernel, cudaStream_t s);
// One context's share of a batched step launch (the constants other than the break
// thresholds, which travel in `a`, are the launch's). The per-step fields of `a` (in, out,
// step, breakPending, breakStep, reduceDiff) are not read: launch s of a run derives them
// from the state at its start (rec, cur0, step0, pend0) and s, the way the host loop of a
// single context sets them, so a run of launches needs no host work between steps and can
// be captured as one CUDA graph.
template <class LP>
struct BatchEntry {
    StepArgs<LP> a;
    PRec<LP> *rec[2];   // the context's two record buffers
    long long step0;    // timestep of launch 0
    int cur0;           // record buffer holding the state at launch 0
    int pend0;          // link update of step0 - 1 still to apply at launch 0
    int reduceEvery10;  // gridService reads the diff maxima every 10 steps
    // the break pass of two-pass runs: both ends' slots, side slots, initial lengths
    const int *slotA, *slotB, *sideSlot;
    const LP *L0link;
    long long L;
};
// whether rows of these widths run in the item kernel (else: per-context launches)
template <class LP>
bool batch_fits(int maxContacts, int maxEnds);
// sets the item kernel's shared-memory limit (call once before a launch is captured)
template <class LP>
void prepare_step_batch();
// particles per CTA of the batch kernel `kernel` (HIDEM_STEP_KERNEL_*, not AUTO)
int batch_particles_per_cta(int kernel);
// tbl[offs[e] .. offs[e + 1]) = e for e < count: the entry of every CTA of a batch launch
void launch_block_table(const int *offs, int count, int *tbl, cudaStream_t s);
// entries, firstBlocks (nentries + 1 CTA offsets), blockEntry (the entry of each CTA):
// device arrays; run: the launch's step within the run (each entry's step is its first
// step + run); maxContacts / maxEnds: the widest rows over all entries (shared memory of
// the item kernel)
template <class LP>
void launch_step_batch(const Consts<LP> &c, const BatchEntry<LP> *entries, const int *firstBlocks,
                       const int *blockEntry, int run, int totalBlocks, int maxContacts, int maxEnds,
                       int kernel, cudaStream_t s);

// the two-pass step over a run's entries: force pass, integrate pass (in place, with the
// diff maxima every 10 steps) over the particles' CTAs (firstBlocks, blockEntry,
// totalBlocks as for the thread kernels); break pass (when t dt > breakTime) over the links'
// CTAs (linkFirst, linkEntry, totalLinkBlocks: kStepThreads links per CTA)
template <class LP>
void launch_two_pass_batch(const Consts<LP> &c, const BatchEntry<LP> *entries, const int *firstBlocks,
                           const int *blockEntry, const int *linkFirst, const int *linkEntry, int run,
                           int totalBlocks, int totalLinkBlocks, cudaStream_t s);

template <class LP>
void launch_integrate(const Consts<LP> &c, PRec<LP> *rec, const uint8_t *type, const LP *force,
                      int n, cudaStream_t s);
template <class LP>
// endA / endB: the storage slots of every link's two ends
void launch_link_break(const Consts<LP> &c, const PRec<LP> *rec, const int *endA, const int *endB,
                       const int *sideSlot, uint8_t *sState, uint8_t *linkState, const LP *L0link,
                       long long L, long long step, int2 *events, unsigned long long *eventCount,
                       long long eventCap, cudaStream_t s);
// slotA[l] = slotOf[linkA[l]], slotB[l] = slotOf[linkB[l]]
void launch_link_slots(const int *linkA, const int *linkB, const int *slotOf, long long L, int *slotA,
                       int *slotB, cudaStream_t st);
// Kinetic energy of the particles (double precision): out[0] translational, out[1]
// rotational, out[2] largest squared speed; `partial` holds 3 * nb doubles
template <class LP>
void launch_energy(const Consts<LP> &c, const PRec<LP> *rec, int n, double *partial, int nb,
                   double *out, cudaStream_t s);
// MeshAccel grid of a collision mesh (m's grid fields set, sizes zeroed first): the count
// pass (fill false) writes sizes; the fill pass writes values at starts
template <class LP>
void launch_mesh_cells(const MeshView<LP> &m, int ntri, LP cellSize, LP maxDist, int *sizes,
                       const int *starts, int *values, bool fill, cudaStream_t s);
// The query lists of a collision mesh (m's reference lists set): per cell, the
// triangles that may lie within `reach` of the cell's box grown by `margin`, plus those
// flagged in keep; count pass (fill false) into qSizes, fill pass into qValues at qStarts
template <class LP>
void launch_mesh_prune(const MeshView<LP> &m, double cellSize, double margin, double reach,
                       const uint8_t *keep, int *qSizes, const int *qStarts, int *qValues, bool fill,
                       cudaStream_t s);
// Linear and angular momentum (about the origin) of the particles in double precision:
// out[0..2] sum m v, out[3..5] sum x (x) m v + I w; `partial` holds 6 * nb doubles
template <class LP>
void launch_momentum(const Consts<LP> &c, const PRec<LP> *rec, int n, double *partial, int nb,
                     double *out, cudaStream_t s);
template <class LP>
void launch_max_diff(const PRec<LP> *rec, int n, unsigned long long *out, int nb, cudaStream_t s);

}  // namespace hidem
