/*
 * mfcfd_internal.h - data shared by the host set-up, the kernels and the C ABI.
 */
#pragma once

#include <stdint.h>
#include <functional>
#include <new>
#include <stdexcept>
#include <string>
#include <system_error>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/mfcfd.h"

namespace mfcfd {

constexpr int MAX_CONN = 27;      // conn(27, max_points), data_structure.f90:80
constexpr int MAX_SLOTS = 32;     // distinct neighbours a point's lists may name
constexpr int LIST_STRIDE = 28;   // bytes per (point, list) entry table: <= 27 entries
constexpr int GEO_STRIDE = 48;    // doubles per point: 6 lists x 8
constexpr int NDIR = 6;           // xpos, xneg, ypos, yneg, zpos, zneg

// status 0, 1, 2 and 5/6 (supersonic inlet / outlet: not in any split list;
// the sweeps copy the increment of the nearest neighbour, the state update
// its state)
enum PointClass : int8_t { CLS_INTERIOR = 0, CLS_WALL = 1, CLS_OUTER = 2, CLS_SUPERSONIC = 3 };

// geo layout within one list's 8 doubles
enum { G_XX = 0, G_YY, G_ZZ, G_XY, G_YZ, G_ZX, G_DET, G_DNUM };

// One neighbour term of an LdelU / UdelU sum: neighbour, list (bits 0-7)
// and neighbour slot (bits 8-15), and the weighted offsets in the
// consumer's frame (dels*w, delt*w, deln*w).
struct SweepEntry {
    int32_t k;
    int32_t pad;
    double w[3];
    // leaves the fields unset, so sizing a large table does not zero it
    // first: the set-up writes every entry
    SweepEntry() {}
};

constexpr int SWEEP_MAX_ENTRIES = 96;   // per point and direction (checked at set-up)

// Everything the set-up derives from the cloud (host copy).
struct Topology {
    int n = 0;
    int cap = 22;
    std::vector<int8_t> cls;
    // split lists exactly as stored by the reference (1-based ids, flat
    // column-major with leading dimension cap, plus a tail pad)
    std::vector<int32_t> split[NDIR];
    std::vector<int32_t> split_cnt[NDIR];
    int split_overflows = 0;
    std::vector<int32_t> alias;             // 1-based values, 0 = none
    std::vector<int32_t> point_with_alias;  // 1-based ids, 0 = none
    // effective lists: the entries each flux / D_inv / sweep routine reads
    std::vector<int32_t> slot_nbr;          // n*MAX_SLOTS, 0-based, -1 unused
    std::vector<uint8_t> nslot;
    std::vector<uint8_t> slot_mask;         // n*MAX_SLOTS, bit d: slot in list d
    std::vector<uint8_t> list_cnt;          // n*6
    std::vector<uint8_t> list_ent;          // n*6*LIST_STRIDE slot indices
    std::vector<double> geo;                // n*GEO_STRIDE
    std::vector<double> eps2;               // (VL*min_dist)^3 squared
    // least-squares weights 1/dist**power when power != 0 (else empty):
    // per conn entry (q-derivatives, xyz distance) and per neighbour slot
    // (fluxes, distance in the point's frame)
    std::vector<double> wq, wf;
    // sweep schedules (0-based ids)
    std::vector<int32_t> fwd_level, bwd_level;   // per point, -1 if not swept
    std::vector<int32_t> fwd_lvl_ptr, fwd_lvl_pts, bwd_lvl_ptr, bwd_lvl_pts;
    std::vector<int32_t> fwd_off, bwd_off;        // n+1 entry offsets
    std::vector<uint8_t> fwd_cnt, bwd_cnt;        // n*6
    std::vector<SweepEntry> fwd_ent, bwd_ent;
    std::vector<uint32_t> fwd_need, bwd_need;     // slots with terms in the sweep
    std::vector<uint32_t> fwd_old, bwd_old;       // slots read from before the sweep (backup driver)
    std::vector<uint8_t> sweep_slot_mask;         // n*MAX_SLOTS: lists of the sweep terms per slot
    std::vector<double> outer_delt;               // backup driver: D_inv_outer's 1/delt operand, NaN: time step
    int sweep_variant = 0;
    std::vector<uint8_t> swept;                   // 1 if the sweeps update the point
    std::vector<uint8_t> consumer_shared;         // 1: reads published flux increments
    int shared_frame = 0;
    double frame0[9] = {0};
    int max_level_width = 0;
    std::vector<int32_t> wall_idx, outer_idx, interior_idx;   // 0-based, index order
    std::vector<int32_t> ss_inlet_idx, ss_outlet_idx;          // status 5, 6
    // supersonic points: the sweeps' copy source (nearest neighbour, -1 if
    // none within 1e6) per point, and the state update's copies in the
    // reference's order (outlets, then inlets) with their sources (nearest
    // non-wall neighbour, -1 if none within 1e5)
    std::vector<int32_t> copy_src;
    std::vector<int32_t> ss_pts, ss_src;
    // swept points outside the shared frame (walls; outer points under the
    // backup driver) whose phase-A neighbour fluxes the chain schedule takes
    // from a kernel run before the sweeps; empty when they are more than an
    // eighth of the cloud (the table would cost more memory than it saves)
    std::vector<int32_t> g0_pts;
    // storage permutation (empty: storage is the reference's index order):
    // perm[logical] = storage index, inv[storage] = logical index.  The split
    // lists, alias and point_with_alias keep logical ids; everything else
    // above is in storage order once permute_topology has run.
    std::vector<int32_t> perm, inv;
};

// One point of a sweep as a warp of the chain schedule reads it: the point,
// the offset of its terms, the term count of each list (5 bits per list) and
// CI_* bits.  All of a point's staged inputs are addressed from this record.
struct ChainItem {
    int32_t p;
    int32_t off;
    uint32_t cnt;
    uint32_t info;
};
enum : uint32_t {
    CI_WALL = 1,      // wall point (LdelU counts its lists twice, zpos skipped)
    CI_SHARED = 2,    // consumer in the shared frame (reads published increments)
    CI_PUBLISH = 4,   // some consumer reads this point's increment from global memory
    CI_COPY = 8,      // supersonic point: copies its nearest neighbour's increment
    CI_OUTER = 16,    // outer point (backup driver): octant lists, z+ over conn, own D_inv
    CI_G0 = 32,       // the neighbour fluxes of phase A were computed before the sweep
                      // (k_g0), at block info >> CI_G0_SHIFT of DevCloud::g0
};
constexpr int CI_G0_SHIFT = 8;
// Doubles per point of DevCloud::g0: the sweep's T layout, (list * MAX_SLOTS +
// slot) * 5 + component.
constexpr int G0_DOUBLES = NDIR * MAX_SLOTS * 5;
// Bits the chain schedule adds to SweepEntry::pad (bits 0-15: list, slot).
constexpr int32_t ENT_RING = 1 << 17;   // producer's increment is in the warp's ring
constexpr int ENT_RING_SHIFT = 18;      // ring slot (4 bits)
constexpr int32_t ENT_CHAIN_BITS = 0xff << 16;
// The single entry of a supersonic point: k = the copy source (-1: none).
// With ENT_COPY_NEW the source is updated earlier in the same sweep (a
// dependency); without it the copy reads the source's increment from before
// the sweep (the previous iteration's delUn).
constexpr int32_t ENT_COPY = 1 << 24;
constexpr int32_t ENT_COPY_NEW = 1 << 25;
// Backup driver: the producer comes later in the sweep's order, so the term
// uses its increment from before the sweep (published in dg_old / dU_old).
constexpr int32_t ENT_OLD = 1 << 26;
inline bool entry_is_dependency(const SweepEntry &e) {
    if (e.pad & ENT_OLD) return false;
    return !(e.pad & ENT_COPY) || (e.pad & ENT_COPY_NEW);
}
constexpr int CHAIN_RING = 8;           // increments a warp keeps in shared memory
// Published flux increments: per point 6 lists x (5 components + 1 pad), so
// every list's record starts on a 16-byte boundary (cp.async.cg copies).
constexpr int DG_STRIDE = 36;
constexpr int DG_LIST = 6;

// Static warp assignment of the sweep points for the chain schedule: warp
// lists (CSR, each in topological order), the owner warp of every point and
// the per-point records, per direction.  A point goes to the warp that just
// processed its deepest dependency when that warp is free to continue, so
// critical chains stay inside one warp; otherwise to the warp idle the
// longest.  The builder also marks each term of T's entry lists with where
// its producer's increment comes from (ENT_* bits).
struct ChainSchedule {
    int warps = 0;
    std::vector<int32_t> ptr[2], pts[2], owner[2];
    std::vector<ChainItem> items[2];
    int64_t terms_ring = 0, terms_local = 0, terms_cross = 0;   // swept producers
};
void build_chain_schedule(Topology &T, int warps, ChainSchedule &S);
// The warp assignment of one direction: the points of lpts (level-major),
// their levels, and each point's deepest-level dependencies cand[coff[p] ..
// coff[p+1]) in entry order; gives every point's owner warp and each warp's
// points in order.
void chain_assign(const int32_t *lpts, int nsw, const int32_t *level, const int32_t *coff, const int32_t *cand, int n,
                  int warps, std::vector<int32_t> &owner, std::vector<std::vector<int32_t>> &lists);

// Set-up passes on the GPU (mfcfd_prep.cu), equal to the host's.  The split
// pass leaves T untouched and sets *overflow when a list exceeds `cap`
// (the caller then stores the lists on the host, in the reference's order).
int prep_split_gpu(int device, int n, int cap, const std::vector<int8_t> &cls, const double *x, const double *y,
                   const double *z, const double *tan1, const double *tan2, const double *nor, const int32_t *nbhs,
                   const int32_t *conn, Topology &T, bool *overflow, std::string &err);
int prep_alias_gpu(int device, int n, const int32_t *nbhs, const int32_t *conn, std::vector<int32_t> &alias,
                   std::vector<int32_t> &pwa, std::string &err);
// level[p] of every point of `order` from its dependencies deps[doff[p] ..
// doff[p+1]) (0-based ids); other points get -1.
int prep_levels_gpu(int device, int n, const std::vector<int> &order, const std::vector<int32_t> &doff,
                    const std::vector<int32_t> &deps, std::vector<int32_t> &level, std::string &err);
void build_pre_order(const Topology &T, std::vector<int32_t> &order);

// Device-resident set-up (mfcfd_prep.cu; mfcfd_params.gpu_setup = 1 on a
// handle created with its device).  Every topology array the kernels read
// is computed on the device, in storage order, from the cloud uploaded once,
// with the host path's values (the same operations in the same order); the
// host classifies and orders the points, evaluates the limiter's eps2 (the
// C library's pow) and assigns the chain schedule's warps from a few arrays
// per point.  device_setup_supported() names the configurations it covers;
// the others take the host set-up.
struct DevCloud;
using DevAlloc = std::function<int(void **ptr, size_t bytes)>;
struct DevTopology {
    // kept on the device for the queries (stencils, alias, levels)
    int32_t *split[NDIR] = {};     // the reference's storage: cap*n + 64 per list, logical ids and columns
    int32_t *split_cnt = nullptr;  // NDIR*n, logical
    int32_t *alias = nullptr;      // n, logical, 1-based values
    int32_t *pwa = nullptr;        // n, 1-based logical ids, 0: none
    int32_t *level[2] = {};        // n, storage order, -1: not swept
    // host copies: level pointers (info), and what the chain schedule's warp
    // assignment reads (levels, level-major points, deepest dependencies)
    std::vector<int32_t> lvl_ptr[2];
    std::vector<int32_t> h_level[2], h_lpts[2], h_coff[2], h_cand[2];
    std::vector<int32_t> g0_pts;
    int64_t split_overflows = 0;
    int64_t n_ent[2] = {0, 0};    // sweep terms per direction
    int max_width = 0;
};
bool device_setup_supported(const mfcfd_params &P, const Topology &T);
// T: classify_points' result; T.perm / T.inv receive the storage order
// (morton_order's, computed on the device; empty for MFCFD_ORDER_INDEX);
// eps2 in the reference's index order.  Fills d's topology pointers and
// counts and dt; every allocation goes through `alloc` (owned by the
// caller, also on failure).
int device_setup(int device, const mfcfd_params &P, Topology &T, const double *x, const double *y,
                 const double *z, const double *tan1, const double *tan2, const double *nor, const int32_t *nbhs,
                 const int32_t *conn, const std::vector<double> &eps2, cudaStream_t s, const DevAlloc &alloc,
                 DevCloud &d, DevTopology &dt, std::string &err);
// The chain schedule of a device set-up for `warps` warps: d.ch_* (allocated
// through alloc; the caller frees the previous ones), the entries' chain
// bits re-marked on the device; terms[3] as ChainSchedule::terms_*.
int device_chain_schedule(int device, DevTopology &dt, DevCloud &d, int warps, cudaStream_t s,
                          const DevAlloc &alloc, int64_t terms[3], std::string &err);
// Storage order along a Morton (Z-order) curve of the coordinates, quantised
// to 21 bits per axis over the cloud's bounding box; points with the same
// key keep their index order.  perm[logical] = storage index.
void morton_order(int n, const double *x, const double *y, const double *z, std::vector<int32_t> &perm);
// Relabel the set-up from logical to storage order: every per-point array
// is moved to its point's storage index and every point id is mapped, with
// all orders (levels, index lists, supersonic copies, the residual's wall
// then interior order) kept as they were.  Results do not change: each
// point's arithmetic reads the same values in the same order.
void permute_topology(Topology &T, const std::vector<int32_t> &perm);

// Host threads for the set-up passes, one pool for every set-up running in
// the process at once (the host's cores less two).  take_setup_threads
// grants up to `want` (possibly 0); give_setup_threads returns them.  A
// thread that runs set-ups for others (a server worker) holds one for itself.
int take_setup_threads(int want);
void give_setup_threads(int k);

// Runs f (the body of an entry point) and turns an exception into a status,
// with the message in *err when err is not null, so that nothing is thrown
// across the C ABI.  Host memory or a host thread that cannot be had gives
// MFCFD_ERR_NOMEM.
template <class F>
int host_guard(std::string *err, F &&f) noexcept {
    int code;
    const char *msg;
    try {
        return f();
    } catch (const std::bad_alloc &) {
        code = MFCFD_ERR_NOMEM, msg = "host memory exhausted";
    } catch (const std::length_error &) {
        code = MFCFD_ERR_NOMEM, msg = "host allocation too large";
    } catch (const std::system_error &) {
        code = MFCFD_ERR_NOMEM, msg = "a host thread could not be started";
    } catch (...) {
        code = MFCFD_ERR_UNSUPPORTED, msg = "unexpected host failure";
    }
    if (err) {
        try {
            *err = msg;
        } catch (...) {
        }
    }
    return code;
}

// Validation of the inputs, the point classes and the class index lists
// (T.n, T.cap, T.cls, T.*_idx); the first step of build_topology.
int classify_points(const mfcfd_params &P, int n, const int32_t *status, const int32_t *nbhs, const int32_t *conn,
                    Topology &T, std::string &err);
// The limiter's epsilon per point, (vl_const*min_dist)**3 squared
// (limiters.f90:251-253), at perm[i] (perm null: index order).
void limiter_eps2(const mfcfd_params &P, int n, const double *min_dist, const int32_t *perm, std::vector<double> &eps2);
// One split-list entry written past a list's capacity into the storage that
// follows it (list d, flat index within the list's array, 1-based id).
struct SpillWrite {
    int d;
    size_t at;
    int32_t value;
};
// The spilled writes of the reference's split storage, in its order, from
// every point's full list counts cnt[d][i] (T: classes and index lists).
void split_spill_writes(const Topology &T, const double *x, const double *y, const double *z, const double *tan1,
                        const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn,
                        const int32_t *const cnt[NDIR], std::vector<SpillWrite> &out);

// Build everything above.  Returns MFCFD_OK or an error code with a message.
int build_topology(const mfcfd_params &P, int n, const int32_t *status, const double *x,
                   const double *y, const double *z, const double *tan1, const double *tan2,
                   const double *nor, const int32_t *nbhs, const int32_t *conn,
                   const double *min_dist, Topology &T, std::string &err);

// Device-side views (plain pointers, passed to kernels by value).
struct DevCloud {
    int n;
    int shared_frame;
    double frame0[9];
    double power, cfl;
    int inner_iterations;         // second-order q-derivative passes
    int update_variant;           // MFCFD_UPDATE_*
    double rho_inf, u1_inf, u2_inf, u3_inf, pr_inf;
    // geometry
    const double *x, *y, *z;
    const double *frame;          // 9 per point: tan1, tan2, nor
    const int8_t *cls;
    const int32_t *nbhs;
    const int32_t *conn;          // 27 per point, 0-based
    const double *eps2;
    const double *wq, *wf;        // weights (power != 0), else null: weight 1
    const int32_t *slot_nbr;
    const uint8_t *nslot;
    const uint8_t *slot_mask;
    const uint8_t *list_cnt;
    const uint8_t *list_ent;
    const double *geo;
    const uint8_t *swept;
    const uint8_t *consumer_shared;
    // sweep schedules
    const int32_t *fwd_lvl_ptr, *fwd_lvl_pts, *bwd_lvl_ptr, *bwd_lvl_pts;
    int n_fwd_levels, n_bwd_levels;
    const int32_t *fwd_off, *bwd_off;
    const uint8_t *fwd_cnt, *bwd_cnt;
    const SweepEntry *fwd_ent, *bwd_ent;
    const uint32_t *fwd_need, *bwd_need;
    const uint32_t *fwd_old, *bwd_old;
    const uint8_t *sweep_slot_mask;
    const double *outer_delt;
    int sweep_variant;            // MFCFD_SWEEPS_*
    double *dg_old;               // DG_STRIDE per point: increments from before the sweep (backup)
    const int32_t *res_order;     // wall then interior ids, index order
    int n_res;
    int n_wall;                   // the first n_wall entries of res_order
    int n_swept;                  // points in each sweep order
    int max_width;                // widest sweep level
    int sweep_mode;               // MFCFD_SWEEP_*
    int precision;                // MFCFD_PRECISION_*
    int *sweep_counter;           // 2 work counters (forward, backward)
    int *err;                     // set when a bounded poll gave up
    int spin_limit;               // poll rounds before a wait gives up (0: the default)
    int withhold1;                // failure-detection hook: this point (1-based) publishes
                                  // none of its sweep increments; 0: off
    // chain schedule (per direction: 0 forward, 1 backward)
    int ch_warps, ch_wpb;         // warps and warps per block
    int ch_spread;                // one chain block per SM (mfcfd_params.chain_spread)
    int flux_grid;                // blocks of the fused flux kernel; 0: one per FLUX_WARPS points
    const int32_t *pre_order;     // all points, forward sweep order first (fused flux)
    const int32_t *ch_ptr[2], *ch_pts[2], *ch_own[2];
    const ChainItem *ch_items[2];
    const int32_t *g0_pts;        // points of the g0 blocks (Topology::g0_pts)
    double *g0;                   // G0_DOUBLES per g0 point, computed by k_g0 each iteration
    int n_g0;
    // state (Fortran layout, point-major)
    double *prim, *U, *q, *qm, *dq, *delt, *flux_res, *dUp, *dUn, *dinv;
    double *dq_tmp;               // 15 per point: inner-iteration output (or null)
    double *dU_old;               // 5 per point: delUn before the sweeps (supersonic copies)
    int n_ss;                     // supersonic points (state-update copies)
    const int32_t *ss_pts, *ss_src;
    double *gold;                 // 30 per point: fluxes of prim in frame0
    double *dgf, *dgb;            // DG_STRIDE per point: published flux increments
    double *res_sqr;              // per point (residual sum terms)
    double *partial;              // reduction scratch
    double *res_dev;              // per-iteration res_new history
};

// The clouds of one group chain-sweep launch (mfcfd_run_group), passed as
// the kernel's parameters: MFCFD_GROUP_MAX_CLOUDS views and the first block
// of each cloud (block_start[count] = the grid).
struct ChainGroup {
    int count;
    int block_start[MFCFD_GROUP_MAX_CLOUDS + 1];
    DevCloud cloud[MFCFD_GROUP_MAX_CLOUDS];
};
static_assert(sizeof(ChainGroup) <= 32000, "a group launch's parameters must stay within 32 KB");

// Streams of one handle: the main stream (high priority) and a side stream
// that runs the flux residual beside the chain schedule's forward sweep,
// with the events that fork and join them.
struct IterStreams {
    cudaStream_t main, side;
    cudaEvent_t fork, join;
};

// kernel launchers (mfcfd_kernels.cu)
// ev: null, or MFCFD_NPHASE+1 events recorded around the phases (ev[2] on
// the side stream under the chain schedule).
// part: ITER_ALL, or (chain schedule only) ITER_PRE -- every launch before
// the sweeps, the flux residual on the side stream ending in st.join, with
// st.fork recorded on the main stream where the forward sweep may start --
// and ITER_POST, the state update and residual after the backward sweep.
enum IterPart { ITER_ALL = 0, ITER_PRE = 1, ITER_POST = 2 };
cudaError_t launch_iteration(const DevCloud &d, int iter_slot, const IterStreams &st,
                             double *U_next, double *q_next, cudaEvent_t *ev, IterPart part = ITER_ALL);
// One chain sweep (forward or backward) of every cloud of g in one launch;
// all the group's clouds have chain blocks of wpb warps and one precision.
cudaError_t launch_chain_group(const ChainGroup &g, int wpb, int precision, int spread, int forward,
                               cudaStream_t s);
// Whether the group kernel of this shape keeps the single-cloud kernel's
// blocks per SM (so chain_block_slots holds for it too).
bool chain_group_fits(int device, int wpb, int precision, int spread);
cudaError_t launch_conserved_q(const DevCloud &d, cudaStream_t s);
// rows [a, a+rows) of width w: scatter from an index-order buffer to storage
// order (dst[perm[a+i]] = src[i]), or gather the reverse
cudaError_t launch_rows(const double *src, double *dst, const int32_t *perm, int a, int rows, int w, bool scatter,
                        cudaStream_t s);
// out[0..2] (device) = -sum over wall points of (p - p_inf) A nor
cudaError_t launch_forces(const DevCloud &d, cudaStream_t s, double area_each, const double *area, double *out);
int reduction_blocks(int n);
// streaming multiprocessors of a device (cached per device)
int device_sms(int device);
// Launch shape of the chain sweep for about `want` warps: warps per block
// and blocks (at most SMs - 16 blocks); returns the warps, 0 if the kernel
// cannot run on the device.
int chain_shape(int device, int want, int spread, int *wpb, int *blocks);
// Per-device launch set-up (kernel attributes), done before a stream capture.
void prepare_launches(int device);
// Chain-sweep blocks that may run at once, in slots of a sixth of an SM: a
// block takes 6 / (its blocks per SM, at most 3), i.e. 2 for a 4-warp block
// of the mixed-precision sweep (three per SM), 3 for a 4-warp block of the
// FP64 sweep, 6 for an 8-warp block; see k_sweep_chain.
int chain_slot_capacity(int device);
// slots (sixths of an SM) of one chain block of the given shape and
// precision (MFCFD_PRECISION_*)
int chain_block_slots(int device, int wpb, int precision, int spread = 0);
// File formats of the reference program (mfcfd_io.cpp).  Handle-less calls
// leave their message in g_io_err (mfcfd_last_error(NULL)).
extern thread_local std::string g_io_err;
int io_count_input_points(const char *path, int32_t *n);
int io_read_input_point_data(const char *path, int32_t n, int32_t *status, double *x, double *y,
                             double *z, double *tan1, double *tan2, double *nor, int32_t *nbhs,
                             int32_t *conn, double *min_dist);
int io_read_stored_solution(const char *path, int32_t n, double *prim);
int io_write_primal_output(const std::string &dir, int32_t n, const int32_t *status, const double *x,
                           const double *y, const double *z, const double *prim, const double *flux_res,
                           const double *dq);
int io_write_residue(const char *path, int32_t t0, int32_t iters, const double *res_hist, int append);

// k nearest neighbours (mfcfd_knn.cu): on `device` (>= 0) or the host's
// threads, the same arrays either way.
int knn_connectivity(int device, int n, const double *x, const double *y, const double *z, int k, int32_t *nbhs,
                     int32_t *conn, double *min_dist, std::string &err);

// Mixed precision: fold each sweep term's 3x3 solve into its weight (saving
// the three weights first into saved[dir], 3 per term, when non-null), or
// put the saved weights back (fold false).
cudaError_t launch_fold_terms(const DevCloud &d, double *const saved[2], bool fold, cudaStream_t s);

// Allocation-free residual (mfcfd_residual_noalloc); the current device must
// be the handle's.
int residual_noalloc(const DevCloud &d, cudaStream_t s, double *res_new, std::string &err);

}  // namespace mfcfd
