/*
 * dsx.h -- C ABI of the B200-native dsDecompX particle-bookkeeping engine.
 *
 * Plain pointers and sizes only; every pointer argument named `device` is a
 * CUDA device pointer (or managed memory), `stream` is a cudaStream_t passed
 * as void*.  Every entry point returns DSX_OK or a negative DSX_E_* code and
 * never throws; dsx_last_error() gives the message of the calling thread's
 * last failure.  Messages start with "dsDecompX:" like the reference's
 * exceptions (docs/05_API_Reference.md:432).
 *
 * Two surfaces:
 *
 *  1. The single-rank drop-in (dsx_rank_*), called by the C++ Decomp /
 *     ParticleInfo shim in include/dsdecompx.hpp.  It operates in place on the
 *     caller's device SoA arrays, exactly where the reference's
 *     ExecutionMode::Cuda calls its src/cuda launch_* kernels on one rank.
 *
 *  2. The virtual grid (dsx_grid_*): P subdomains of one box held on one GPU,
 *     the multi-rank behaviour of the reference (one MPI rank per subdomain)
 *     with every neighbor "send" turned into a write into the receiver's
 *     slots.  Each call is the batched counterpart of the reference's
 *     collective call on all ranks at once.
 *
 * Array ids (dsx_grid_read / dsx_grid_write): 0..10 x y z vx vy vz fx fy fz
 * mass charge (double), 11 type, 12 global_id (int32), 13+f registered field f.
 */
#ifndef DSX_H
#define DSX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSX_OK 0
#define DSX_E_INVALID (-1)     /* std::invalid_argument in the reference */
#define DSX_E_LOGIC (-2)       /* std::logic_error */
#define DSX_E_RUNTIME (-3)     /* std::runtime_error (CUDA failure) */
#define DSX_E_LENGTH (-4)      /* std::length_error (capacity) */
#define DSX_E_OVERFLOW (-5)    /* ghost capacity exceeded; call grew it, retry */

/* dsdecompx::FieldType (include/field.hpp:22-29) */
enum { DSX_INT32 = 0, DSX_INT64 = 1, DSX_UINT32 = 2, DSX_UINT64 = 3,
       DSX_FLOAT32 = 4, DSX_FLOAT64 = 5 };
/* dsdecompx::ReduceOp (include/field.hpp:31-36) */
enum { DSX_SUM = 0, DSX_MIN = 1, DSX_MAX = 2, DSX_REPLACE = 3 };
/* dsdecompx::GridPolicy (include/grid.hpp:26-33) */
enum { DSX_MANUAL = 0, DSX_BALANCED = 1, DSX_TOPOLOGY_AWARE = 2, DSX_DYNAMIC = 3 };

const char* dsx_last_error(void);
const char* dsx_version(void);

/* ------------------------------------------------------------------------
 * 1. Single-rank drop-in
 * ---------------------------------------------------------------------- */

/* Periodic box of the rank (dsdecompx::GlobalDomain, include/domain.hpp:7-11). */
typedef struct dsx_domain {
    double lower[3];
    double upper[3];
    int periodic[3];
} dsx_domain;

/* dsdecompx::MigrationResult (include/config.hpp:42-49) */
typedef struct dsx_migration_result {
    int ownership_changed;
    long long previous_owned_count;
    long long retained_count;
    long long sent_count;
    long long received_count;
    long long new_owned_count;
} dsx_migration_result;

/* Replaces the 1-rank branch of Decomposition::migrate_particles
 * (src/migration.cpp:147-389 with rank_count == 1, launch_classify_destinations
 * src/cuda/classify.cu:46-63 + launch_build_migration_layout
 * src/cuda/migration_layout.cu:48-110 + unpack src/cuda/unpack.cu:61-71):
 * every owned particle stays in its slot and gets the Host-path periodic wrap
 * of its position.  x, y, z: device arrays of `owned` doubles. */
int dsx_rank_migrate(double* x, double* y, double* z, long long owned,
                     const dsx_domain* domain, void* stream,
                     dsx_migration_result* result);

/* ------------------------------------------------------------------------
 * 2. Virtual grid of P subdomains on one GPU
 * ---------------------------------------------------------------------- */

typedef struct dsx_grid dsx_grid;

/* dsdecompx::Config (include/config.hpp:20-40) for P virtual ranks. */
typedef struct dsx_grid_desc {
    int nranks;               /* P, 1..1024 */
    int dims[3];              /* Manual policy; 0 entries are filled like MPI_Dims_create */
    int policy;               /* DSX_MANUAL .. DSX_DYNAMIC */
    double lower[3], upper[3];
    int periodic[3];
    double halo_width;
    int edges_and_corners;    /* HaloConfig::include_edges_and_corners */
    double dyn_interval;      /* DynamicLoadBalanceConfig (defaults 1, 1.10, 0.5, 0.10) */
    double dyn_threshold;
    double dyn_relaxation;
    double dyn_min_fraction;
} dsx_grid_desc;

typedef struct dsx_field_desc {
    const char* name;
    int type;                 /* DSX_INT32 .. DSX_FLOAT64 */
    int components;
} dsx_field_desc;

/* Host only (no GPU needed): the process grid dims[3] and the neighbor list
 * of rank `rank` that a grid created from `desc` uses, in the format of
 * dsx_grid_neighbors.  Mirrors initialize_topology + refresh_domain_geometry
 * (src/topology.cpp:18-176) and choose_process_grid (src/grid.cpp:79-122). */
int dsx_plan_topology(const dsx_grid_desc* desc, int rank, int* dims, int* count,
                      int* info, double* shifts);

/* Creates the grid with room for `particles` owned particles in total (the
 * count migration conserves) and `ghost_capacity` ghosts (0: estimated; grown
 * on overflow). */
int dsx_grid_create(const dsx_grid_desc* desc, const dsx_field_desc* fields,
                    int nfields, long long particles, long long ghost_capacity,
                    dsx_grid** out);
int dsx_grid_destroy(dsx_grid* grid);

/* Topology as the reference's Topology reports it for rank `rank`
 * (include/topology.hpp:19-41): dims[3], coords[3], local {lower[3], upper[3]};
 * neighbors: count and per entry {rank, dx, dy, dz, slot} + shift[3]. */
int dsx_grid_topology(dsx_grid* grid, int rank, int* dims, int* coords, double* local);
int dsx_grid_neighbors(dsx_grid* grid, int rank, int* count, int* info, double* shifts);
/* Current axis cuts, axis by axis (dims[a]+1 each); synchronizes `stream`. */
int dsx_grid_cuts(dsx_grid* grid, double* out, void* stream);

/* Owned particles of every subdomain, host arrays concatenated in rank order
 * with counts[P] (sum == particles).  arrays[13 + nfields]: core arrays in
 * array-id order, then fields; null core arrays are zero-filled.
 * Replaces the state (no ghosts). */
int dsx_grid_upload(dsx_grid* grid, const long long* counts,
                    const void* const* arrays, void* stream);

/* Inverse of dsx_grid_upload: counts[P] and the owned particles of every
 * subdomain, concatenated in rank order, into host (or device) arrays of at
 * least `particles` entries; null entries are skipped.  Synchronizes. */
int dsx_grid_download(dsx_grid* grid, long long* counts, void* const* arrays, void* stream);

/* Totals of the last migrate / halo build: {owned particles, emigrants,
 * ghosts, boundary owners}; synchronizes `stream`. */
int dsx_grid_totals(dsx_grid* grid, long long* out4, void* stream);

/* Counts per subdomain (owned, ghosts); synchronizes `stream`. */
int dsx_grid_counts(dsx_grid* grid, long long* owned, long long* ghosts, void* stream);

/* Host copy of `count` entries of array `array` of subdomain `rank` starting
 * at local slot `start` (owned slots first, then ghosts, as one rank's
 * ParticleInfo holds them).  Synchronizes `stream`. */
int dsx_grid_read(dsx_grid* grid, int rank, int array, long long start,
                  long long count, void* host_out, void* stream);
int dsx_grid_write(dsx_grid* grid, int rank, int array, long long start,
                   long long count, const void* host_in, void* stream);

/* Device pointers of the current storage.  base[13 + nfields]: start of each
 * array; owned particles of subdomain s are [owned_offset + obase[s], +n[s])
 * and its ghosts [ghost_offset + gbase[s], +g[s]).  The pointers change after
 * a migrate (the owned half flips) and after a capacity growth: re-read them
 * after every call, as the reference asks of ParticleInfo users
 * (docs/04_Using_in_Your_Code.md:357-358).  obase/gbase/n/g: device arrays. */
typedef struct dsx_grid_view {
    void* base[32];
    long long owned_offset;
    long long ghost_offset;
    const int* n;             /* [P]   owned per subdomain (device) */
    const int* obase;         /* [P+1] */
    const int* g;             /* [P]   ghosts per receiver (device) */
    const int* gbase;         /* [P+1] */
    const int* halo_totals;   /* {ghosts, boundary owners} (device) */
    long long particles;      /* total owned (host) */
    long long ghost_capacity; /* host */
    int nranks;
} dsx_grid_view;
int dsx_grid_view_get(dsx_grid* grid, dsx_grid_view* out);

/* Decomp::migrate on all P ranks (src/runtime.cpp:983-1019), including the
 * automatic Dynamic rebalance.  results: null, or P x {changed, previous,
 * retained, sent, received, new_owned} (synchronizes). */
int dsx_grid_migrate(dsx_grid* grid, void* stream, long long* results);

/* Decomp::exchange_halo on all ranks (src/runtime.cpp:862-981).  Rebuilds the
 * plan when rebuild != 0 or no valid plan exists, else refreshes it in place
 * (positions_only: x, y, z only).  results: null, or P x {ghost_count,
 * layout_changed, storage_reallocated, plan_reused} (synchronizes; a ghost
 * overflow is then detected, the capacity grown and the build redone). */
int dsx_grid_exchange_halo(dsx_grid* grid, int rebuild, int positions_only,
                           void* stream, long long* results);

/* Decomp::reverse_halo (src/halo.cpp:1288-1347): owner forces += ghost forces,
 * images summed in neighbor order (bit-identical to the Host path). */
int dsx_grid_reverse_halo(dsx_grid* grid, void* stream);

/* Decomp::reverse_exchange / forward_exchange (src/halo.cpp:1210-1286,
 * 1396-1532) on registered fields (indices into the create-time list). */
int dsx_grid_reverse_exchange(dsx_grid* grid, int nfields, const int* field_ids,
                              const int* ops, void* stream);
int dsx_grid_forward_exchange(dsx_grid* grid, int nfields, const int* field_ids,
                              void* stream);

/* Decomp::rebalance (src/runtime.cpp:1021-1041): work (host, P entries) or
 * null for owned counts; then migrate.  results: P x {attempted, changed,
 * new_owned} (synchronizes). */
int dsx_grid_rebalance(dsx_grid* grid, const double* work, int force, void* stream,
                       long long* results, double* imbalance);

int dsx_grid_set_halo_width(dsx_grid* grid, double width);
int dsx_grid_invalidate_halo(dsx_grid* grid);

/* Adjoint of the ghost position copy: owner_grad[i] += sum over the ghost
 * images of i of ghost_cot[slot], in the same deterministic order as
 * reverse_halo.  Arrays are device SoA: ghost_cot_{x,y,z} indexed by ghost
 * slot (0..ghosts-1, the grid's ghost order), owner_grad_{x,y,z} by owned
 * index (0..particles-1 of the current owned half). */
int dsx_grid_halo_backward(dsx_grid* grid, const double* ghost_cot_x,
                           const double* ghost_cot_y, const double* ghost_cot_z,
                           double* owner_grad_x, double* owner_grad_y,
                           double* owner_grad_z, void* stream);

/* Batched step: migrate -> halo build -> callback(user, stream, view) ->
 * reverse_halo.  capture != 0 captures the step in CUDA graphs (one per owned
 * half) on first use and replays them; the callback must then only enqueue
 * work on `stream` that reads counts from the view's device arrays.  The
 * callback must be idempotent: a step whose ghost build overflowed is redone
 * after the capacity grows.  Capture needs a created stream (not the default
 * stream; DSX_E_INVALID).  status (optional) gets the step's device status
 * bits (0 == ok). */
typedef void (*dsx_step_callback)(void* user, void* stream, const dsx_grid_view* view);
int dsx_grid_step(dsx_grid* grid, dsx_step_callback callback, void* user, int capture,
                  void* stream, unsigned* status);

/* Batched steps queued back to back (no counterpart call in the reference,
 * whose ranks finish each call before the next): the step's graph (captured
 * as dsx_grid_step with capture != 0 does, same callback contract) is queued
 * on `stream` and the call returns.  The previous asynchronous step is checked
 * first, at the end of its halo build (its callback and reverse sum may still
 * be running), so the GPU is never left without the next step; an overflowed
 * ghost region is grown and that step's build, callback and reverse sum are
 * redone there, before anything builds on it (so the callback must be
 * idempotent, as for dsx_grid_step).  dsx_grid_step_wait completes the
 * pending step and returns the OR of the status bits of the asynchronous
 * steps since the last wait; every other dsx_grid_* call on the grid (but
 * dsx_grid_view_get, dsx_grid_step_kernel_count and the topology queries)
 * completes the pending step first, and so reports its failure.  Needs a created stream (DSX_E_INVALID
 * for a default stream). */
int dsx_grid_step_async(dsx_grid* grid, dsx_step_callback callback, void* user, void* stream);
int dsx_grid_step_wait(dsx_grid* grid, unsigned* status);

/* Split-phase halo exchange (Decomp::begin_halo_exchange /
 * end_halo_exchange, dsDecompX src/halo.cpp:296-872): begin enqueues the
 * refresh along the plan or the plan build on stream and returns at once, so
 * interior work can run on other streams; end waits for it (growing the ghost
 * region and rebuilding if it overflowed) and fills results like
 * dsx_grid_exchange_halo.  Between the two, every other operation on the
 * grid fails with DSX_E_LOGIC, as does end without begin or a second begin.
 * On an explicit (non-default) stream the two halves are captured CUDA graphs,
 * one launch each: begin's segment is the refresh or the build, end's the
 * completion (the build's status and totals to the host). */
int dsx_grid_begin_halo_exchange(dsx_grid* grid, int rebuild, int positions_only, void* stream);
int dsx_grid_end_halo_exchange(dsx_grid* grid, void* stream, long long* results);

/* How a halo refresh (exchange_halo along a valid plan, full or positions
 * only) walks the plan: 0 ghost by ghost, gathering the owner of every
 * ghost; 1 owner by owner, reading each boundary owner once and writing all
 * its images; 2 tile by tile, the tile's owners brought into shared memory
 * whole and the images written in ghost-slot order (a record whose copied
 * arrays exceed 100 KB per tile falls back to 0); 3 (the default) 2 for a
 * full refresh that copies nine arrays or more (positions, velocities and
 * at least three fields), else 0.  All write the same values; DSX_E_INVALID
 * for another kind. */
int dsx_grid_set_refresh_kind(dsx_grid* grid, int kind);

/* CTAs per SM that begin_halo_exchange's refresh may occupy (0, the default:
 * every resident CTA).  A small number leaves room on every SM for interior
 * work launched on other streams between begin and end. */
int dsx_grid_set_split_share(dsx_grid* grid, int ctas_per_sm);

/* Owning subdomain of n positions (Decomposition::owner_rank, dsDecompX
 * src/migration.cpp:74-98: one periodic wrap, then the cut planes): x, y, z
 * and out are device arrays of n; enqueued on stream. */
int dsx_grid_owner_rank(dsx_grid* grid, const double* x, const double* y, const double* z,
                        long long n, int* out, void* stream);

/* Decomp::has_out_of_domain_particles (dsDecompX src/runtime.cpp:828-840)
 * for every subdomain: flags (optional, host, P ints) gets 1 where an owned
 * particle belongs to another subdomain, any (optional) their OR -- the
 * reference's all-rank answer.  Synchronizes stream. */
int dsx_grid_out_of_domain(dsx_grid* grid, int* flags, int* any, void* stream);

/* Cut planes (Decomposition::set_axis_cuts, dsDecompX src/decomp.cpp:146-163):
 * cuts holds axis 0, 1, 2 concatenated, dims[a] + 1 values each, as
 * dsx_grid_cuts returns them; they must span the domain and increase
 * strictly (DSX_E_INVALID otherwise).  The halo plan becomes invalid. */
int dsx_grid_set_cuts(dsx_grid* grid, const double* cuts, void* stream);

/* New box (Decomp::rescale_domain and update_domain, dsDecompX
 * src/decomp.cpp:104-144, src/runtime.cpp:843-849): every cut plane keeps
 * its fraction of the extent and the periodic shifts follow the new extent.
 * invalidate_plan == 0 (rescale_domain) keeps the halo plan, so a refreshing
 * exchange_halo moves the ghosts with the new shifts; != 0 (update_domain)
 * invalidates it.  Periodicity cannot change; particle positions are the
 * caller's to rescale. */
int dsx_grid_rescale_domain(dsx_grid* grid, const double* lower, const double* upper,
                            int invalidate_plan, void* stream);

/* Autotuning of the batched step's launch shapes on the grid's current
 * particles: times each candidate by replaying the step's idempotent parts
 * (nothing of the current owned half changes) and keeps the fastest --
 * the classify pass's threads per 512-particle tile (64, 128, 256), the move
 * with its tile records staged in shared memory by bulk copies (in one pass
 * of up to 100 KB per tile, or in passes of at most 56 KB) or read directly, the
 * reverse sum's CTAs per SM (4, 8, 16, 32) -- and sizes the
 * ghost region to at least 1.25x the ghosts of the current particles (the
 * per-neighbour send lists are slices of it).  Afterwards the halo plan is
 * invalid (call exchange_halo or step next) and captured steps are
 * re-captured.  report (optional) gets the choices and the measured times
 * (milliseconds per launch; -1 where a candidate does not apply).  A grid of
 * one subdomain has nothing to tune and keeps the defaults. */
typedef struct dsx_tune_report {
    int classify_threads;
    int move_staged;         /* move kind: 1 staged (one pass if it fits), 2 staged in passes,
                                3 staged without the force arrays, 0 direct reads */
    int reverse_ctas_per_sm;
    long long ghost_capacity;
    float classify_ms[3];    /* 64, 128, 256 threads per tile */
    float move_ms[4];        /* staged, direct reads, staged in passes, staged without forces */
    float reverse_ms[4];     /* 4, 8, 16, 32 CTAs per SM */
    int classify_combine;    /* 1: a warp's immigrant counters combined per destination
                                before one atomic each (pays when many emigrants share
                                few destinations) */
    float classify_combined_ms[3];   /* the combined form at 64, 128, 256 threads */
} dsx_tune_report;
int dsx_grid_autotune(dsx_grid* grid, void* stream, dsx_tune_report* report);

/* Sets the batched step's launch shapes directly (as dsx_grid_autotune would
 * choose them; for re-using a tuning, and for tests that force each kind):
 * classify_threads 64, 128 or 256; move_kind as dsx_tune_report.move_staged
 * (a kind that does not fit the record's shared-memory budget falls back to
 * staged passes or direct reads); reverse_ctas_per_sm 0 (two waves of the
 * grid's SMs) or 1..32; classify_combine as dsx_tune_report.classify_combine.
 * Results are identical for every setting. */
int dsx_grid_set_tuning(dsx_grid* grid, int classify_threads, int move_kind,
                        int reverse_ctas_per_sm, int classify_combine);

/* ---- sharded grids: the P subdomains split over several processes ----
 *
 * Each process keeps a grid of all P subdomains that holds particles only in
 * the subdomains it owns.  After a local migrate or halo build the particles
 * and ghost lists that belong to another process's subdomains are sent there,
 * and each process assembles its subdomains in the reference's order
 * (retained, then immigrants by source rank; ghosts by the receiver's
 * neighbor blocks).  These calls are the local pieces of that exchange. */

/* Emigrants of the last migration (dsx_grid_migrate, dsx_grid_rebalance or a
 * batched step) per (destination, source): pairs[t * P + q] (synchronizes).
 * DSX_E_LOGIC when the particles were replaced since (upload, assemble). */
int dsx_grid_migration_pairs(dsx_grid* grid, long long* pairs, void* stream);

/* The current plan's send lists, 26 per sender (entry q * 26 + n: sender q's
 * list toward its neighbor n): length and first ghost slot (relative to the
 * view's ghost_offset).  All zero without a plan (synchronizes). */
int dsx_grid_send_lists(dsx_grid* grid, int* length, int* first_slot, void* stream);

/* One copy of `count` records of every particle array into the next owned
 * layout: from source `source` (-1: the grid's current owned particles, index
 * src_index in the view's owned numbering; k >= 0: outside buffer k) to
 * subdomain dst_rank at position dst_index. */
typedef struct dsx_segment {
    int source;
    long long src_index;
    int dst_rank;
    long long dst_index;
    long long count;
} dsx_segment;

/* Replaces the owned particles: counts[P] are the new per-subdomain counts,
 * sources[32 * k + a] the address of element 0 of array a (dsx_grid_view
 * order: 13 core arrays, then the fields) in outside buffer k (device
 * memory), segments fill the new layout (positions not covered are left
 * undefined).  The halo plan becomes invalid (synchronizes). */
int dsx_grid_assemble(dsx_grid* grid, const long long* counts, int nsources,
                      const void* const* sources, long long nsegments, const dsx_segment* segments,
                      void* stream);

/* Work per subdomain (P values) for the automatic Dynamic rebalance of the
 * next dsx_grid_migrate, instead of this grid's owned counts (a sharded grid
 * passes the counts of all processes); null clears it. */
int dsx_grid_set_rebalance_work(dsx_grid* grid, const double* work);

/* Device-to-device copies, all in one kernel on `stream` (stream ordered;
 * the list itself may be reused when the call returns). */
typedef struct dsx_copy {
    const void* src;
    void* dst;
    long long bytes;
} dsx_copy;
int dsx_copy_segments(const dsx_copy* copies, long long n, void* stream);

/* Plain launches, for comparison runs: plain != 0 makes the per-call
 * operations (dsx_grid_migrate, a rebuilding dsx_grid_exchange_halo,
 * dsx_grid_reverse_halo) launch each of their tile kernels once per subdomain
 * over that subdomain's tiles, reading the layout to the host first -- the
 * launch pattern of one process per subdomain, as the reference runs P ranks.
 * Results are identical to the default (one launch per phase for all
 * subdomains); dsx_grid_step is not affected. */
int dsx_grid_set_plain(dsx_grid* grid, int plain);

/* Per-kernel timing of the batched step, for benchmarks: enable != 0 makes
 * the next steps record a CUDA event after every kernel (inside a captured
 * graph they are event-record nodes; captured graphs are rebuilt when the
 * setting changes).  dsx_grid_kernel_times fills names/ms (milliseconds) for
 * the intervals of the last step, in launch order, and returns how many. */
int dsx_grid_profile(dsx_grid* grid, int enable);
int dsx_grid_kernel_times(dsx_grid* grid, int max, const char** names, float* ms);

/* Number of this library's kernel launches in one batched step (for reports). */
int dsx_grid_step_kernel_count(dsx_grid* grid);

/* ------------------------------------------------------------------------
 * Allocation-free migrate.  No counterpart in the reference (its migrate grows
 * device buffers with cudaMalloc as needed).
 *
 * For callers that cannot allocate device memory: a solver whose framework
 * owns all GPU memory through its own pool, a latency-critical loop where an
 * allocation's implicit device synchronization is not acceptable, or a plugin
 * that must not change the process's memory footprint.  Such a caller cannot
 * create a dsx_grid (which allocates its storage); this call migrates the
 * caller's own arrays instead: the owned particles of `desc->nranks`
 * subdomains, concatenated in rank order (counts_in[P] on the host; arrays_in
 * and arrays_out: the 13 core device arrays in array-id order, no registered
 * fields), into arrays_out in the migrated order -- the same result as
 * dsx_grid_migrate on the same grid, cuts and particles.  cuts: host array of
 * the axis cuts (dims[a]+1 per axis) or null for uniform cuts; desc->dims must
 * be explicit; there is no automatic Dynamic rebalance.  counts_out[P] and
 * results (null or P x 6, as dsx_grid_migrate) are host arrays; the call
 * synchronizes `stream`.
 *
 * Limits: at most 64 subdomains and 262144 particles (DSX_E_LENGTH beyond).
 * Input and output arrays must not overlap (DSX_E_INVALID otherwise); cuts
 * must span the domain and increase strictly, as for dsx_grid_set_cuts.
 * Scratch: one fixed 2.2 MB device array inside the library, placed on a GPU
 * at the first call there (or when the library's device code is loaded, if
 * module loading is eager) and held until the process exits; nothing else is
 * allocated.  The first call on a device looks up that array's device address
 * (and may make the driver load the library's device code): make the first
 * call before any CUDA-graph capture.  All calls share the array and it keeps the previous
 * call's contents, so calls that overlap on the GPU (other streams or host
 * threads) race: serialize them.  Errors: a DSX_E_* code and, if `error` is
 * not null, a message in the caller's buffer of `error_capacity` bytes. */
int dsx_migrate_noalloc(const dsx_grid_desc* desc, const double* cuts,
                        const long long* counts_in, const void* const* arrays_in,
                        long long* counts_out, void* const* arrays_out,
                        long long* results, void* stream, char* error,
                        int error_capacity);

#ifdef __cplusplus
}
#endif

#endif
