/*
 * dsx_oracle: a plain-C, single-threaded restatement of dsDecompX's Host-mode
 * particle bookkeeping (migrate, exchange_halo, reverse_halo,
 * reverse_exchange, the forward field copy and the dynamic cut-plane
 * rebalance) for a virtual Cartesian grid of P subdomains held in one process.
 *
 * TEST INFRASTRUCTURE ONLY.  It is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.  It is
 * itself pinned against the reference's own Host path (built from the
 * reference sources into oracle/_ref) and against the committed golden
 * fixtures under tests/golden/.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the dsDecompX source tree).
 */
#ifndef DSX_ORACLE_H
#define DSX_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid orc_grid;

/* policy: 0 Manual, 1 Balanced, 2 TopologyAware, 3 Dynamic
 * dynamic: {interval, imbalance_threshold, relaxation, minimum_cell_fraction}
 * field types: 0 Int32, 1 Int64, 2 UInt32, 3 UInt64, 4 Float32, 5 Float64 */
orc_grid* orc_create(int nranks, const int* dims, int policy,
                     const double* lower, const double* upper,
                     const int* periodic, double halo_width,
                     int edges_and_corners, const double* dynamic,
                     int nfields, const int* types,
                     const long long* components, char* error,
                     int error_length);
void orc_destroy(orc_grid* g);
const char* orc_last_error(orc_grid* g);

int orc_size(orc_grid* g);
int orc_topology(orc_grid* g, int rank, int* dims, int* coords, double* local);
int orc_neighbors(orc_grid* g, int rank, int* count, int* info, double* shifts);
int orc_cuts(orc_grid* g, double* out);
int orc_owner_rank(orc_grid* g, long long n, const double* positions, int* out);

int orc_set_owned(orc_grid* g, int rank, long long n,
                  const double* const* core, const int* type,
                  const int* global_id, const void* const* fields);
int orc_counts(orc_grid* g, int rank, long long* owned, long long* ghosts);
int orc_halo_blocks(orc_grid* g, int rank, int* count, long long* out);
int orc_set_rebalance_work(orc_grid* g, const double* work);
/* array ids: 0..10 x y z vx vy vz fx fy fz mass charge, 11 type,
 * 12 global_id, 13+f registered field f */
int orc_read(orc_grid* g, int rank, int array, long long start,
             long long count, void* out);
int orc_write(orc_grid* g, int rank, int array, long long start,
              long long count, const void* in);

/* results per rank: {changed, previous, retained, sent, received, new_owned} */
int orc_migrate(orc_grid* g, long long* results);
/* results per rank: {ghost_count, layout_changed, 0, plan_reused} */
int orc_exchange_halo(orc_grid* g, int rebuild, long long* results);
int orc_reverse_halo(orc_grid* g);
/* ops: 0 Sum, 1 Min, 2 Max, 3 Replace */
int orc_reverse_exchange(orc_grid* g, int nfields, const int* field_ids,
                         const int* ops);
int orc_forward_exchange(orc_grid* g, int nfields, const int* field_ids);
/* results per rank: {attempted, geometry_changed, new_owned} */
int orc_rebalance(orc_grid* g, const double* local_work, int force,
                  long long* results, double* imbalance);
int orc_set_halo_width(orc_grid* g, double width);
int orc_invalidate_halo(orc_grid* g);
/* cuts: axis 0, 1, 2 concatenated (dims[a] + 1 each) */
int orc_set_cuts(orc_grid* g, const double* cuts);
/* invalidate != 0: update_domain, else rescale_domain */
int orc_rescale_domain(orc_grid* g, const double* lower, const double* upper, int invalidate);

#ifdef __cplusplus
}
#endif

#endif
