/* Sharded virtual grid, native: the P subdomains of one box split over
 * several processes (one GPU each), every collective call one exchange step
 * with the processes that own neighboring blocks.
 *
 * The reference runs one MPI rank per subdomain (dsDecompX
 * include/dsdecompx.hpp:70-248, src/runtime.cpp:862-1041).  Here a process
 * owns a block of subdomains and keeps a grid of all P (dsx_grid_*) that
 * holds particles only in its own; after each local call the particles and
 * ghost lists that belong to another process's subdomains are sent there,
 * and every process assembles its subdomains in the reference's order
 * (retained, then immigrants by source rank; ghosts in the receiver's
 * neighbor-block order), so each subdomain's arrays equal the reference's.
 *
 * The two communication steps come from the caller as a transport: a sum
 * over all shards of a small vector, and point-to-point byte messages
 * between device buffers (an MPI host: MPI_Allreduce and CUDA-aware
 * MPI_Isend / MPI_Irecv; a NCCL host: ncclAllReduce and grouped
 * ncclSend / ncclRecv).  Every shard makes the same transport calls in the
 * same order.  Errors follow dsx.h (DSX_OK or a negative DSX_E_* code,
 * message in dsx_last_error). */
#ifndef DSX_SHARD_H
#define DSX_SHARD_H

#include "dsx.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsx_transport {
    void* user;
    /* values[0..n) := their sum over all shards (every shard gets it). */
    int (*allreduce_i64)(void* user, long long* values, long long n);
    int (*allreduce_f64)(void* user, double* values, long long n);
    /* Sends send[k] (send_bytes[k] device bytes) to shard send_to[k] and
     * receives recv_bytes[k] bytes from shard recv_from[k] into recv[k]
     * (device).  Both kinds of buffer are in use by the work queued on
     * `stream` so far (the sends are being filled, the receive buffers of
     * an earlier call may still be read): a transport whose transfers are
     * not ordered on `stream` (MPI) synchronizes it before touching them.
     * The call returns once the received bytes are in place for later work
     * on `stream` and the send buffers may be refilled by it.  Peers appear
     * once each, ascending; zero-byte messages are left out on both sides. */
    int (*exchange)(void* user, int nsend, const int* send_to, const void* const* send,
                    const long long* send_bytes, int nrecv, const int* recv_from,
                    void* const* recv, const long long* recv_bytes, void* stream);
} dsx_transport;

typedef struct dsx_shard dsx_shard;

/* desc and fields as dsx_grid_create (desc->nranks = P subdomains in all);
 * particles: this shard's owned-particle capacity; owners: the shard of
 * every subdomain (P values), or null for contiguous Cartesian blocks (the
 * factorisation of nshards that divides the process grid with the least cut
 * area, else contiguous runs of subdomain ranks).  The transport is copied. */
int dsx_shard_create(const dsx_grid_desc* desc, const dsx_field_desc* fields, int nfields,
                     long long particles, long long ghost_capacity, int shard, int nshards,
                     const int* owners, const dsx_transport* transport, dsx_shard** out);
int dsx_shard_destroy(dsx_shard* shard);

/* The shard of every subdomain (P values). */
int dsx_shard_owners(dsx_shard* shard, int* owners);

/* Host only (no GPU needed): the shard of every subdomain of the process
 * grid dims[3] (dims[0] * dims[1] * dims[2] values, subdomain rank order)
 * that dsx_shard_create chooses when given no owners, so that a process can
 * load just its own subdomains' particles before it creates its shard. */
int dsx_shard_plan_owners(const int* dims, int nshards, int* owners);

/* This shard's particles: counts[P] (zero outside its subdomains) and host
 * or device arrays as dsx_grid_upload. */
int dsx_shard_upload(dsx_shard* shard, const long long* counts, const void* const* arrays,
                     void* stream);

/* This shard's owned particles into host or device arrays (as
 * dsx_grid_download: counts[P] out, subdomains in rank order). */
int dsx_shard_download(dsx_shard* shard, long long* counts, void* const* arrays, void* stream);

/* Decomp::migrate on every shard (with the Dynamic rebalance over all
 * shards' counts).  results: null, or P x {changed, previous, retained, sent,
 * received, new_owned}, filled for this shard's subdomains. */
int dsx_shard_migrate(dsx_shard* shard, void* stream, long long* results);

/* Decomp::rebalance with work per subdomain (P values, this shard's entries
 * used; null: owned counts).  results: null, or P x {attempted, changed,
 * new_owned} for this shard's subdomains; imbalance: null or one value. */
int dsx_shard_rebalance(dsx_shard* shard, const double* work, int force, void* stream,
                        long long* results, double* imbalance);

/* Decomp::exchange_halo: builds (rebuild != 0, or no plan) or refreshes
 * (positions_only: x, y, z) this shard's receivers' ghosts.  results: null,
 * or P x {ghost_count, layout_changed, storage_reallocated, plan_reused} for
 * this shard's subdomains. */
int dsx_shard_exchange_halo(dsx_shard* shard, int rebuild, int positions_only, void* stream,
                            long long* results);

/* Decomp::reverse_halo: every ghost's force (in the assembled ghost region)
 * added to its owner, in the reference's order. */
int dsx_shard_reverse_halo(dsx_shard* shard, void* stream);

/* One fused step on every shard: migrate (with the Dynamic rebalance over
 * all shards' counts), halo build, callback(user, stream, view), reverse_halo
 * -- the batched step of dsx_grid_step for a sharded grid.  The counts of
 * every shard are summed before anything moves (one all-reduce), so each
 * shard plans its layout on the host and its kernels write retained
 * particles and ghost images straight to their final slots; the transport
 * then carries only the emigrants to other shards' subdomains, the ghost
 * lists toward other shards' receivers and, after the callback, those
 * ghosts' forces.  The view gives this shard's owned particles and its own
 * receivers' ghosts (halo_totals: {ghosts, boundary owners}); the callback
 * must not call the field exchanges (they refuse with DSX_E_LOGIC until the
 * next halo build).  Afterwards the per-call calls start from a rebuild
 * (exchange_halo builds the plan anew).  status as dsx_grid_step's. */
int dsx_shard_step(dsx_shard* shard, dsx_step_callback callback, void* user, void* stream,
                   unsigned* status);

/* Host only (no GPU needed): the layout dsx_shard_step plans on `shard`
 * from the counts summed over every shard (sums: 58 P + P * P + nshards
 * values in the step's all-reduce order -- per subdomain retained particles,
 * retained boundary owners and images, the retained part of its 26 send
 * lists; per destination its immigrants, their part of each list, their
 * boundary owners and images; the emigrant pairs [t * P + q]; each shard's
 * storage).  out (6 + 4 nshards values): owned particles after the step,
 * outgoing emigrants, ghost slots, this shard's receivers' ghosts, boundary
 * owners, images; then per shard p: emigrants sent to p, emigrants received
 * from p, ghosts sent to p, ghosts received from p. */
int dsx_shard_plan_step(const dsx_grid_desc* desc, const int* owners, int shard, int nshards,
                        const long long* sums, long long nsums, long long* out);

/* The grid-level form of dsx_shard_step, for hosts that keep their own
 * dsx_grid per process: owners[P] the shard of every subdomain, shard and
 * nshards this process's place, transport as in dsx_shard_create. */
int dsx_grid_sharded_step(dsx_grid* grid, const int* owners, int shard, int nshards,
                          const dsx_transport* transport, dsx_step_callback callback, void* user,
                          void* stream, unsigned* status);

/* Field exchanges as dsx_grid_forward_exchange / dsx_grid_reverse_exchange,
 * on the assembled ghosts. */
int dsx_shard_forward_exchange(dsx_shard* shard, int nfields, const int* field_ids, void* stream);
int dsx_shard_reverse_exchange(dsx_shard* shard, int nfields, const int* field_ids,
                               const int* ops, void* stream);

/* Owned particles: the local grid's view (owned half, per-subdomain counts).
 * Ghosts: the assembled region -- base[a] its arrays, ghost_offset 0,
 * ghost_capacity its capacity, g / gbase (device, P and P + 1 values) and
 * halo_totals (device {ghosts, 0}) this shard's receivers' blocks. */
int dsx_shard_owned_view(dsx_shard* shard, dsx_grid_view* out);
int dsx_shard_ghost_view(dsx_shard* shard, dsx_grid_view* out);

/* The local grid's totals as dsx_grid_totals ({owned particles, emigrants
 * of the last migrate, ghosts of its own lists, boundary owners}). */
int dsx_shard_totals(dsx_shard* shard, long long* out4, void* stream);

/* Kernels of this library launched for this shard so far (benchmarks). */
int dsx_shard_launches(dsx_shard* shard, long long* count);

/* Host counts per subdomain (zero outside this shard's subdomains), read
 * after the work queued on `stream`. */
int dsx_shard_counts(dsx_shard* shard, long long* owned, long long* ghosts, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DSX_SHARD_H */
