// Launch wrappers of the hand-written sm_100a kernels (dsx_kernels.cu).
// Every wrapper enqueues on `stream` and never synchronizes.
#pragma once

#include "dsx_device.cuh"

#include <vector>

namespace dsx {

// Optional per-kernel timing: when `on`, every launch wrapper records an
// event after its kernel (inside a captured graph these become event-record
// nodes), so that the host can read each kernel's duration of the last step.
struct Marks {
    static constexpr int kMax = 48;
    cudaEvent_t ev[kMax] = {};
    const char* name[kMax] = {};
    int count = 0;
    bool on = false;
    void mark(cudaStream_t s, const char* what) {
        if (!on || count >= kMax || !ev[count]) return;
        name[count] = what;
        // external: inside stream capture this becomes a real event-record
        // node that every replay of the graph executes
        cudaEventRecordWithFlags(ev[count++], s, cudaEventRecordExternal);
    }
};

// Scratch shared by the phases of one step (device buffers owned by the
// engine; sizes in the engine's allocate()).
struct Scratch {
    int* cnt = nullptr;        // [kHaloCounters][stride] per-tile counters
    int* pre = nullptr;        // [kHaloCounters][stride] exclusive prefixes
    int stride = 0;            // max_tiles + 1
    int* imm_total = nullptr;  // [P] immigrants per destination
    int* imm_base = nullptr;   // [P]
    int* emig_src = nullptr;   // [ncap]
    int* emig_dst = nullptr;   // [ncap]
    int* emig_hist = nullptr;  // [max_chunks][P]
    int* emig_info = nullptr;  // {E, nchunks}
    long long* mig_results = nullptr;  // [P][6]
    unsigned* mask = nullptr;  // [ncap] halo neighbor mask per owned particle
    unsigned short* dest16 = nullptr;  // [max_tiles * 512] destination per tile slot (fused step)
    int* tile_bases = nullptr;         // [max_tiles * 32] step counter bases per tile
    int* out_flags = nullptr;          // [P] out-of-domain flags
    int* list_len = nullptr;   // [P*26] send-list lengths
    int* send_base = nullptr;  // [P*26] first ghost slot of each send list
    int* g = nullptr;          // [P] ghosts per receiver
    int* gbase = nullptr;      // [P+1]
    int* ghost_owner = nullptr;  // [gcap] owned index of each ghost
    int* ghost_entry = nullptr;  // [gcap] sender r*26+n of each ghost
    int* bowner = nullptr;     // [ncap] owned index of each boundary owner
    int* boff = nullptr;       // [ncap+1] CSR offsets into bslot
    int* bslot = nullptr;      // [gcap] ghost slots of each boundary owner, n ascending
    int* bfirst = nullptr;     // [ncap] ghost slot of each boundary owner's first image
    int* tile_b0 = nullptr;    // [max_tiles + 1] first boundary owner of each tile (refresh)
    // sharded step only (null otherwise): emigrants per (destination, source)
    // from the classify, and the gap before each source's group of
    // immigrants that other shards fill
    int* pairs = nullptr;      // [P*P] pairs[t * P + q]
    int* gap = nullptr;        // [P*P] gap[t * P + q]
    int* halo_info = nullptr;  // {G, B}
    int* cbase = nullptr;      // [P*28] per subdomain: tile prefix -> global index
    // fused step
    int* imm_list = nullptr;   // [P*26] immigrants per (destination, send list)
    int* imm_bnd = nullptr;    // [P] immigrant boundary owners per destination
    int* imm_img = nullptr;    // [P] immigrant images per destination
    int* list_ret = nullptr;   // [P*26] retained part of each send list
    int* cbase_imm = nullptr;  // [P*28] bases of the immigrant parts
    int* imm_tile_start = nullptr;  // [P+1] tiles over the immigrant segments
    unsigned* ticket = nullptr;     // [1] CTAs done in the step's counter scan (0 between launches)
    int4* imm_tiles = nullptr;      // their descriptors
    int* cnt2 = nullptr;       // [28][stride] immigrant-tile counters
    int* pre2 = nullptr;
    int max_chunks = 0;
    Marks* marks = nullptr;
    // launch shapes the autotuner picks (these defaults are the untuned choice)
    int classify_threads = 128;   // threads per 512-particle tile of the step classify: 64/128/256
    int classify_combine = 0;     // immigrant counters combined per warp before the atomics
    int move_staged = 1;          // 1: staged (one pass if it fits), 2: staged in passes,
                                  // 3: staged without forces, 0: direct reads
    int refresh_kind = 3;         // refresh walk: 0 ghost by ghost, 1 owner by owner (the CSR),
                                  // 2 tile by tile with the owners staged (when the stage fits),
                                  // 3 tile by tile for a full refresh of 9 or more arrays, else 0
    int reverse_per_sm = 0;       // CTAs per SM of the reverse sum; 0: one wave of the default shape
};

void launch_layout(const Grid& G, const int* n, int* obase, int* tile_start, int4* tiles,
                   cudaStream_t s);

// Plain launches: host copies of the layout's tile starts and of the
// boundary-owner starts per subdomain; with them every tile kernel of a
// per-call operation is launched once per subdomain over its own tiles (the
// way one process per subdomain would launch), instead of once for all.
struct PlainLaunch {
    const int* tile_start = nullptr;      // [P+1]
    const int* boundary_start = nullptr;  // [P+1]
};

void launch_migrate(const Grid& G, const Arrays& A, long long src_off, long long dst_off,
                    const Scratch& S, cudaStream_t s, const PlainLaunch* plain = nullptr);

void launch_halo_build(const Grid& G, const Arrays& A, long long owned_off,
                       long long ghost_off, const Scratch& S, cudaStream_t s,
                       const PlainLaunch* plain = nullptr);

// migrate + plan build as one pipeline (the batched step); G: current layout,
// Gn: the same grid with the next layout current.
void launch_fused_step(const Grid& G, const Grid& Gn, const Arrays& A, long long src_off,
                       long long dst_off, long long ghost_off, const Scratch& S, cudaStream_t s,
                       bool counters_zeroed = false);

// The pipeline's parts, in order (the autotuner replays them one by one):
// classify (destinations, masks, tile counters), the counter scan and the
// next layout, the move (idempotent for a fixed current half), and the
// emigrant placement plus the immigrants' ghost images.
void launch_step_classify(const Grid& G, const Arrays& A, long long src_off, const Scratch& S,
                          cudaStream_t s, bool counters_zeroed = false);
void launch_step_layout(const Grid& G, const Scratch& S, cudaStream_t s);
void launch_step_move(const Grid& G, const Arrays& A, long long src_off, long long dst_off,
                      long long ghost_off, const Scratch& S, cudaStream_t s);
void launch_step_finish(const Grid& G, const Grid& Gn, const Arrays& A, long long src_off,
                        long long dst_off, long long ghost_off, const Scratch& S, cudaStream_t s);
// The finish in its two parts: the emigrants' stable multi-split into the
// next half (local_imm: emigrants expected per destination, checked; gap:
// null, or P x P slots left before each source's group for other shards'
// immigrants), then the immigrants' masks and ghost images.
void launch_step_emigrants(const Grid& G, const Arrays& A, long long src_off, long long dst_off,
                           const Scratch& S, const int* local_imm, const int* gap, cudaStream_t s);
void launch_step_immigrant_halo(const Grid& Gn, const Arrays& A, long long dst_off,
                                long long ghost_off, const Scratch& S, cudaStream_t s);
// A sharded step's pieces around its host-planned layout: the counter scan
// alone, the per-subdomain export of the scanned counters (29 P + 1 ints, see
// k_step_export), and the tile bases and descriptors of the planned layout
// (imm_in: immigrants per subdomain whose ghost images this grid makes).
void launch_step_scan(const Grid& G, const Scratch& S, cudaStream_t s);
void launch_step_export(const Grid& G, const Scratch& S, int* out, cudaStream_t s);
void launch_step_bases(const Grid& G, const Scratch& S, const int* imm_in, cudaStream_t s);
// Move kinds that apply to this record, as bits: 1 direct reads (kind 0),
// 2 staged (kind 1: one pass when a tile of the record fits 100 KB of shared
// memory, else passes of at most 56 KB), 4 staged in passes although one
// pass fits (kind 2), 8 staged in one pass without the force arrays, which
// the stays read from HBM (kind 3: ghosts never need their owner's force).
int staged_move_modes(const Arrays& A);

// ctas_per_sm > 0 caps the grid at that many CTAs per SM (the split phase
// leaves room on every SM for independent work on other streams); 0 fills
// the GPU with resident CTAs.
void launch_halo_refresh(const Grid& G, const Arrays& A, long long owned_off,
                         long long ghost_off, bool positions_only, const Scratch& S,
                         cudaStream_t s, int ctas_per_sm = 0);

struct FieldOps {
    int count = 0;
    int index[kMaxFields] = {};   // field index into Arrays::f
    int type[kMaxFields] = {};    // dsdecompx::FieldType order
    int components[kMaxFields] = {};
    int op[kMaxFields] = {};      // dsdecompx::ReduceOp order
};

void launch_forward_fields(const Grid& G, const Arrays& A, long long owned_off,
                           long long ghost_off, const FieldOps& F, const Scratch& S,
                           cudaStream_t s);

// owner[i] (+)= sum over its images of ghost[slot], images in neighbor order;
// used for reverse_halo (forces) and for the halo adjoint.
void launch_reverse_sum3(const Grid& G, double* ox, double* oy, double* oz,
                         const double* gx, const double* gy, const double* gz,
                         const Scratch& S, cudaStream_t s, const PlainLaunch* plain = nullptr);

void launch_reverse_fields(const Grid& G, const Arrays& A, long long owned_off,
                           long long ghost_off, const FieldOps& F, const Scratch& S,
                           cudaStream_t s);

// Dynamic cut-plane rebalance on the device (dsDecompX src/runtime.cpp:345-447)
// from the owned counts (work == nullptr) or a per-subdomain work metric.
struct RebalanceParams {
    double threshold = 1.10;
    double relaxation = 0.5;
    double minimum_fraction = 0.10;
    double halo_width = 0.0;
    int force = 0;
    long long interval = 1;   // 0: automatic rebalance disabled
    int automatic = 0;        // 1: the migrate-time check (counts the call)
    // the batched step's first kernel also clears the status word and the
    // step's immigrant counters (instead of two memset nodes before it)
    int clear_status = 0;
    int* zero = nullptr;
    int nzero = 0;
};
// out: {attempted, changed, imbalance(bits)} written to `result` (3 doubles)
void launch_rebalance(const Grid& G, const double* work, RebalanceParams params,
                      long long* call_counter, double* result, cudaStream_t s);

// 1-rank drop-in migrate: wraps positions in place (every particle stays).
void launch_wrap_inplace(double* x, double* y, double* z, long long n, const double* lower,
                         const double* extent, const int* periodic, cudaStream_t s);

// owner_rank of n positions (device arrays) into out[n].
void launch_owner_rank(const Grid& G, const double* x, const double* y, const double* z,
                       long long n, int* out, cudaStream_t s);
// flags[s] = 1 if an owned particle of subdomain s (current layout) belongs
// to another subdomain.
void launch_out_of_domain(const Grid& G, const double* x, const double* y, const double* z,
                          int* flags, cudaStream_t s);

// Emigrants of the last migration per (destination, source), dest-major
// P x P, from the emigrant list and the old layout's offsets.
void launch_pair_counts(int P, const Scratch& S, const int* obase_old, long long ncap, int* pairs,
                        cudaStream_t s);

// One device-to-device copy; launch_copies splits them into pieces of at
// most kCopyPiece bytes and runs them all in one kernel on `s`.
struct CopyPiece {
    const unsigned char* src;
    unsigned char* dst;
    long long bytes;
};
constexpr long long kCopyPiece = 256 * 1024;
cudaError_t launch_copies(const std::vector<CopyPiece>& copies, cudaStream_t s);

// Records a named timing mark on `s` (no-op unless S.marks->on).
void mark(const Scratch& S, cudaStream_t s, const char* what);

}  // namespace dsx
