// Host side of the engine: topology tables, device storage, orchestration of
// the kernels in dsx_kernels.cu, CUDA-graph capture of the batched step, and
// the extern "C" entry points declared in include/dsx.h.
#include "dsx.h"
#include "dsx_errors.h"
#include "dsx_shard.h"
#include "dsx_kernels.cuh"

#include <algorithm>
#include <climits>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_error;

struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& message) : std::runtime_error(message), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& message) {
    throw Failure(code, "dsDecompX: " + message);
}

void cuda_check(cudaError_t status, const char* what) {
    if (status != cudaSuccess)
        fail(DSX_E_RUNTIME, std::string(what) + ": " + cudaGetErrorString(status));
}

template <class F>
int guarded(F&& body) {
    try {
        body();
        return DSX_OK;
    } catch (const Failure& e) {
        g_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_error = std::string("dsDecompX: ") + e.what();
        return DSX_E_RUNTIME;
    }
}

std::size_t field_type_size(int type) {
    switch (type) {
    case DSX_INT32: case DSX_UINT32: case DSX_FLOAT32: return 4;
    case DSX_INT64: case DSX_UINT64: case DSX_FLOAT64: return 8;
    default: fail(DSX_E_INVALID, "unsupported field type");
    }
}

// ------------------------------------------------------------ topology

// Lower is better; ties broken on (px, py, pz) (dsDecompX src/grid.cpp:12-22).
double balanced_score(const int* g, const double* len) {
    const double lx = len[0] / g[0], ly = len[1] / g[1], lz = len[2] / g[2];
    const double surface = 2.0 * (1.0 / lx + 1.0 / ly + 1.0 / lz);
    const double longest = std::max({lx, ly, lz});
    const double shortest = std::min({lx, ly, lz});
    return surface * (1.0 + 0.05 * std::log(longest / shortest));
}

// All virtual ranks share one GPU, i.e. one node: the topology-aware score
// of dsDecompX src/grid.cpp:28-75 with a single node.
double single_node_score(const int* g, const double* len, const int* periodic) {
    const double local[3] = {len[0] / g[0], len[1] / g[1], len[2] / g[2]};
    const double face[3] = {local[1] * local[2], local[0] * local[2], local[0] * local[1]};
    double cost = 0.0;
    for (int x = 0; x < g[0]; ++x)
        for (int y = 0; y < g[1]; ++y)
            for (int z = 0; z < g[2]; ++z) {
                const int source = (x * g[1] + y) * g[2] + z;
                for (int a = 0; a < 3; ++a) {
                    int c[3] = {x, y, z};
                    if (++c[a] == g[a]) {
                        if (!periodic[a] || g[a] == 1) continue;
                        c[a] = 0;
                    }
                    if ((c[0] * g[1] + c[1]) * g[2] + c[2] == source) continue;
                    cost += face[a] * 1.0;
                }
            }
    return cost / (local[0] * local[1] * local[2] * g[0] * g[1] * g[2]) +
           0.01 * balanced_score(g, len);
}

void choose_grid(int n, const double* len, const int* periodic, int policy, int* out) {
    double best_score = std::numeric_limits<double>::infinity();
    int best[3] = {n, 1, 1};
    for (int px = 1; px <= n; ++px) {
        if (n % px) continue;
        const int rest = n / px;
        for (int py = 1; py <= rest; ++py) {
            if (rest % py) continue;
            const int cand[3] = {px, py, rest / py};
            const double score = policy == DSX_TOPOLOGY_AWARE ? single_node_score(cand, len, periodic)
                                                              : balanced_score(cand, len);
            const bool less = std::make_tuple(score, cand[0], cand[1], cand[2]) <
                              std::make_tuple(best_score, best[0], best[1], best[2]);
            if (less) {
                best_score = score;
                std::copy(cand, cand + 3, best);
            }
        }
    }
    std::copy(best, best + 3, out);
}

// Fills zero entries with a balanced factorization, largest first, like
// MPI_Dims_create.
bool fill_dims(int n, int* dims) {
    int fixed = 1, free_count = 0;
    for (int a = 0; a < 3; ++a) {
        if (dims[a] < 0) return false;
        if (dims[a] > 0) fixed *= dims[a];
        else ++free_count;
    }
    if (!free_count) return fixed == n;
    if (n % fixed) return false;
    int rest = n / fixed;
    std::vector<int> factors;
    for (int f = 2; rest > 1 && f * f <= rest; ++f)
        while (rest % f == 0) { factors.push_back(f); rest /= f; }
    if (rest > 1) factors.push_back(rest);
    std::sort(factors.rbegin(), factors.rend());
    std::vector<int> grid(static_cast<std::size_t>(free_count), 1);
    for (int f : factors) *std::min_element(grid.begin(), grid.end()) *= f;
    std::sort(grid.rbegin(), grid.rend());
    std::size_t k = 0;
    for (int a = 0; a < 3; ++a) if (dims[a] == 0) dims[a] = grid[k++];
    return true;
}

int direction_slot(int dx, int dy, int dz) {
    const int raw = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
    return raw < 13 ? raw : raw - 1;
}

struct Neighbor {
    int rank = -1;
    int dir[3] = {0, 0, 0};
    int slot = -1;
    double shift[3] = {0, 0, 0};
};

// The 26-direction neighbor list of one subdomain, in the reference's loop
// order and with its rules (dsDecompX src/topology.cpp:85-167): directions
// that move along an unsplit axis are skipped, periodic wrap gives the image
// shift +L (coordinate below 0) or -L (at or past dims), a non-periodic
// boundary gives rank -1.
std::vector<Neighbor> neighbors_of(const int* c, const int* dims, const dsx_grid_desc& d) {
    std::vector<Neighbor> out;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                if (!d.edges_and_corners && std::abs(dx) + std::abs(dy) + std::abs(dz) != 1) continue;
                const int dir[3] = {dx, dy, dz};
                bool unsplit = false;
                for (int a = 0; a < 3; ++a) unsplit = unsplit || (dir[a] != 0 && dims[a] == 1);
                if (unsplit) continue;
                Neighbor nb;
                int nc[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
                bool outside = false;
                for (int a = 0; a < 3 && !outside; ++a) {
                    if (nc[a] >= 0 && nc[a] < dims[a]) continue;
                    if (!d.periodic[a]) { outside = true; break; }
                    const double extent = d.upper[a] - d.lower[a];
                    if (nc[a] < 0) { nc[a] += dims[a]; nb.shift[a] = extent; }
                    else { nc[a] -= dims[a]; nb.shift[a] = -extent; }
                }
                for (int a = 0; a < 3; ++a) nb.dir[a] = dir[a];
                nb.slot = direction_slot(dx, dy, dz);
                nb.rank = outside ? -1 : (nc[0] * dims[1] + nc[1]) * dims[2] + nc[2];
                out.push_back(nb);
            }
    return out;
}

// ------------------------------------------------------------ device memory

struct DeviceBlock {
    void* p = nullptr;
    ~DeviceBlock() { if (p) cudaFree(p); }
};

template <class T>
T* device_alloc(std::vector<void*>& owned, std::size_t count) {
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<std::size_t>(count, 1) * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

void dsx::set_last_error(const char* message) { g_error = message ? message : ""; }

namespace {

// sender entry of receiver (q, m): the entry of r = nbr(q,m) that points
// toward -d_m (the MPI backend's tag matching, dsDecompX
// src/backends/mpi_backend.cpp:398-433)
int sender_entry_of(const std::vector<std::vector<Neighbor>>& topo, int q, int m) {
    const Neighbor& nb = topo[static_cast<std::size_t>(q)][static_cast<std::size_t>(m)];
    if (nb.rank < 0) return -1;
    const int want = direction_slot(-nb.dir[0], -nb.dir[1], -nb.dir[2]);
    const auto& list = topo[static_cast<std::size_t>(nb.rank)];
    for (std::size_t n = 0; n < list.size(); ++n)
        if (list[n].slot == want && list[n].rank == q) return nb.rank * dsx::kMaxNeighbors + static_cast<int>(n);
    return -1;
}

struct ShardPlan {
    std::vector<int> n_next, obase_next, tile_start_next;   // P, P+1, P+1
    std::vector<int> imm_base, imm_tiles_in, imm_tile_start, local_imm;   // P, P, P+1, P
    std::vector<int> gap;                                    // P*P
    std::vector<long long> results;                          // P*6
    std::vector<int> list_ret, list_len, send_base;          // P*26
    std::vector<int> g, gbase;                               // P, P+1
    std::vector<int> cbase_ret, cbase_imm;                   // P*28
    long long own_total = 0, out_total = 0, ghosts = 0, own_ghosts = 0, boundary = 0, images = 0;
    int emigrants = 0;
    // per peer shard: outgoing emigrants [out_start, out_end) of the next
    // half; outgoing ghost lists [gout_start, gout_end) of the ghost region
    std::vector<long long> out_start, out_end, gout_start, gout_end;
    std::vector<long long> recv_particles, recv_ghosts;      // per peer
};

// The layout of one shard's fused step (see dsx_grid::sharded_step), from
// `sum`, the sum over every shard of: [0, 29P) the export of k_step_export
// (retained particles, boundary owners and images of the retained parts,
// the retained part of every send list), [29P, 58P) the immigrant counters
// (per destination: total, per list, boundary owners, images), [58P, 58P +
// P*P) the emigrant pairs [t * P + q], then one storage entry per shard.
// local_emigrants: this shard's own emigrants (not summed).
ShardPlan plan_shard_layout(int P, const std::vector<std::vector<Neighbor>>& topo,
                            const std::vector<long long>& sum, const std::vector<int>& owners,
                            int shard, int nshards, int local_emigrants) {
    const int E = dsx::kMaxNeighbors;
    auto sender_entry = [&](int q, int m) { return sender_entry_of(topo, q, m); };
    ShardPlan pl;
    const long long* stays = sum.data();
    const long long* bret = stays + P;
    const long long* iret = bret + P;
    const long long* lret = iret + P;                       // P * 26
    const long long* imm_total = lret + static_cast<std::size_t>(P) * E;
    const long long* imm_list = imm_total + P;             // P * 26
    const long long* imm_bnd = imm_list + static_cast<std::size_t>(P) * E;
    const long long* imm_img = imm_bnd + P;
    const long long* pairs = imm_img + P;                   // P * P, [t * P + q]
    auto own = [&](int t) { return owners[static_cast<std::size_t>(t)] == shard; };
    auto pair = [&](int t, int q) { return pairs[static_cast<std::size_t>(t) * P + q]; };
    pl.emigrants = local_emigrants;
    // owned layout: own subdomains contiguous in rank order, then the
    // outgoing emigrants by (destination's shard, destination)
    pl.n_next.assign(P, 0);
    pl.obase_next.assign(P + 1, 0);
    pl.tile_start_next.assign(P + 1, 0);
    pl.imm_base.assign(P, 0);
    pl.imm_tiles_in.assign(P, 0);
    pl.imm_tile_start.assign(P + 1, 0);
    pl.local_imm.assign(P, 0);
    pl.gap.assign(static_cast<std::size_t>(P) * P, 0);
    pl.results.assign(static_cast<std::size_t>(P) * 6, 0);
    for (int t = 0; t < P; ++t) {
        long long local = 0;
        for (int q = 0; q < P; ++q)
            if (own(q)) local += pair(t, q);
        pl.local_imm[t] = static_cast<int>(local);
        if (own(t)) {
            pl.n_next[t] = static_cast<int>(stays[t] + imm_total[t]);
            pl.imm_tiles_in[t] = static_cast<int>(imm_total[t]);
            long long before_remote = 0;
            for (int q = 0; q < P; ++q) {
                if (own(q)) pl.gap[static_cast<std::size_t>(t) * P + q] = static_cast<int>(before_remote);
                else before_remote += pair(t, q);
            }
            long long sent = 0;
            for (int d = 0; d < P; ++d) sent += pair(d, t);
            long long* o = &pl.results[static_cast<std::size_t>(6) * t];
            o[1] = stays[t] + sent;
            o[2] = stays[t];
            o[3] = sent;
            o[4] = imm_total[t];
            o[5] = stays[t] + imm_total[t];
            o[0] = (o[3] != 0 || o[4] != 0) ? 1 : 0;
        }
    }
    for (int t = 0; t < P; ++t) {
        pl.obase_next[t + 1] = pl.obase_next[t] + pl.n_next[t];
        pl.tile_start_next[t + 1] = pl.tile_start_next[t] + (pl.n_next[t] + dsx::kTile - 1) / dsx::kTile;
        pl.imm_tile_start[t + 1] = pl.imm_tile_start[t] + (pl.imm_tiles_in[t] + dsx::kTile - 1) / dsx::kTile;
        if (own(t)) pl.imm_base[t] = pl.obase_next[t] + static_cast<int>(stays[t]);
    }
    pl.own_total = pl.obase_next[P];
    pl.out_start.assign(nshards, 0);
    pl.out_end.assign(nshards, 0);
    long long at = pl.own_total;
    for (int p = 0; p < nshards; ++p) {
        pl.out_start[p] = at;
        if (p != shard)
            for (int t = 0; t < P; ++t)
                if (owners[t] == p) {
                    pl.imm_base[t] = static_cast<int>(at);
                    at += pl.local_imm[t];
                }
        pl.out_end[p] = at;
    }
    pl.out_total = at - pl.own_total;
    // remote immigrants each peer sends: groups (own t, source q of p)
    pl.recv_particles.assign(nshards, 0);
    for (int t = 0; t < P; ++t)
        if (own(t))
            for (int q = 0; q < P; ++q)
                if (!own(q)) pl.recv_particles[owners[q]] += pair(t, q);
    // ghost layout: list lengths, receiver order, list bases
    pl.list_ret.assign(static_cast<std::size_t>(P) * E, 0);
    pl.list_len.assign(static_cast<std::size_t>(P) * E, 0);
    pl.send_base.assign(static_cast<std::size_t>(P) * E, 0);
    pl.g.assign(P, 0);
    pl.gbase.assign(P + 1, 0);
    for (int r = 0; r < P; ++r)
        for (std::size_t n = 0; n < topo[r].size(); ++n) {
            if (topo[r][n].rank < 0) continue;
            const std::size_t e = static_cast<std::size_t>(r) * E + n;
            pl.list_ret[e] = static_cast<int>(lret[e]);
            pl.list_len[e] = static_cast<int>(lret[e] + imm_list[e]);
        }
    std::vector<int> order;
    for (int q = 0; q < P; ++q)
        if (own(q)) order.push_back(q);
    const std::size_t own_receivers = order.size();
    for (int p = 0; p < nshards; ++p)
        if (p != shard)
            for (int q = 0; q < P; ++q)
                if (owners[q] == p) order.push_back(q);
    pl.gout_start.assign(nshards, 0);
    pl.gout_end.assign(nshards, 0);
    pl.recv_ghosts.assign(nshards, 0);
    long long run = 0;
    for (std::size_t k = 0; k < order.size(); ++k) {
        const int q = order[k];
        if (k == own_receivers) pl.own_ghosts = run;
        const int p = owners[q];
        if (!own(q) && (k == own_receivers || owners[order[k - 1]] != p)) pl.gout_start[p] = run;
        pl.gbase[q] = static_cast<int>(run);
        for (std::size_t m = 0; m < topo[q].size(); ++m) {
            const int e = sender_entry(q, static_cast<int>(m));
            if (e < 0) continue;
            const int r = e / E;
            const bool present = own(q) || own(r);
            const long long len = present ? pl.list_len[static_cast<std::size_t>(e)] : 0;
            pl.send_base[static_cast<std::size_t>(e)] = static_cast<int>(run);
            if (own(q) && !own(r)) pl.recv_ghosts[owners[r]] += len;
            run += len;
        }
        pl.g[q] = own(q) ? static_cast<int>(run - pl.gbase[q]) : 0;
        if (!own(q)) pl.gout_end[p] = run;
    }
    if (order.size() == own_receivers) pl.own_ghosts = run;
    pl.ghosts = run;
    pl.gbase[P] = static_cast<int>(run);
    // counter bases of own senders: lists (retained part, immigrant
    // part), boundary owners and images (retained first)
    pl.cbase_ret.assign(static_cast<std::size_t>(P) * dsx::kHaloCounters, 0);
    pl.cbase_imm.assign(static_cast<std::size_t>(P) * dsx::kHaloCounters, 0);
    long long bb = 0, ib = 0;
    for (int r = 0; r < P; ++r) {
        if (!own(r)) continue;
        for (std::size_t n = 0; n < topo[r].size(); ++n) {
            if (topo[r][n].rank < 0) continue;
            const std::size_t e = static_cast<std::size_t>(r) * E + n;
            pl.cbase_ret[static_cast<std::size_t>(r) * dsx::kHaloCounters + n] = pl.send_base[e];
            pl.cbase_imm[static_cast<std::size_t>(r) * dsx::kHaloCounters + n] = pl.send_base[e] + pl.list_ret[e];
        }
        int* cr = &pl.cbase_ret[static_cast<std::size_t>(r) * dsx::kHaloCounters];
        int* ci = &pl.cbase_imm[static_cast<std::size_t>(r) * dsx::kHaloCounters];
        cr[dsx::kBoundaryCounter] = static_cast<int>(bb);
        ci[dsx::kBoundaryCounter] = static_cast<int>(bb + bret[r]);
        cr[dsx::kImageCounter] = static_cast<int>(ib);
        ci[dsx::kImageCounter] = static_cast<int>(ib + iret[r]);
        bb += bret[r] + imm_bnd[r];
        ib += iret[r] + imm_img[r];
    }
    pl.boundary = bb;
    pl.images = ib;
    return pl;
}

}  // namespace


struct dsx_grid {
    dsx_grid_desc desc{};
    int P = 1;
    int dims[3] = {1, 1, 1};
    struct Field {
        std::string name;
        int type = DSX_FLOAT64;
        int components = 1;
        int bytes = 8;
    };
    std::vector<Field> fields;
    std::vector<std::vector<Neighbor>> topo;   // per rank
    std::vector<std::array<int, 3>> coords;
    double halo_width = 0.0;
    long long ncap = 0, gcap = 0;
    long long total = 0;   // owned particles in the grid (conserved)

    // device storage
    std::vector<void*> arrays_owned;    // particle arrays (reallocated on growth)
    std::vector<void*> scratch_owned;   // ghost-sized scratch (reallocated on growth)
    std::vector<void*> fixed_owned;     // everything else
    dsx::Arrays A;
    dsx::Scratch S;
    double* cuts = nullptr;
    int cut_offset[3] = {0, 0, 0};
    int* layout[2][3] = {};   // [which][n, obase, tile_start]
    int4* layout_tiles[2] = {};   // per-tile descriptors of each layout
    int cur = 0;              // current layout index
    unsigned long long layout_version = 0;   // moves with every new layout
    int parity = 0;           // current owned half
    unsigned* status = nullptr;
    long long* call_counter = nullptr;
    double* rebalance_result = nullptr;   // [6]: automatic, explicit
    double* work = nullptr;               // [P]
    int* pairs = nullptr;                 // [P*P] emigrants per (destination, source)
    bool pairs_valid = false;             // the emigrant list belongs to the current layout
    std::vector<double> next_work;        // work of the next per-call migrate's rebalance
    // static topology tables
    int* d_nn = nullptr;
    int* d_nbr = nullptr;
    int* d_recv_entry = nullptr;
    int* d_sender_of = nullptr;
    double* d_shift = nullptr;
    signed char* d_dir = nullptr;
    unsigned* d_lut = nullptr;
    unsigned* d_lut_empty = nullptr;   // the same shape, every mask 0 (no halo)
    int* d_coord = nullptr;
    // plain launches (per-call operations, one launch per subdomain)
    bool plain = false;
    std::vector<int> plain_tiles, plain_bounds;
    dsx::PlainLaunch plain_launch;

    // host state
    bool plan_valid = false;
    bool ghosts_valid = false;
    std::vector<long long> last_ghosts;
    unsigned* pinned_status = nullptr;   // [4]: status, G, B, pad
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    dsx::Marks marks;
    dsx_step_callback graph_callback = nullptr;
    void* graph_user = nullptr;
    cudaStream_t graph_stream = nullptr;
    // Asynchronous steps: each step graph copies its build status (before the
    // callback) to pinned_build[4 * parity] and records build_done[parity]
    // there, so the next step can check it while this one's callback and
    // reverse sum still run.
    unsigned* pinned_build = nullptr;             // [8]: per parity status, G, B, pad
    cudaEvent_t build_done[2] = {nullptr, nullptr};
    // the build-status copy runs on a branch of the step graph, so the
    // callback does not wait for it (fork and join events, side stream)
    cudaStream_t side_stream = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    bool async_inflight = false;                  // a step whose status is unchecked
    int async_parity = 0;
    unsigned async_status = 0;                    // bits of the checked asynchronous steps
    cudaStream_t async_stream = nullptr;

    ~dsx_grid() {
        if (async_inflight) cudaStreamSynchronize(async_stream);
        async_inflight = false;
        destroy_graphs();
        for (auto& e : build_done) if (e) cudaEventDestroy(e);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (join_ev) cudaEventDestroy(join_ev);
        if (side_stream) cudaStreamDestroy(side_stream);
        if (pinned_build) cudaFreeHost(pinned_build);
        free_shard_buffers();
        for (auto& e : marks.ev) if (e) cudaEventDestroy(e);
        for (void* p : arrays_owned) cudaFree(p);
        for (void* p : scratch_owned) cudaFree(p);
        for (void* p : fixed_owned) cudaFree(p);
        if (pinned_status) cudaFreeHost(pinned_status);
    }

    // Split-phase halo as two captured graph segments: segment 1 is the
    // exchange itself, per {full refresh, positions-only refresh, build} and
    // owned half; segment 2 the completion (status and totals to the host),
    // per owned half.  Rebuilt like the step's graphs when the storage, the
    // box or the launch shapes change.
    cudaGraphExec_t split_begin[3][2] = {};
    cudaGraphExec_t split_end[2] = {nullptr, nullptr};
    int split_ctas_per_sm = 0;

    void destroy_graphs() {
        settle_async();
        for (auto& g : graph) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
        for (auto& row : split_begin)
            for (auto& g : row) {
                if (g) cudaGraphExecDestroy(g);
                g = nullptr;
            }
        for (auto& g : split_end) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
    }

    // Captures `enqueue` into `exec` once, then launches it on `stream`.
    template <class F>
    void run_captured(cudaGraphExec_t& exec, cudaStream_t stream, F&& enqueue) {
        if (!exec) {
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            enqueue();
            cuda_check(cudaStreamEndCapture(stream, &g), "end capture");
            const cudaError_t st = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            cuda_check(st, "instantiate graph");
        }
        cuda_check(cudaGraphLaunch(exec, stream), "launch graph");
    }

    static bool capturable(cudaStream_t stream) {
        return stream != nullptr && stream != cudaStreamLegacy && stream != cudaStreamPerThread;
    }

    long long owned_off() const { return parity ? ncap : 0; }
    long long next_off() const { return parity ? 0 : ncap; }
    long long ghost_off() const { return 2 * ncap; }

    dsx::Grid params() const {
        dsx::Grid G;
        G.P = P;
        for (int a = 0; a < 3; ++a) {
            G.dims[a] = dims[a];
            G.periodic[a] = desc.periodic[a] ? 1 : 0;
            G.lower[a] = desc.lower[a];
            G.upper[a] = desc.upper[a];
            G.extent[a] = desc.upper[a] - desc.lower[a];
            G.cut_offset[a] = cut_offset[a];
        }
        G.width = halo_width;
        G.ncap = ncap;
        G.gcap = gcap;
        G.tile = dsx::kTile;
        G.max_tiles = static_cast<int>((ncap + dsx::kTile - 1) / dsx::kTile) + P;
        G.nn = d_nn;
        G.nbr = d_nbr;
        G.recv_entry = d_recv_entry;
        G.sender_of = d_sender_of;
        G.shift = d_shift;
        G.dir = d_dir;
        G.lut = d_lut;
        G.coord = d_coord;
        G.cuts = cuts;
        G.n = layout[cur][0];
        G.obase = layout[cur][1];
        G.tile_start = layout[cur][2];
        G.tiles = layout_tiles[cur];
        G.n_next = layout[cur ^ 1][0];
        G.obase_next = layout[cur ^ 1][1];
        G.tile_start_next = layout[cur ^ 1][2];
        G.tiles_next = layout_tiles[cur ^ 1];
        G.status = status;
        return G;
    }

    void setup(const dsx_grid_desc& d, const dsx_field_desc* f, int nfields, long long particles,
               long long ghost_capacity) {
        desc = d;
        P = d.nranks;
        if (P < 1 || P > dsx::kMaxRanks) fail(DSX_E_INVALID, "nranks must be in 1..1024");
        for (int a = 0; a < 3; ++a)
            if (!(d.upper[a] > d.lower[a])) fail(DSX_E_INVALID, "global-domain extent must be positive");
        if (d.halo_width < 0.0) fail(DSX_E_INVALID, "halo width cannot be negative");
        if (!(d.dyn_threshold >= 1.0) || !(d.dyn_relaxation > 0.0 && d.dyn_relaxation <= 1.0) ||
            !(d.dyn_min_fraction > 0.0 && d.dyn_min_fraction <= 1.0) || d.dyn_interval < 0)
            fail(DSX_E_INVALID, "invalid dynamic load-balance configuration");
        if (nfields < 0 || nfields > dsx::kMaxFields)
            fail(DSX_E_INVALID, "at most 16 custom fields are supported on CUDA particle memory");
        if (particles < 0 || particles >= (1ll << 30)) fail(DSX_E_INVALID, "particle count out of range");
        for (int i = 0; i < nfields; ++i) {
            Field fd;
            fd.name = f[i].name ? f[i].name : "";
            fd.type = f[i].type;
            fd.components = f[i].components;
            if (fd.name.empty() || fd.components <= 0)
                fail(DSX_E_INVALID, "invalid or undersized custom particle field");
            for (const auto& other : fields)
                if (other.name == fd.name) fail(DSX_E_INVALID, "duplicate custom particle field '" + fd.name + "'");
            fd.bytes = static_cast<int>(field_type_size(fd.type)) * fd.components;
            fields.push_back(fd);
        }
        // process grid (dsDecompX src/topology.cpp:18-55)
        if (d.policy != DSX_MANUAL) {
            const double len[3] = {d.upper[0] - d.lower[0], d.upper[1] - d.lower[1], d.upper[2] - d.lower[2]};
            choose_grid(P, len, d.periodic, d.policy, dims);
        } else {
            for (int a = 0; a < 3; ++a) dims[a] = d.dims[a];
        }
        if (!fill_dims(P, dims)) fail(DSX_E_INVALID, "process-grid dimensions do not match communicator size");
        halo_width = d.halo_width;
        ncap = std::max<long long>(particles, 1);
        gcap = ghost_capacity > 0 ? ghost_capacity : std::max<long long>(ncap, 1 << 16);
        build_topology();
        allocate_fixed();
        allocate_arrays();
        allocate_ghost_scratch();
        cuda_check(cudaMallocHost(reinterpret_cast<void**>(&pinned_status), 4 * sizeof(unsigned)),
                   "cudaMallocHost");
        cuda_check(cudaMallocHost(reinterpret_cast<void**>(&pinned_build), 8 * sizeof(unsigned)),
                   "cudaMallocHost");
        for (auto& e : build_done)
            cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
        cuda_check(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming), "create event");
        cuda_check(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming), "create event");
        cuda_check(cudaStreamCreateWithFlags(&side_stream, cudaStreamNonBlocking), "create stream");
        S.marks = &marks;
        last_ghosts.assign(static_cast<std::size_t>(P), 0);
    }

    void build_topology() {
        topo.assign(static_cast<std::size_t>(P), {});
        coords.assign(static_cast<std::size_t>(P), {});
        for (int s = 0; s < P; ++s) {
            int c[3] = {s / (dims[1] * dims[2]), (s / dims[2]) % dims[1], s % dims[2]};
            coords[static_cast<std::size_t>(s)] = {c[0], c[1], c[2]};
            topo[static_cast<std::size_t>(s)] = neighbors_of(c, dims, desc);
        }
    }

    // sender entry of receiver (q, m): the entry of r = nbr(q,m) that points
    // toward -d_m (the MPI backend's tag matching, dsDecompX
    // src/backends/mpi_backend.cpp:398-433)
    int sender_entry(int q, int m) const { return sender_entry_of(topo, q, m); }

    void allocate_fixed() {
        const int E = dsx::kMaxNeighbors;
        std::vector<int> nn(P), nbr(P * E, -1), recv_entry(P * E, -1), sender_of(P * E, -1);
        std::vector<double> shift(P * E * 3, 0.0);
        std::vector<signed char> dir(P * E * 3, 0);
        std::vector<unsigned> lut(static_cast<std::size_t>(P) * 64, 0u);
        for (int s = 0; s < P; ++s) {
            const auto& list = topo[static_cast<std::size_t>(s)];
            nn[s] = static_cast<int>(list.size());
            for (std::size_t n = 0; n < list.size(); ++n) {
                const int idx = s * E + static_cast<int>(n);
                nbr[idx] = list[n].rank;
                for (int a = 0; a < 3; ++a) {
                    shift[3 * idx + a] = list[n].shift[a];
                    dir[3 * idx + a] = static_cast<signed char>(list[n].dir[a]);
                }
                sender_of[idx] = sender_entry(s, static_cast<int>(n));
                if (sender_of[idx] >= 0) recv_entry[sender_of[idx]] = idx;
            }
            // flags bit 2a: below lower+w on axis a; bit 2a+1: above upper-w
            for (unsigned flags = 1; flags < 64; ++flags) {
                unsigned mask = 0;
                for (std::size_t n = 0; n < list.size(); ++n) {
                    if (list[n].rank < 0) continue;
                    bool hit = true;
                    for (int a = 0; a < 3; ++a) {
                        if (list[n].dir[a] < 0 && !(flags & (1u << (2 * a)))) hit = false;
                        if (list[n].dir[a] > 0 && !(flags & (2u << (2 * a)))) hit = false;
                    }
                    if (hit) mask |= 1u << n;
                }
                lut[static_cast<std::size_t>(s) * 64 + flags] = mask;
            }
        }
        auto up = [&](auto* dst, const auto& src) {
            cuda_check(cudaMemcpy(dst, src.data(), src.size() * sizeof(src[0]), cudaMemcpyHostToDevice),
                       "upload topology");
        };
        d_nn = device_alloc<int>(fixed_owned, nn.size());
        d_nbr = device_alloc<int>(fixed_owned, nbr.size());
        d_recv_entry = device_alloc<int>(fixed_owned, recv_entry.size());
        d_sender_of = device_alloc<int>(fixed_owned, sender_of.size());
        d_shift = device_alloc<double>(fixed_owned, shift.size());
        d_dir = device_alloc<signed char>(fixed_owned, dir.size());
        d_lut = device_alloc<unsigned>(fixed_owned, lut.size());
        d_lut_empty = device_alloc<unsigned>(fixed_owned, lut.size());
        std::vector<int> coord(static_cast<std::size_t>(P));
        for (int s = 0; s < P; ++s) {
            const auto& c = coords[static_cast<std::size_t>(s)];
            coord[static_cast<std::size_t>(s)] = (c[0] << 20) | (c[1] << 10) | c[2];
        }
        d_coord = device_alloc<int>(fixed_owned, coord.size());
        up(d_nn, nn); up(d_nbr, nbr); up(d_recv_entry, recv_entry); up(d_sender_of, sender_of);
        up(d_shift, shift); up(d_dir, dir); up(d_lut, lut); up(d_coord, coord);
        up(d_lut_empty, std::vector<unsigned>(lut.size(), 0u));

        // uniform cuts (dsDecompX src/topology.cpp:63-75)
        std::vector<double> c;
        for (int a = 0; a < 3; ++a) {
            cut_offset[a] = static_cast<int>(c.size());
            const double extent = desc.upper[a] - desc.lower[a];
            for (int i = 0; i <= dims[a]; ++i)
                c.push_back(desc.lower[a] + extent * static_cast<double>(i) / static_cast<double>(dims[a]));
        }
        cuts = device_alloc<double>(fixed_owned, c.size());
        up(cuts, c);

        for (auto& l : layout) {
            l[0] = device_alloc<int>(fixed_owned, P + 1);
            l[1] = device_alloc<int>(fixed_owned, P + 1);
            l[2] = device_alloc<int>(fixed_owned, P + 1);
            cuda_check(cudaMemset(l[0], 0, sizeof(int) * (P + 1)), "memset");
            cuda_check(cudaMemset(l[1], 0, sizeof(int) * (P + 1)), "memset");
            cuda_check(cudaMemset(l[2], 0, sizeof(int) * (P + 1)), "memset");
        }
        const int tiles_cap = static_cast<int>((ncap + dsx::kTile - 1) / dsx::kTile) + P;
        for (auto& t : layout_tiles) t = device_alloc<int4>(fixed_owned, tiles_cap);
        // the status word, then the plan's totals {G, B} (S.halo_info, four
        // words): one copy brings the status and the totals to the host
        status = device_alloc<unsigned>(fixed_owned, 8);
        cuda_check(cudaMemset(status, 0, 8 * sizeof(unsigned)), "memset");
        call_counter = device_alloc<long long>(fixed_owned, 1);
        cuda_check(cudaMemset(call_counter, 0, sizeof(long long)), "memset");
        rebalance_result = device_alloc<double>(fixed_owned, 6);
        work = device_alloc<double>(fixed_owned, P);

        const int max_tiles = static_cast<int>((ncap + dsx::kTile - 1) / dsx::kTile) + P;
        S.stride = max_tiles + 1;
        // 30 counters per tile: the fused step's (28 halo + stays + emigrants)
        S.cnt = device_alloc<int>(fixed_owned, static_cast<std::size_t>(30) * S.stride);
        S.pre = device_alloc<int>(fixed_owned, static_cast<std::size_t>(30) * S.stride);
        S.cnt2 = device_alloc<int>(fixed_owned, static_cast<std::size_t>(dsx::kHaloCounters) * S.stride);
        S.pre2 = device_alloc<int>(fixed_owned, static_cast<std::size_t>(dsx::kHaloCounters) * S.stride);
        // immigrant totals, per-list, boundary and image counts in one block
        S.imm_total = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * (3 + dsx::kMaxNeighbors));
        S.imm_list = S.imm_total + P;
        S.imm_bnd = S.imm_list + static_cast<std::size_t>(P) * dsx::kMaxNeighbors;
        S.imm_img = S.imm_bnd + P;
        S.list_ret = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * E);
        S.cbase_imm = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * dsx::kHaloCounters);
        S.imm_tile_start = device_alloc<int>(fixed_owned, P + 1);
        S.ticket = device_alloc<unsigned>(fixed_owned, 1);
        cuda_check(cudaMemset(S.ticket, 0, sizeof(unsigned)), "memset");
        S.imm_tiles = device_alloc<int4>(fixed_owned, static_cast<std::size_t>(max_tiles));
        S.imm_base = device_alloc<int>(fixed_owned, P);
        S.emig_src = device_alloc<int>(fixed_owned, ncap);
        S.emig_dst = device_alloc<int>(fixed_owned, ncap);
        S.max_chunks = static_cast<int>((ncap + dsx::kTile - 1) / dsx::kTile);
        S.emig_hist = device_alloc<int>(fixed_owned, static_cast<std::size_t>(S.max_chunks) * P);
        S.emig_info = device_alloc<int>(fixed_owned, 4);
        cuda_check(cudaMemset(S.emig_info, 0, 4 * sizeof(int)), "memset");
        S.mig_results = device_alloc<long long>(fixed_owned, static_cast<std::size_t>(P) * 6);
        // per particle (per-call halo build) and per tile slot (batched step)
        const std::size_t slots = static_cast<std::size_t>(max_tiles) * dsx::kTile;
        S.mask = device_alloc<unsigned>(fixed_owned, std::max<std::size_t>(slots, static_cast<std::size_t>(ncap)));
        S.dest16 = device_alloc<unsigned short>(fixed_owned, slots);
        S.tile_bases = device_alloc<int>(fixed_owned, static_cast<std::size_t>(max_tiles) * 32);
        S.out_flags = device_alloc<int>(fixed_owned, P);
        S.list_len = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * E);
        S.send_base = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * E);
        S.g = device_alloc<int>(fixed_owned, P + 1);
        S.gbase = device_alloc<int>(fixed_owned, P + 1);
        cuda_check(cudaMemset(S.g, 0, sizeof(int) * (P + 1)), "memset");
        cuda_check(cudaMemset(S.gbase, 0, sizeof(int) * (P + 1)), "memset");
        S.bowner = device_alloc<int>(fixed_owned, ncap);
        S.boff = device_alloc<int>(fixed_owned, ncap + 1);
        S.bfirst = device_alloc<int>(fixed_owned, ncap);
        S.tile_b0 = device_alloc<int>(fixed_owned, static_cast<std::size_t>(max_tiles) + 1);
        S.cbase = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * dsx::kHaloCounters);
        S.halo_info = reinterpret_cast<int*>(status + 1);
    }

    // particle arrays [owned A | owned B | ghosts]
    // Every array holds [owned A | owned B | ghosts] plus 4 elements of
    // padding, so a tile read widened to 16-byte boundaries stays inside it.
    void allocate_arrays() {
        const std::size_t len = static_cast<std::size_t>(2 * ncap + gcap) + 4;
        for (int a = 0; a < 11; ++a) A.d[a] = device_alloc<double>(arrays_owned, len);
        A.type = device_alloc<int>(arrays_owned, len);
        A.gid = device_alloc<int>(arrays_owned, len);
        A.f.count = static_cast<int>(fields.size());
        for (std::size_t f = 0; f < fields.size(); ++f) {
            A.f.bytes[f] = fields[f].bytes;
            A.f.base[f] = device_alloc<unsigned char>(arrays_owned, len * fields[f].bytes);
        }
    }

    void allocate_ghost_scratch() {
        S.ghost_owner = device_alloc<int>(scratch_owned, gcap);
        S.ghost_entry = device_alloc<int>(scratch_owned, gcap);
        S.bslot = device_alloc<int>(scratch_owned, gcap);
    }

    // Grows the ghost region; the current owned half survives.
    void grow_ghosts(long long required, cudaStream_t stream) {
        const long long next = std::max<long long>(required + required / 2, gcap + gcap / 2);
        cuda_check(cudaStreamSynchronize(stream), "synchronize before growth");
        destroy_graphs();
        dsx::Arrays old = A;
        std::vector<void*> old_arrays;
        old_arrays.swap(arrays_owned);
        const long long off = owned_off();
        gcap = next;
        allocate_arrays();
        const std::size_t n = static_cast<std::size_t>(total);
        for (int a = 0; a < 11; ++a)
            cuda_check(cudaMemcpyAsync(A.d[a] + off, old.d[a] + off, n * sizeof(double),
                                       cudaMemcpyDeviceToDevice, stream), "grow copy");
        cuda_check(cudaMemcpyAsync(A.type + off, old.type + off, n * sizeof(int), cudaMemcpyDeviceToDevice, stream), "grow copy");
        cuda_check(cudaMemcpyAsync(A.gid + off, old.gid + off, n * sizeof(int), cudaMemcpyDeviceToDevice, stream), "grow copy");
        for (std::size_t f = 0; f < fields.size(); ++f)
            cuda_check(cudaMemcpyAsync(A.f.base[f] + off * fields[f].bytes, old.f.base[f] + off * fields[f].bytes,
                                       n * fields[f].bytes, cudaMemcpyDeviceToDevice, stream), "grow copy");
        cuda_check(cudaStreamSynchronize(stream), "grow copy");
        for (void* p : old_arrays) cudaFree(p);
        for (void* p : scratch_owned) cudaFree(p);
        scratch_owned.clear();
        allocate_ghost_scratch();
        plan_valid = false;
        ghosts_valid = false;
    }

    // -------------------------------------------------------- operations

    // Plain mode (per-call operations only): the current layout's tile starts
    // on the host, read after the work queued so far.
    const dsx::PlainLaunch* plain_layout(cudaStream_t stream) {
        if (!plain) return nullptr;
        plain_tiles = read_ints(layout[cur][2], P + 1, stream);
        plain_launch.tile_start = plain_tiles.data();
        plain_launch.boundary_start = nullptr;
        return &plain_launch;
    }

    // Plain mode after a plan build: where each subdomain's boundary owners
    // start (the reverse sum is then launched per subdomain).
    void plain_boundaries(cudaStream_t stream) {
        if (!plain) return;
        const std::vector<int> cb = read_ints(S.cbase, P * dsx::kHaloCounters, stream);
        const std::vector<int> info = read_ints(S.halo_info, 2, stream);
        plain_bounds.assign(static_cast<std::size_t>(P) + 1, 0);
        for (int r = 0; r < P; ++r)
            plain_bounds[static_cast<std::size_t>(r)] =
                cb[static_cast<std::size_t>(r) * dsx::kHaloCounters + dsx::kBoundaryCounter];
        plain_bounds[static_cast<std::size_t>(P)] = info[1];
    }

    // first_of_step: the batched step's rebalance, which also clears the
    // status word and the step's immigrant counters (their memsets skipped)
    void enqueue_rebalance(cudaStream_t stream, bool automatic_rebalance,
                           const double* work_in = nullptr, bool first_of_step = false) {
        const dsx::Grid G = params();
        if (desc.policy == DSX_DYNAMIC) {
            // Decomp::migrate: ++migration_calls, automatic rebalance every
            // `interval` calls unless called from rebalance()
            // (dsDecompX src/runtime.cpp:983-993)
            dsx::RebalanceParams p;
            p.threshold = desc.dyn_threshold;
            p.relaxation = desc.dyn_relaxation;
            p.minimum_fraction = desc.dyn_min_fraction;
            p.halo_width = halo_width;
            p.automatic = 1;
            p.interval = automatic_rebalance ? static_cast<long long>(desc.dyn_interval) : 0;
            if (first_of_step) {
                p.clear_status = 1;
                p.zero = S.imm_total;
                p.nzero = P * (3 + dsx::kMaxNeighbors);
            }
            dsx::launch_rebalance(G, work_in, p, call_counter, rebalance_result, stream);
            dsx::mark(S, stream, "rebalance");
        }
    }

    void commit_migrate() {
        sharded_ghosts = false;
        pairs_valid = true;
        plain_bounds.clear();
        parity ^= 1;
        cur ^= 1;
        ++layout_version;
        plan_valid = false;
        ghosts_valid = false;
        std::fill(last_ghosts.begin(), last_ghosts.end(), 0);
    }

    void enqueue_halo_build(cudaStream_t stream, const dsx::PlainLaunch* pl = nullptr) {
        dsx::launch_halo_build(params(), A, owned_off(), ghost_off(), S, stream, pl);
    }

    void enqueue_reverse(cudaStream_t stream, const dsx::PlainLaunch* pl = nullptr) {
        const long long o = owned_off(), g = ghost_off();
        dsx::launch_reverse_sum3(params(), A.d[6] + o, A.d[7] + o, A.d[8] + o, A.d[6] + g, A.d[7] + g,
                                 A.d[8] + g, S, stream, pl);
    }

    unsigned read_status(cudaStream_t stream) {
        cuda_check(cudaMemcpyAsync(pinned_status, status, 3 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                   stream), "read status");
        cuda_check(cudaStreamSynchronize(stream), "synchronize");
        return pinned_status[0];
    }

    void clear_status(cudaStream_t stream) {
        cuda_check(cudaMemsetAsync(status, 0, sizeof(unsigned), stream), "clear status");
    }

    std::vector<int> read_ints(const int* device, int count, cudaStream_t stream) {
        std::vector<int> out(static_cast<std::size_t>(count));
        cuda_check(cudaMemcpyAsync(out.data(), device, sizeof(int) * count, cudaMemcpyDeviceToHost, stream), "read");
        cuda_check(cudaStreamSynchronize(stream), "synchronize");
        return out;
    }

    void migrate(cudaStream_t stream, long long* results, bool automatic_rebalance = true) {
        not_pending("migrate");
        clear_status(stream);
        // work supplied for this migrate's automatic rebalance (pageable
        // source: the copy is staged before the call returns)
        const double* work_in = nullptr;
        if (!next_work.empty()) {
            cuda_check(cudaMemcpyAsync(work, next_work.data(), sizeof(double) * P,
                                       cudaMemcpyHostToDevice, stream), "upload work");
            work_in = work;
            next_work.clear();
        }
        if (plain) {
            // the rebalance may move the cut planes but not the layout
            enqueue_rebalance(stream, automatic_rebalance, work_in);
            dsx::launch_migrate(params(), A, owned_off(), next_off(), S, stream,
                                plain_layout(stream));
        } else {
            enqueue_rebalance(stream, automatic_rebalance, work_in);
            // the batched step's classify, layout and staged move over an
            // empty halo table: every halo mask is 0, so the pipeline lays
            // out and writes no ghost and leaves what migrate alone leaves
            // (the old layout's plan is dropped either way)
            dsx::Grid G = params();
            G.lut = d_lut_empty;
            dsx::launch_step_classify(G, A, owned_off(), S, stream);
            dsx::launch_step_layout(G, S, stream);
            dsx::launch_step_move(G, A, owned_off(), next_off(), ghost_off(), S, stream);
            dsx::launch_step_emigrants(G, A, owned_off(), next_off(), S, S.imm_total, nullptr, stream);
        }
        commit_migrate();
        if (results) {
            cuda_check(cudaMemcpyAsync(results, S.mig_results, sizeof(long long) * 6 * P,
                                       cudaMemcpyDeviceToHost, stream), "read migration results");
            const unsigned st = read_status(stream);
            if (st & dsx::kStatusMigrationMismatch) fail(DSX_E_RUNTIME, "migration count mismatch");
            if (st & dsx::kStatusCutsInvalid)
                fail(DSX_E_INVALID, "dynamic cuts must be strictly increasing and span the domain");
        }
    }

    // Builds the plan; grows the ghost region and rebuilds when it overflowed.
    void build_checked(cudaStream_t stream) {
        sharded_ghosts = false;
        for (;;) {
            clear_status(stream);
            enqueue_halo_build(stream, plain_layout(stream));
            const unsigned st = read_status(stream);
            if (st & dsx::kStatusCopyTimeout)
                fail(DSX_E_RUNTIME, "a bulk copy of particle records did not complete within 1 s");
            if (!(st & dsx::kStatusGhostOverflow)) break;
            grow_ghosts(static_cast<long long>(static_cast<int>(pinned_status[1])), stream);
        }
        plan_valid = true;
        ghosts_valid = true;
        plain_boundaries(stream);
    }

    void exchange_halo(bool rebuild, bool positions_only, cudaStream_t stream, long long* results) {
        not_pending("exchange_halo");
        sharded_ghosts = false;
        if (rebuild) plan_valid = false;
        bool reused = false;
        if (P == 1) {
            // one rank owns the whole periodic box: no ghosts (dsDecompX src/halo.cpp:325-350)
            plan_valid = false;
            ghosts_valid = false;
        } else if (plan_valid) {
            dsx::launch_halo_refresh(params(), A, owned_off(), ghost_off(), positions_only, S, stream);
            reused = true;
        } else if (results) {
            build_checked(stream);
        } else {
            clear_status(stream);
            enqueue_halo_build(stream);
            plain_bounds.clear();
            plan_valid = true;
            ghosts_valid = true;
        }
        report_halo(rebuild, reused, stream, results);
    }

    // Per subdomain {ghosts, layout changed, storage reallocated, plan reused}.
    void report_halo(bool rebuild, bool reused, cudaStream_t stream, long long* results) {
        if (results) {
            std::vector<int> g(static_cast<std::size_t>(P), 0);
            if (ghosts_valid) g = read_ints(S.g, P, stream);
            for (int s = 0; s < P; ++s) {
                const long long now = ghosts_valid ? g[static_cast<std::size_t>(s)] : 0;
                long long* o = results + 4 * s;
                o[0] = now;
                o[1] = (rebuild || now != last_ghosts[static_cast<std::size_t>(s)] || (now != 0 && !reused)) ? 1 : 0;
                o[2] = 0;
                o[3] = reused ? 1 : 0;
                last_ghosts[static_cast<std::size_t>(s)] = now;
            }
        } else if (!ghosts_valid) {
            std::fill(last_ghosts.begin(), last_ghosts.end(), 0);
        }
    }

    // Split-phase halo (Decomp::begin_halo_exchange / end_halo_exchange,
    // dsDecompX src/halo.cpp:296-872): begin enqueues the refresh or one
    // build attempt on the stream and returns; work on other streams can run
    // meanwhile; end waits, grows the ghost region and rebuilds after an
    // overflow, and returns the counts.  Nothing else may run on the grid in
    // between (the reference's logic_error).
    bool halo_pending = false, pending_rebuild = false, pending_reused = false, pending_build = false;

    void not_pending(const char* what) {
        settle_async();
        if (halo_pending)
            fail(DSX_E_LOGIC, std::string(what) + " while a split halo exchange is in progress");
    }

    // Segment 1 is a captured graph on an explicit stream (the default
    // streams cannot capture; plain mode reads layouts on the host): one
    // launch, and begin returns.  Refreshes use split_ctas_per_sm (0: every
    // resident CTA) so that interior work on other streams finds SM room.
    void begin_halo(bool rebuild, bool positions_only, cudaStream_t stream) {
        not_pending("begin_halo_exchange");
        sharded_ghosts = false;
        if (rebuild) plan_valid = false;
        pending_rebuild = rebuild;
        pending_reused = false;
        pending_build = false;
        const bool graphs = capturable(stream) && !plain;
        if (P == 1) {
            plan_valid = false;
            ghosts_valid = false;
        } else if (plan_valid) {
            auto enqueue = [&] {
                dsx::launch_halo_refresh(params(), A, owned_off(), ghost_off(), positions_only, S,
                                         stream, split_ctas_per_sm);
            };
            if (graphs) run_captured(split_begin[positions_only ? 1 : 0][parity], stream, enqueue);
            else enqueue();
            pending_reused = true;
        } else {
            if (graphs) {
                run_captured(split_begin[2][parity], stream, [&] {
                    clear_status(stream);
                    enqueue_halo_build(stream);
                });
                plain_bounds.clear();
            } else {
                clear_status(stream);
                enqueue_halo_build(stream, plain_layout(stream));
            }
            pending_build = true;
        }
        pending_graphs = graphs;
        halo_pending = true;
    }

    bool pending_graphs = false;

    void end_halo(cudaStream_t stream, long long* results) {
        if (!halo_pending) fail(DSX_E_LOGIC, "end_halo_exchange without begin_halo_exchange");
        halo_pending = false;
        if (pending_build) {
            unsigned st;
            if (pending_graphs) {
                // segment 2: the build's status and totals to the host
                run_captured(split_end[parity], stream, [&] {
                    cuda_check(cudaMemcpyAsync(pinned_status, status, 3 * sizeof(unsigned),
                                               cudaMemcpyDeviceToHost, stream), "read status");
                });
                cuda_check(cudaStreamSynchronize(stream), "synchronize");
                st = pinned_status[0];
            } else {
                st = read_status(stream);
            }
            if (st & dsx::kStatusCopyTimeout)
                fail(DSX_E_RUNTIME, "a bulk copy of particle records did not complete within 1 s");
            if (st & dsx::kStatusGhostOverflow) {
                grow_ghosts(static_cast<long long>(static_cast<int>(pinned_status[1])), stream);
                build_checked(stream);
            } else {
                plan_valid = true;
                ghosts_valid = true;
                plain_boundaries(stream);
            }
        }
        report_halo(pending_rebuild, pending_reused, stream, results);
    }

    void reverse_halo(cudaStream_t stream) {
        not_pending("reverse_halo");
        if (P == 1 || !ghosts_valid) return;
        if (plain && static_cast<int>(plain_bounds.size()) == P + 1) {
            plain_launch.boundary_start = plain_bounds.data();
            enqueue_reverse(stream, &plain_launch);
        } else {
            enqueue_reverse(stream);
        }
    }

    dsx::FieldOps field_ops(int nf, const int* ids, const int* ops, const char* what) {
        if (nf > dsx::kMaxFields) fail(DSX_E_INVALID, std::string("at most 16 fields can be ") + what);
        dsx::FieldOps F;
        F.count = nf;
        for (int i = 0; i < nf; ++i) {
            if (!ids || ids[i] < 0 || ids[i] >= static_cast<int>(fields.size()))
                fail(DSX_E_INVALID, std::string("missing or undersized ") + what + " field");
            for (int j = 0; j < i; ++j)
                if (ids[j] == ids[i])
                    fail(DSX_E_INVALID, std::string("duplicate ") + what + " field '" +
                                            fields[static_cast<std::size_t>(ids[i])].name + "'");
            const Field& f = fields[static_cast<std::size_t>(ids[i])];
            F.index[i] = ids[i];
            F.type[i] = f.type;
            F.components[i] = f.components;
            F.op[i] = ops ? ops[i] : DSX_REPLACE;
            if (F.op[i] < DSX_SUM || F.op[i] > DSX_REPLACE) fail(DSX_E_INVALID, "unknown reduce operation");
        }
        return F;
    }

    void reverse_exchange(int nf, const int* ids, const int* ops, cudaStream_t stream) {
        not_pending("reverse_exchange");
        if (sharded_ghosts)
            fail(DSX_E_LOGIC, "a sharded step's ghosts exchange fields through dsx_shard_reverse_exchange");
        const dsx::FieldOps F = field_ops(nf, ids, ops, "reverse-exchanged");
        if (P == 1 || !ghosts_valid || nf == 0) return;
        dsx::launch_reverse_fields(params(), A, owned_off(), ghost_off(), F, S, stream);
    }

    void forward_exchange(int nf, const int* ids, cudaStream_t stream) {
        not_pending("forward_exchange");
        if (sharded_ghosts)
            fail(DSX_E_LOGIC, "a sharded step's ghosts exchange fields through dsx_shard_forward_exchange");
        const dsx::FieldOps F = field_ops(nf, ids, nullptr, "forward-exchanged");
        if (P == 1 || !ghosts_valid || nf == 0) return;
        dsx::launch_forward_fields(params(), A, owned_off(), ghost_off(), F, S, stream);
    }

    void rebalance(const double* host_work, bool force, cudaStream_t stream, long long* results,
                   double* imbalance) {
        not_pending("rebalance");
        if (host_work) {
            for (int s = 0; s < P; ++s)
                if (!std::isfinite(host_work[s]) || host_work[s] < 0.0)
                    fail(DSX_E_INVALID, "rebalance local_work must be finite and non-negative");
            cuda_check(cudaMemcpyAsync(work, host_work, sizeof(double) * P, cudaMemcpyHostToDevice, stream),
                       "upload work");
        }
        clear_status(stream);
        dsx::RebalanceParams p;
        p.threshold = desc.dyn_threshold;
        p.relaxation = desc.dyn_relaxation;
        p.minimum_fraction = desc.dyn_min_fraction;
        p.halo_width = halo_width;
        p.force = force ? 1 : 0;
        p.automatic = 0;
        dsx::launch_rebalance(params(), host_work ? work : nullptr, p, call_counter, rebalance_result + 3, stream);
        double r[3] = {0, 0, 1};
        cuda_check(cudaMemcpyAsync(r, rebalance_result + 3, sizeof(r), cudaMemcpyDeviceToHost, stream), "read");
        const unsigned st = read_status(stream);
        if (st & dsx::kStatusCutsInvalid)
            fail(DSX_E_INVALID, "dynamic cuts must be strictly increasing and span the domain");
        if (r[1] != 0.0) plan_valid = false;
        std::vector<long long> mig(static_cast<std::size_t>(6 * P));
        migrate(stream, mig.data(), false);
        for (int s = 0; s < P; ++s) {
            if (results) {
                results[3 * s + 0] = r[0] != 0.0;
                results[3 * s + 1] = r[1] != 0.0;
                results[3 * s + 2] = mig[static_cast<std::size_t>(6 * s + 5)];
            }
            if (imbalance) imbalance[s] = r[2];
        }
    }

    dsx_grid_view view() const {
        dsx_grid_view v{};
        for (int a = 0; a < 11; ++a) v.base[a] = A.d[a];
        v.base[11] = A.type;
        v.base[12] = A.gid;
        for (std::size_t f = 0; f < fields.size(); ++f) v.base[13 + f] = A.f.base[f];
        v.owned_offset = owned_off();
        v.ghost_offset = ghost_off();
        v.n = layout[cur][0];
        v.obase = layout[cur][1];
        v.g = S.g;
        v.gbase = S.gbase;
        v.halo_totals = S.halo_info;
        v.particles = total;
        v.ghost_capacity = gcap;
        v.nranks = P;
        return v;
    }

    void enqueue_step(dsx_step_callback cb, void* user, cudaStream_t stream, bool build_event = false) {
        marks.count = 0;
        // a Dynamic grid's rebalance opens the step and clears the status and
        // the immigrant counters itself
        const bool dynamic = desc.policy == DSX_DYNAMIC;
        if (!dynamic) clear_status(stream);
        marks.mark(stream, "start");
        enqueue_rebalance(stream, true, nullptr, dynamic);
        {
            const dsx::Grid G = params();
            cur ^= 1;
            const dsx::Grid Gn = params();
            cur ^= 1;
            dsx::launch_fused_step(G, Gn, A, owned_off(), next_off(), ghost_off(), S, stream, dynamic);
        }
        if (build_event) {
            // the build's status and totals, then the event the next
            // asynchronous step waits on (an event node of the graph), on a
            // branch that joins the step again after the reverse sum
            unsigned* out = pinned_build + 4 * parity;
            cuda_check(cudaEventRecord(fork_ev, stream), "fork");
            cuda_check(cudaStreamWaitEvent(side_stream, fork_ev, 0), "fork");
            cuda_check(cudaMemcpyAsync(out, status, 3 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                       side_stream), "read build status");
            cuda_check(cudaEventRecordWithFlags(build_done[parity], side_stream, cudaEventRecordExternal),
                       "record build event");
            cuda_check(cudaEventRecord(join_ev, side_stream), "join");
        }
        // the rest of the step reads the next layout
        parity ^= 1;
        cur ^= 1;
        const dsx_grid_view v = view();
        // inside the callback the new plan is the current one (field
        // exchanges called from it act on these ghosts)
        const bool saved_plan = plan_valid, saved_ghosts = ghosts_valid;
        plan_valid = ghosts_valid = true;
        if (cb) cb(user, stream, &v);
        plan_valid = saved_plan;
        ghosts_valid = saved_ghosts;
        marks.mark(stream, "callback");
        enqueue_reverse(stream);
        // the status after the build is the step's (nothing later sets a
        // bit): a step with the build's copy needs no second one
        if (!build_event)
            cuda_check(cudaMemcpyAsync(pinned_status, status, 3 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                       stream), "read status");
        else
            cuda_check(cudaStreamWaitEvent(stream, join_ev, 0), "join");
        parity ^= 1;
        cur ^= 1;
        ++layout_version;
    }

    // Decomposition::set_axis_cuts (dsDecompX src/decomp.cpp:146-163): the
    // cuts must span the domain and increase strictly; the plan is invalid.
    void set_cuts(const double* host, cudaStream_t stream) {
        not_pending("set_cuts");
        int total_cuts = 0;
        for (int a = 0; a < 3; ++a) {
            const double* c = host + total_cuts;
            bool ok = c[0] == desc.lower[a] && c[dims[a]] == desc.upper[a];
            for (int i = 0; i < dims[a]; ++i) ok = ok && c[i] < c[i + 1];
            if (!ok) fail(DSX_E_INVALID, "dynamic cuts must be strictly increasing and span the domain");
            total_cuts += dims[a] + 1;
        }
        cuda_check(cudaStreamSynchronize(stream), "synchronize before new cuts");
        cuda_check(cudaMemcpy(cuts, host, sizeof(double) * total_cuts, cudaMemcpyHostToDevice), "upload cuts");
        plan_valid = false;
        ghosts_valid = false;
    }

    // Decomposition::rescale_domain / update_domain (dsDecompX
    // src/decomp.cpp:104-144): every cut keeps its fraction of the extent and
    // the periodic shifts follow the new extent; rescale keeps the halo plan
    // (same grid, same neighbours: a refresh uses the new shifts), update
    // invalidates it.  Positions are the caller's.
    void rescale_domain(const double* lower, const double* upper, bool invalidate,
                        cudaStream_t stream) {
        not_pending("rescale_domain");
        for (int a = 0; a < 3; ++a)
            if (!(upper[a] > lower[a])) fail(DSX_E_INVALID, "global-domain extent must be positive");
        const int total_cuts = dims[0] + dims[1] + dims[2] + 3;
        std::vector<double> c(static_cast<std::size_t>(total_cuts));
        cuda_check(cudaStreamSynchronize(stream), "synchronize before rescale");
        cuda_check(cudaMemcpy(c.data(), cuts, sizeof(double) * total_cuts, cudaMemcpyDeviceToHost), "read cuts");
        for (int a = 0, off = 0; a < 3; off += dims[a] + 1, ++a) {
            const double old_extent = desc.upper[a] - desc.lower[a];
            const double new_extent = upper[a] - lower[a];
            for (int i = 0; i <= dims[a]; ++i) {
                double& cut = c[static_cast<std::size_t>(off + i)];
                const double fraction = (cut - desc.lower[a]) / old_extent;
                cut = lower[a] + fraction * new_extent;
            }
        }
        for (int a = 0; a < 3; ++a) {
            desc.lower[a] = lower[a];
            desc.upper[a] = upper[a];
        }
        cuda_check(cudaMemcpy(cuts, c.data(), sizeof(double) * total_cuts, cudaMemcpyHostToDevice), "upload cuts");
        build_topology();
        const int E = dsx::kMaxNeighbors;
        std::vector<double> shift(static_cast<std::size_t>(P) * E * 3, 0.0);
        for (int s = 0; s < P; ++s) {
            const auto& list = topo[static_cast<std::size_t>(s)];
            for (std::size_t n = 0; n < list.size(); ++n)
                for (int a = 0; a < 3; ++a)
                    shift[3 * (static_cast<std::size_t>(s) * E + n) + a] = list[n].shift[a];
        }
        cuda_check(cudaMemcpy(d_shift, shift.data(), sizeof(double) * shift.size(), cudaMemcpyHostToDevice),
                   "upload shifts");
        destroy_graphs();   // captured kernels hold the old box
        if (invalidate) {
            plan_valid = false;
            ghosts_valid = false;
        }
    }

    // ------------------------------------------------ sharded grids

    // Emigrants of the last migration (per call or batched step) counted per
    // (destination, source), dest-major.
    void migration_pairs(long long* out, cudaStream_t stream) {
        not_pending("migration_pairs");
        if (!pairs_valid) fail(DSX_E_LOGIC, "no migration since the particles were last replaced");
        if (!pairs) pairs = device_alloc<int>(fixed_owned, static_cast<std::size_t>(P) * P);
        dsx::launch_pair_counts(P, S, layout[cur ^ 1][1], ncap, pairs, stream);
        const std::vector<int> h = read_ints(pairs, P * P, stream);
        for (std::size_t i = 0; i < h.size(); ++i) out[i] = h[i];
    }

    // Length and first ghost slot of every send list (sender-major, 26 per
    // sender) of the current plan.
    void send_lists(int* len, int* base, cudaStream_t stream) {
        not_pending("send_lists");
        const std::size_t n = static_cast<std::size_t>(P) * dsx::kMaxNeighbors;
        if (!ghosts_valid || P == 1) {
            std::fill(len, len + n, 0);
            std::fill(base, base + n, 0);
            return;
        }
        cuda_check(cudaMemcpyAsync(len, S.list_len, sizeof(int) * n, cudaMemcpyDeviceToHost, stream), "read");
        cuda_check(cudaMemcpyAsync(base, S.send_base, sizeof(int) * n, cudaMemcpyDeviceToHost, stream), "read");
        cuda_check(cudaStreamSynchronize(stream), "synchronize");
    }

    // The next owned half from segments of the current half and of outside
    // buffers, then the halves swap: counts[P] are the new owned counts; a
    // segment copies `count` records of every array from source `source`
    // (-1: the current owned half; k >= 0: sources[32 k + a] is array a's
    // element 0) at src_index to subdomain dst_rank at dst_index.
    void assemble(const long long* counts, int nsources, const void* const* sources, long long nseg,
                  const dsx_segment* segs, cudaStream_t stream) {
        not_pending("assemble");
        std::vector<long long> ob(static_cast<std::size_t>(P) + 1, 0);
        for (int s = 0; s < P; ++s) {
            if (counts[s] < 0 || counts[s] > INT_MAX) fail(DSX_E_INVALID, "particle count out of range");
            ob[static_cast<std::size_t>(s) + 1] = ob[static_cast<std::size_t>(s)] + counts[s];
        }
        const long long sum = ob[static_cast<std::size_t>(P)];
        if (sum > ncap) fail(DSX_E_LENGTH, "particle storage is smaller than the assembled counts");
        const int narrays = 13 + static_cast<int>(fields.size());
        long long bytes[32];
        unsigned char* dst_base[32];
        const long long src_off = owned_off(), dst_off = next_off();
        unsigned char* cur_base[32];
        for (int a = 0; a < narrays; ++a) {
            bytes[a] = a < 11 ? 8 : a < 13 ? 4 : fields[static_cast<std::size_t>(a - 13)].bytes;
            unsigned char* b = static_cast<unsigned char*>(
                a < 11 ? static_cast<void*>(A.d[a]) : a == 11 ? static_cast<void*>(A.type) :
                a == 12 ? static_cast<void*>(A.gid) : static_cast<void*>(A.f.base[a - 13]));
            dst_base[a] = b + dst_off * bytes[a];
            cur_base[a] = b + src_off * bytes[a];
        }
        std::vector<dsx::CopyPiece> copies;
        for (long long k = 0; k < nseg; ++k) {
            const dsx_segment& g = segs[k];
            if (g.count < 0 || g.src_index < 0 || g.dst_index < 0 || g.dst_rank < 0 || g.dst_rank >= P ||
                g.source < -1 || g.source >= nsources)
                fail(DSX_E_INVALID, "segment out of range");
            if (g.dst_index + g.count > counts[g.dst_rank])
                fail(DSX_E_INVALID, "segment past the end of its subdomain");
            if (g.source == -1 && g.src_index + g.count > total)
                fail(DSX_E_INVALID, "segment past the end of the owned particles");
            if (!g.count) continue;
            for (int a = 0; a < narrays; ++a) {
                const unsigned char* src =
                    g.source < 0 ? cur_base[a]
                                 : static_cast<const unsigned char*>(sources[32 * g.source + a]);
                if (!src) fail(DSX_E_INVALID, "null source array");
                copies.push_back({src + g.src_index * bytes[a],
                                  dst_base[a] + (ob[static_cast<std::size_t>(g.dst_rank)] + g.dst_index) * bytes[a],
                                  g.count * bytes[a]});
            }
        }
        cuda_check(dsx::launch_copies(copies, stream), "assemble copies");
        std::vector<int> c(static_cast<std::size_t>(P) + 1, 0);
        for (int s = 0; s < P; ++s) c[static_cast<std::size_t>(s)] = static_cast<int>(counts[s]);
        const int next = cur ^ 1;
        cuda_check(cudaMemcpyAsync(layout[next][0], c.data(), sizeof(int) * (P + 1), cudaMemcpyHostToDevice,
                                   stream), "assemble counts");
        cur ^= 1;
        ++layout_version;
        dsx::launch_layout(params(), layout[cur][0], layout[cur][1], layout[cur][2], layout_tiles[cur], stream);
        parity ^= 1;
        total = sum;
        plan_valid = false;
        ghosts_valid = false;
        pairs_valid = false;
        plain_bounds.clear();
        std::fill(last_ghosts.begin(), last_ghosts.end(), 0);
        cuda_check(cudaMemsetAsync(S.g, 0, sizeof(int) * (P + 1), stream), "memset");
        cuda_check(cudaMemsetAsync(S.gbase, 0, sizeof(int) * (P + 1), stream), "memset");
        cuda_check(cudaMemsetAsync(S.halo_info, 0, sizeof(int) * 4, stream), "memset");
        cuda_check(cudaStreamSynchronize(stream), "assemble");
    }

    void set_rebalance_work(const double* host_work) {
        if (!host_work) {
            next_work.clear();
            return;
        }
        for (int s = 0; s < P; ++s)
            if (!std::isfinite(host_work[s]) || host_work[s] < 0.0)
                fail(DSX_E_INVALID, "rebalance work must be finite and non-negative");
        next_work.assign(host_work, host_work + P);
    }

    // Replays the step's idempotent parts on the current particles (the
    // current owned half is only read) and keeps the fastest launch shapes.
    void autotune(cudaStream_t stream, dsx_tune_report* out) {
        not_pending("autotune");
        dsx_tune_report r{};
        for (float& v : r.classify_ms) v = -1.0f;
        for (float& v : r.classify_combined_ms) v = -1.0f;
        for (float& v : r.move_ms) v = -1.0f;
        for (float& v : r.reverse_ms) v = -1.0f;
        if (P > 1 && total > 0) {
            cuda_check(cudaStreamSynchronize(stream), "synchronize before tuning");
            destroy_graphs();
            dsx::Marks* saved_marks = S.marks;
            S.marks = nullptr;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
            cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
            auto time = [&](auto&& launch) {
                constexpr int kReps = 5;
                launch();
                cuda_check(cudaEventRecord(e0, stream), "record");
                for (int i = 0; i < kReps; ++i) launch();
                cuda_check(cudaEventRecord(e1, stream), "record");
                cuda_check(cudaEventSynchronize(e1), "synchronize");
                float ms = 0.0f;
                cuda_check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
                return ms / kReps;
            };
            auto pick = [](const float* ms, const int* value, int n, int fallback) {
                int best = fallback;
                float t = -1.0f;
                for (int i = 0; i < n; ++i)
                    if (ms[i] >= 0.0f && (t < 0.0f || ms[i] < t)) {
                        t = ms[i];
                        best = value[i];
                    }
                return best;
            };
            const long long src = owned_off(), dst = next_off();
            auto grids = [&](dsx::Grid& G, dsx::Grid& Gn) {
                G = params();
                cur ^= 1;
                Gn = params();
                cur ^= 1;
            };
            dsx::Grid G, Gn;
            grids(G, Gn);
            clear_status(stream);
            const int shapes[3] = {64, 128, 256};
            float best_classify = -1.0f;
            int best_threads = 128, best_combine = 0;
            for (int c = 0; c < 2; ++c)
                for (int i = 0; i < 3; ++i) {
                    S.classify_threads = shapes[i];
                    S.classify_combine = c;
                    const float ms = time([&] { dsx::launch_step_classify(G, A, src, S, stream); });
                    (c ? r.classify_combined_ms : r.classify_ms)[i] = ms;
                    if (best_classify < 0.0f || ms < best_classify) {
                        best_classify = ms;
                        best_threads = shapes[i];
                        best_combine = c;
                    }
                }
            S.classify_threads = best_threads;
            S.classify_combine = best_combine;
            // the next layout's plan; the ghost region grows until it fits
            for (;;) {
                clear_status(stream);
                dsx::launch_step_classify(G, A, src, S, stream);
                dsx::launch_step_layout(G, S, stream);
                const unsigned st = read_status(stream);
                if (!(st & dsx::kStatusGhostOverflow)) break;
                grow_ghosts(static_cast<long long>(static_cast<int>(pinned_status[1])), stream);
                grids(G, Gn);
            }
            const long long gho = ghost_off();
            // staged, direct reads, staged in passes, staged without forces
            const int kinds[4] = {1, 0, 2, 3};
            const int bits[4] = {2, 1, 4, 8};
            const int modes = dsx::staged_move_modes(A);
            for (int i = 0; i < 4; ++i) {
                if (!(modes & bits[i])) continue;
                S.move_staged = kinds[i];
                r.move_ms[i] = time([&] { dsx::launch_step_move(G, A, src, dst, gho, S, stream); });
            }
            S.move_staged = pick(r.move_ms, kinds, 4, 1);
            dsx::launch_step_move(G, A, src, dst, gho, S, stream);
            dsx::launch_step_finish(G, Gn, A, src, dst, gho, S, stream);
            // the reverse sum into the next half's forces from the ghost
            // region: both are rewritten by the next step
            const int per_sm[4] = {4, 8, 16, 32};
            for (int i = 0; i < 4; ++i) {
                S.reverse_per_sm = per_sm[i];
                r.reverse_ms[i] = time([&] {
                    dsx::launch_reverse_sum3(Gn, A.d[6] + dst, A.d[7] + dst, A.d[8] + dst, A.d[6] + gho,
                                             A.d[7] + gho, A.d[8] + gho, S, stream);
                });
            }
            S.reverse_per_sm = pick(r.reverse_ms, per_sm, 4, 0);
            const unsigned st = read_status(stream);
            const long long ghosts = static_cast<int>(pinned_status[1]);
            if (!(st & dsx::kStatusGhostOverflow) && gcap < ghosts + ghosts / 4)
                grow_ghosts(ghosts + ghosts / 4, stream);
            clear_status(stream);
            cuda_check(cudaStreamSynchronize(stream), "synchronize after tuning");
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            S.marks = saved_marks;
            plan_valid = false;
            ghosts_valid = false;
            destroy_graphs();
        }
        r.classify_threads = S.classify_threads;
        r.classify_combine = S.classify_combine;
        r.move_staged = S.move_staged;
        r.reverse_ctas_per_sm = S.reverse_per_sm;
        r.ghost_capacity = gcap;
        if (out) *out = r;
    }

    void step(dsx_step_callback cb, void* user, bool capture, cudaStream_t stream, unsigned* status_out) {
        not_pending("the batched step");
        if (capture && (graph_callback != cb || graph_user != user || graph_stream != stream)) {
            destroy_graphs();
            graph_callback = cb;
            graph_user = user;
            graph_stream = stream;
        }
        // where the step's status lands: the build's copy of a captured
        // step (per owned half), else the copy at the end of the step
        const unsigned* st_at = capture ? pinned_build + 4 * parity : pinned_status;
        if (capture) {
            cudaGraphExec_t& exec = graph[parity];
            if (!exec) {
                cudaGraph_t g = nullptr;
                cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
                enqueue_step(cb, user, stream, true);
                cuda_check(cudaStreamEndCapture(stream, &g), "end capture");
                cuda_check(cudaGraphInstantiate(&exec, g, 0), "instantiate graph");
                cudaGraphDestroy(g);
            }
            cuda_check(cudaGraphLaunch(exec, stream), "launch graph");
        } else {
            enqueue_step(cb, user, stream);
        }
        commit_migrate();
        plan_valid = true;
        ghosts_valid = true;
        cuda_check(cudaStreamSynchronize(stream), "synchronize step");
        const unsigned st = finish_step(st_at[0], static_cast<int>(st_at[1]), cb, user, stream);
        if (status_out) *status_out = st;
    }

    // A step whose graph has run: after a ghost-region overflow the owned
    // half is intact, so the capacity grows and the halo build, the callback
    // and the reverse sum are redone; other failures raise.
    unsigned finish_step(unsigned st, int ghosts_needed, dsx_step_callback cb, void* user,
                         cudaStream_t stream) {
        if (st & dsx::kStatusGhostOverflow) {
            grow_ghosts(static_cast<long long>(ghosts_needed), stream);
            build_checked(stream);
            const dsx_grid_view v = view();
            if (cb) cb(user, stream, &v);
            enqueue_reverse(stream);
            st = read_status(stream);
        }
        if (st & dsx::kStatusCopyTimeout)
            fail(DSX_E_RUNTIME, "a bulk copy of particle records did not complete within 1 s");
        if (st & dsx::kStatusMigrationMismatch) fail(DSX_E_RUNTIME, "migration count mismatch");
        if (st & dsx::kStatusCutsInvalid)
            fail(DSX_E_INVALID, "dynamic cuts must be strictly increasing and span the domain");
        return st;
    }

    // Asynchronous batched steps: the step's graph is queued and the call
    // returns.  Before it is queued, the previous asynchronous step's build
    // status is read at that step's build event (its callback and reverse
    // sum may still be running), so the GPU always has the next step in line
    // and a failed build is handled (grown and redone, as in step) before
    // anything builds on it.
    void step_async(dsx_step_callback cb, void* user, cudaStream_t stream) {
        if (halo_pending)
            fail(DSX_E_LOGIC, "the batched step while a split halo exchange is in progress");
        if (async_inflight && async_stream != stream) settle_async();
        if (graph_callback != cb || graph_user != user || graph_stream != stream) {
            destroy_graphs();   // settles a pending step first
            graph_callback = cb;
            graph_user = user;
            graph_stream = stream;
        }
        if (async_inflight) check_async();
        cudaGraphExec_t& exec = graph[parity];
        if (!exec) {
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            enqueue_step(cb, user, stream, true);
            cuda_check(cudaStreamEndCapture(stream, &g), "end capture");
            cuda_check(cudaGraphInstantiate(&exec, g, 0), "instantiate graph");
            cudaGraphDestroy(g);
        }
        const int p = parity;
        cuda_check(cudaGraphLaunch(exec, stream), "launch graph");
        commit_migrate();
        plan_valid = true;
        ghosts_valid = true;
        async_inflight = true;
        async_parity = p;
        async_stream = stream;
    }

    // The pending asynchronous step's build, checked at its event.
    void check_async() {
        async_inflight = false;
        cuda_check(cudaEventSynchronize(build_done[async_parity]), "wait for the step's build");
        const unsigned* b = pinned_build + 4 * async_parity;
        unsigned st = b[0];
        const unsigned failed = dsx::kStatusGhostOverflow | dsx::kStatusCopyTimeout |
                                dsx::kStatusMigrationMismatch | dsx::kStatusCutsInvalid;
        if (st & failed) {
            cuda_check(cudaStreamSynchronize(async_stream), "synchronize step");
            st = finish_step(st, static_cast<int>(b[1]), graph_callback, graph_user, async_stream);
        }
        async_status |= st;
    }

    // Every other call first completes the pending asynchronous step.
    void settle_async() {
        if (!async_inflight) return;
        check_async();
        cuda_check(cudaStreamSynchronize(async_stream), "synchronize step");
    }

    unsigned step_wait() {
        settle_async();
        const unsigned st = async_status;
        async_status = 0;
        return st;
    }

    // ------------------------------------------------------ sharded step
    // One fused step of a grid that holds only the subdomains t with
    // owners[t] == shard, as one process of a sharded grid (include/dsx_shard.h).
    // The counts of every shard are summed first (classify, counter scan,
    // then one all-reduce), so the layout of the next owned half and of the
    // ghost region is planned on the host before anything moves: the move
    // writes retained particles and ghost images straight to their final
    // slots, the emigrants land in the source order of the reference with
    // gaps for the groups other shards send, and only emigrants, ghost lists
    // toward other shards' receivers and those lists' forces cross shards.
    //
    // Ghost region of a shard: its own receivers first (rank order), each
    // block in the receiver's neighbor order with the lists of every sender;
    // then the other shards' receivers (by shard, then rank) holding only
    // the lists of this shard's senders (sent away after the build, their
    // forces returned before the reverse sum).
    ShardPlan plan_shard(const std::vector<long long>& sum, const std::vector<int>& owners, int shard,
                         int nshards, int local_emigrants) const {
        return plan_shard_layout(P, topo, sum, owners, shard, nshards, local_emigrants);
    }

    // message buffers of the sharded step, one per peer and direction (grow only)
    struct PeerBuffer {
        void* data = nullptr;
        long long capacity = 0;
        void* ensure(long long bytes) {
            if (bytes > capacity) {
                cudaFree(data);
                data = nullptr;
                capacity = 0;
                cuda_check(cudaMalloc(&data, static_cast<std::size_t>(bytes)), "cudaMalloc message buffer");
                capacity = bytes;
            }
            return data;
        }
    };
    std::vector<PeerBuffer> shard_send, shard_recv;
    int* d_export = nullptr;        // [29P + 1]
    int* d_local_imm = nullptr;     // [P]
    int* d_imm_tiles_in = nullptr;  // [P]
    int* d_own_totals = nullptr;    // {own receivers' ghosts, boundary owners}
    bool sharded_ghosts = false;    // the ghost region holds a sharded step's layout
    // every subdomain's owned count after the last fused step, valid while
    // layout_version (moved by every call that changes the layout) stands
    std::vector<double> shard_counts;
    unsigned long long shard_counts_version = ~0ull;

    // pinned host staging of the sharded step's counts and planned tables
    unsigned char* shard_pinned = nullptr;
    std::size_t shard_pinned_cap = 0;

    unsigned char* shard_staging(std::size_t bytes) {
        if (bytes > shard_pinned_cap) {
            if (shard_pinned) cudaFreeHost(shard_pinned);
            shard_pinned = nullptr;
            shard_pinned_cap = 0;
            void* p = nullptr;
            cuda_check(cudaMallocHost(&p, bytes), "cudaMallocHost staging");
            shard_pinned = static_cast<unsigned char*>(p);
            shard_pinned_cap = bytes;
        }
        return shard_pinned;
    }

    void free_shard_buffers() {
        if (shard_pinned) cudaFreeHost(shard_pinned);
        shard_pinned = nullptr;
        for (auto& b : shard_send) cudaFree(b.data);
        for (auto& b : shard_recv) cudaFree(b.data);
        shard_send.clear();
        shard_recv.clear();
    }

    long long array_bytes(int a) const {
        return a < 11 ? 8 : a < 13 ? 4 : fields[static_cast<std::size_t>(a - 13)].bytes;
    }

    unsigned char* array_base(int a) const {
        return static_cast<unsigned char*>(
            a < 11 ? static_cast<void*>(A.d[a]) : a == 11 ? static_cast<void*>(A.type) :
            a == 12 ? static_cast<void*>(A.gid) : static_cast<void*>(A.f.base[a - 13]));
    }

    // One message per peer each way: pack `count[p]` records of `arrays`
    // starting at element `first[p]` of `region` (an element offset into
    // the arrays) into peer p's send buffer, one 16-byte aligned section per
    // array; the received messages are scattered by `place(p, buffer
    // sections)`.
    template <class Place>
    void shard_exchange(const dsx_transport& tr, int shard, int nshards, const std::vector<int>& arrays,
                        long long region, const std::vector<long long>& first,
                        const std::vector<long long>& count, const std::vector<long long>& incoming,
                        cudaStream_t stream, Place&& place) {
        auto packed = [&](long long n) {
            long long b = 0;
            for (int a : arrays) b += (n * array_bytes(a) + 15) / 16 * 16;
            return b;
        };
        auto sections = [&](void* buf, long long n) {
            std::vector<unsigned char*> out;
            long long at = 0;
            for (int a : arrays) {
                out.push_back(static_cast<unsigned char*>(buf) + at);
                at += (n * array_bytes(a) + 15) / 16 * 16;
            }
            return out;
        };
        if (static_cast<int>(shard_send.size()) < nshards) {
            shard_send.resize(static_cast<std::size_t>(nshards));
            shard_recv.resize(static_cast<std::size_t>(nshards));
        }
        std::vector<int> to, from;
        std::vector<const void*> sb;
        std::vector<void*> rb;
        std::vector<long long> sn, rn;
        std::vector<dsx::CopyPiece> pack;
        for (int p = 0; p < nshards; ++p) {
            if (p == shard) continue;
            if (count[p] > 0) {
                void* buf = shard_send[p].ensure(packed(count[p]));
                const std::vector<unsigned char*> sec = sections(buf, count[p]);
                for (std::size_t j = 0; j < arrays.size(); ++j) {
                    const long long b = array_bytes(arrays[j]);
                    pack.push_back({array_base(arrays[j]) + (region + first[p]) * b, sec[j], count[p] * b});
                }
                to.push_back(p);
                sb.push_back(buf);
                sn.push_back(packed(count[p]));
            }
            if (incoming[p] > 0) {
                from.push_back(p);
                rb.push_back(shard_recv[p].ensure(packed(incoming[p])));
                rn.push_back(packed(incoming[p]));
            }
        }
        if (!pack.empty()) cuda_check(dsx::launch_copies(pack, stream), "pack messages");
        // every shard makes the same transport calls, with messages or not
        // (a lone shard has no peer to call)
        if (nshards > 1 &&
            tr.exchange(tr.user, static_cast<int>(to.size()), to.data(), sb.data(), sn.data(),
                        static_cast<int>(from.size()), from.data(), rb.data(), rn.data(),
                        stream) != DSX_OK)
            fail(DSX_E_RUNTIME, "transport exchange failed");
        std::vector<dsx::CopyPiece> unpack;
        for (std::size_t k = 0; k < from.size(); ++k)
            place(from[k], sections(rb[k], incoming[from[k]]), unpack);
        if (!unpack.empty()) cuda_check(dsx::launch_copies(unpack, stream), "unpack messages");
    }

    void sharded_step(const int* owners_in, int shard, int nshards, const dsx_transport& tr,
                      dsx_step_callback cb, void* user, cudaStream_t stream, unsigned* status_out) {
        not_pending("the sharded step");
        if (!tr.allreduce_i64 || !tr.allreduce_f64 || !tr.exchange)
            fail(DSX_E_INVALID, "the transport needs both all-reduces and the exchange");
        if (nshards < 1 || shard < 0 || shard >= nshards) fail(DSX_E_INVALID, "shard out of range");
        const std::vector<int> owners(owners_in, owners_in + P);
        for (int t = 0; t < P; ++t)
            if (owners[t] < 0 || owners[t] >= nshards) fail(DSX_E_INVALID, "subdomain owner out of range");
        const int E = dsx::kMaxNeighbors;
        const std::size_t PP = static_cast<std::size_t>(P) * P;
        if (!S.pairs) {
            S.pairs = device_alloc<int>(fixed_owned, PP);
            S.gap = device_alloc<int>(fixed_owned, PP);
            d_export = device_alloc<int>(fixed_owned, static_cast<std::size_t>(29) * P + 1);
            d_local_imm = device_alloc<int>(fixed_owned, P);
            d_imm_tiles_in = device_alloc<int>(fixed_owned, P);
            d_own_totals = device_alloc<int>(fixed_owned, 2);
        }
        clear_status(stream);
        // Dynamic cut planes from the owned counts of every shard: known from
        // the previous fused step's sums while no other call has changed the
        // layout since, else summed now (an all-reduce over one shard is the
        // identity, so a lone shard makes no transport call)
        const double* work_in = nullptr;
        if (desc.policy == DSX_DYNAMIC) {
            std::vector<double> w;
            if (shard_counts_version == layout_version && static_cast<int>(shard_counts.size()) == P) {
                w = shard_counts;
            } else {
                const std::vector<int> n = read_ints(layout[cur][0], P, stream);
                w.assign(n.begin(), n.end());
                if (nshards > 1 && tr.allreduce_f64(tr.user, w.data(), P) != DSX_OK)
                    fail(DSX_E_RUNTIME, "transport all-reduce failed");
            }
            // the staging buffer is idle here (the previous step ended with a
            // synchronising status read) and sized for the counts read below
            // too, so it is not reallocated under this copy
            std::memcpy(shard_staging(std::max(sizeof(double) * P, sizeof(int) * (58 * P + 1 + PP))), w.data(),
                        sizeof(double) * P);
            cuda_check(cudaMemcpyAsync(work, shard_pinned, sizeof(double) * P, cudaMemcpyHostToDevice, stream),
                       "upload work");
            work_in = work;
        }
        enqueue_rebalance(stream, true, work_in);
        const dsx::Grid G = params();
        dsx::launch_step_classify(G, A, owned_off(), S, stream);
        dsx::launch_step_scan(G, S, stream);
        dsx::launch_step_export(G, S, d_export, stream);
        // this shard's counts, summed over every shard
        const std::size_t nx = static_cast<std::size_t>(29) * P;
        int* staged = reinterpret_cast<int*>(shard_staging(sizeof(int) * (2 * nx + 1 + PP)));
        const int* ex = staged;
        const int* imm = staged + nx + 1;
        const int* pr = imm + nx;
        cuda_check(cudaMemcpyAsync(staged, d_export, sizeof(int) * (nx + 1), cudaMemcpyDeviceToHost, stream), "read counts");
        cuda_check(cudaMemcpyAsync(staged + nx + 1, S.imm_total, sizeof(int) * nx, cudaMemcpyDeviceToHost, stream), "read counts");
        cuda_check(cudaMemcpyAsync(staged + 2 * nx + 1, S.pairs, sizeof(int) * PP, cudaMemcpyDeviceToHost, stream), "read counts");
        cuda_check(cudaStreamSynchronize(stream), "read counts");
        std::vector<long long> sum(2 * nx + PP + static_cast<std::size_t>(nshards), 0);
        for (std::size_t k = 0; k < nx; ++k) sum[k] = ex[k];
        for (std::size_t k = 0; k < nx; ++k) sum[nx + k] = imm[k];
        for (std::size_t k = 0; k < PP; ++k) sum[2 * nx + k] = pr[k];
        sum[2 * nx + PP + static_cast<std::size_t>(shard)] = ncap;
        if (nshards > 1 && tr.allreduce_i64(tr.user, sum.data(), static_cast<long long>(sum.size())) != DSX_OK)
            fail(DSX_E_RUNTIME, "transport all-reduce failed");
        const long long* pairs = sum.data() + 2 * nx;
        const long long* imm_total = sum.data() + nx;
        auto pair = [&](int t, int q) { return pairs[static_cast<std::size_t>(t) * P + q]; };
        // every shard checks every shard's storage with the same numbers, so
        // a shortfall anywhere fails everywhere before data moves
        for (int p = 0; p < nshards; ++p) {
            long long need = 0;
            for (int t = 0; t < P; ++t) {
                if (owners[t] == p) need += sum[static_cast<std::size_t>(t)] + imm_total[t];
                else
                    for (int q = 0; q < P; ++q)
                        if (owners[q] == p) need += pair(t, q);
            }
            if (need > sum[2 * nx + PP + static_cast<std::size_t>(p)])
                fail(DSX_E_LENGTH, "particle storage of shard " + std::to_string(p) +
                                       " is smaller than its particles after the step's migration");
        }
        const ShardPlan pl = plan_shard(sum, owners, shard, nshards, ex[nx]);
        if (pl.ghosts > gcap) grow_ghosts(pl.ghosts, stream);   // nothing is written yet
        // the planned layout to the device, through pinned staging (the
        // copies stay asynchronous; the staging is reused only after the
        // step's final synchronize)
        auto round8 = [](std::size_t b) { return (b + 7) / 8 * 8; };
        // twenty tables, each rounded up to 8 bytes
        const std::size_t staging_bytes =
            sizeof(int) * (7 * static_cast<std::size_t>(P) + 4 * (P + 1) + PP + 2 +
                           3 * static_cast<std::size_t>(P) * E + 2 * static_cast<std::size_t>(P) * dsx::kHaloCounters + 5) +
            sizeof(long long) * 6 * static_cast<std::size_t>(P) + 20 * 8;
        unsigned char* stage = shard_staging(staging_bytes);
        std::size_t at = 0;
        auto up = [&](void* dst, const void* src, std::size_t bytes) {
            if (!bytes) return;
            if (at + bytes > staging_bytes) fail(DSX_E_RUNTIME, "plan staging too small");
            std::memcpy(stage + at, src, bytes);
            cuda_check(cudaMemcpyAsync(dst, stage + at, bytes, cudaMemcpyHostToDevice, stream), "upload plan");
            at += round8(bytes);
        };
        const int emig_info[2] = {pl.emigrants, (pl.emigrants + dsx::kTile - 1) / dsx::kTile};
        const int halo_info[2] = {static_cast<int>(pl.ghosts), static_cast<int>(pl.boundary)};
        const int own_totals[2] = {static_cast<int>(pl.own_ghosts), static_cast<int>(pl.boundary)};
        const int images = static_cast<int>(pl.images);
        up(layout[cur ^ 1][0], pl.n_next.data(), sizeof(int) * P);
        up(layout[cur ^ 1][1], pl.obase_next.data(), sizeof(int) * (P + 1));
        up(layout[cur ^ 1][2], pl.tile_start_next.data(), sizeof(int) * (P + 1));
        up(S.imm_base, pl.imm_base.data(), sizeof(int) * P);
        up(S.imm_tile_start, pl.imm_tile_start.data(), sizeof(int) * (P + 1));
        up(d_imm_tiles_in, pl.imm_tiles_in.data(), sizeof(int) * P);
        up(d_local_imm, pl.local_imm.data(), sizeof(int) * P);
        up(S.gap, pl.gap.data(), sizeof(int) * PP);
        up(S.emig_info, emig_info, sizeof(emig_info));
        up(S.mig_results, pl.results.data(), sizeof(long long) * 6 * P);
        up(S.list_ret, pl.list_ret.data(), sizeof(int) * P * E);
        up(S.list_len, pl.list_len.data(), sizeof(int) * P * E);
        up(S.send_base, pl.send_base.data(), sizeof(int) * P * E);
        up(S.g, pl.g.data(), sizeof(int) * P);
        up(S.gbase, pl.gbase.data(), sizeof(int) * (P + 1));
        up(S.cbase, pl.cbase_ret.data(), sizeof(int) * P * dsx::kHaloCounters);
        up(S.cbase_imm, pl.cbase_imm.data(), sizeof(int) * P * dsx::kHaloCounters);
        up(S.halo_info, halo_info, sizeof(halo_info));
        up(d_own_totals, own_totals, sizeof(own_totals));
        up(S.boff + pl.boundary, &images, sizeof(int));
        // stays and ghost images of the retained particles, then the
        // emigrants in the reference's order with gaps for other shards'
        const dsx::Grid Gp = params();
        dsx::launch_step_bases(Gp, S, d_imm_tiles_in, stream);
        dsx::launch_step_move(Gp, A, owned_off(), next_off(), ghost_off(), S, stream);
        dsx::launch_step_emigrants(Gp, A, owned_off(), next_off(), S, d_local_imm, S.gap, stream);
        std::vector<int> all(static_cast<std::size_t>(13 + fields.size()));
        for (std::size_t a = 0; a < all.size(); ++a) all[a] = static_cast<int>(a);
        // emigrants to other shards' subdomains, and their emigrants into the gaps
        std::vector<long long> first(nshards, 0), count(nshards, 0);
        for (int p = 0; p < nshards; ++p) {
            first[p] = pl.out_start[p];
            count[p] = pl.out_end[p] - pl.out_start[p];
        }
        shard_exchange(tr, shard, nshards, all, next_off(), first, count, pl.recv_particles, stream,
                       [&](int p, const std::vector<unsigned char*>& sec, std::vector<dsx::CopyPiece>& out) {
            long long off = 0;
            for (int t = 0; t < P; ++t) {
                if (owners[t] != shard) continue;
                long long before = 0;
                for (int q = 0; q < P; ++q) {
                    const long long c = pair(t, q);
                    if (owners[q] == p && c > 0) {
                        for (std::size_t j = 0; j < all.size(); ++j) {
                            const long long b = array_bytes(all[j]);
                            out.push_back({sec[j] + off * b,
                                           array_base(all[j]) + (next_off() + pl.imm_base[t] + before) * b,
                                           c * b});
                        }
                        off += c;
                    }
                    before += c;
                }
            }
        });
        // the immigrants' ghost images (this shard's and the others')
        cur ^= 1;
        const dsx::Grid Gn = params();
        cur ^= 1;
        dsx::launch_step_immigrant_halo(Gn, A, next_off(), ghost_off(), S, stream);
        // ghost lists toward other shards' receivers, theirs into this shard's blocks
        for (int p = 0; p < nshards; ++p) {
            first[p] = pl.gout_start[p];
            count[p] = pl.gout_end[p] - pl.gout_start[p];
        }
        auto own_rows = [&](int p, auto&& row) {
            long long off = 0;
            for (int q = 0; q < P; ++q) {
                if (owners[q] != shard) continue;
                for (std::size_t m = 0; m < topo[q].size(); ++m) {
                    const int e = sender_entry(q, static_cast<int>(m));
                    if (e < 0 || owners[e / E] != p) continue;
                    const long long len = pl.list_len[static_cast<std::size_t>(e)];
                    if (len > 0) row(off, pl.send_base[static_cast<std::size_t>(e)], len);
                    off += len;
                }
            }
        };
        shard_exchange(tr, shard, nshards, all, ghost_off(), first, count, pl.recv_ghosts, stream,
                       [&](int p, const std::vector<unsigned char*>& sec, std::vector<dsx::CopyPiece>& out) {
            own_rows(p, [&](long long off, long long slot, long long len) {
                for (std::size_t j = 0; j < all.size(); ++j) {
                    const long long b = array_bytes(all[j]);
                    out.push_back({sec[j] + off * b, array_base(all[j]) + (ghost_off() + slot) * b, len * b});
                }
            });
        });
        // the new layout is the current one for the callback and the reverse sum
        parity ^= 1;
        cur ^= 1;
        ++layout_version;
        total = pl.own_total;
        pairs_valid = false;
        plan_valid = false;
        ghosts_valid = false;
        sharded_ghosts = true;
        plain_bounds.clear();
        std::fill(last_ghosts.begin(), last_ghosts.end(), 0);
        if (cb) {
            dsx_grid_view v = view();
            v.halo_totals = d_own_totals;
            cb(user, stream, &v);
        }
        // forces of this shard's blocks back to the senders' shards, and the
        // forces of this shard's lists from theirs
        const std::vector<int> forces = {6, 7, 8};
        {
            // gather this shard's receivers' ghosts of each peer's lists
            std::vector<long long> back(nshards, 0);
            for (int p = 0; p < nshards; ++p)
                if (p != shard) back[p] = pl.recv_ghosts[p];
            std::vector<long long> theirs(nshards, 0);
            for (int p = 0; p < nshards; ++p) theirs[p] = pl.gout_end[p] - pl.gout_start[p];
            if (static_cast<int>(shard_send.size()) < nshards) {
                shard_send.resize(static_cast<std::size_t>(nshards));
                shard_recv.resize(static_cast<std::size_t>(nshards));
            }
            std::vector<int> to, from;
            std::vector<const void*> sb;
            std::vector<void*> rb;
            std::vector<long long> sn, rn;
            std::vector<dsx::CopyPiece> pack, unpack;
            auto packed = [&](long long n) { return 3 * ((n * 8 + 15) / 16 * 16); };
            auto section = [&](void* buf, long long n, int j) {
                return static_cast<unsigned char*>(buf) + j * ((n * 8 + 15) / 16 * 16);
            };
            for (int p = 0; p < nshards; ++p) {
                if (p == shard) continue;
                if (back[p] > 0) {
                    void* buf = shard_send[p].ensure(packed(back[p]));
                    own_rows(p, [&](long long off, long long slot, long long len) {
                        for (int j = 0; j < 3; ++j)
                            pack.push_back({array_base(forces[j]) + (ghost_off() + slot) * 8,
                                            section(buf, back[p], j) + off * 8, len * 8});
                    });
                    to.push_back(p);
                    sb.push_back(buf);
                    sn.push_back(packed(back[p]));
                }
                if (theirs[p] > 0) {
                    void* buf = shard_recv[p].ensure(packed(theirs[p]));
                    for (int j = 0; j < 3; ++j)
                        unpack.push_back({section(buf, theirs[p], j),
                                          array_base(forces[j]) + (ghost_off() + pl.gout_start[p]) * 8,
                                          theirs[p] * 8});
                    from.push_back(p);
                    rb.push_back(buf);
                    rn.push_back(packed(theirs[p]));
                }
            }
            if (!pack.empty()) cuda_check(dsx::launch_copies(pack, stream), "pack forces");
            if (nshards > 1 &&
                tr.exchange(tr.user, static_cast<int>(to.size()), to.data(), sb.data(), sn.data(),
                            static_cast<int>(from.size()), from.data(), rb.data(), rn.data(),
                            stream) != DSX_OK)
                fail(DSX_E_RUNTIME, "transport exchange failed");
            if (!unpack.empty()) cuda_check(dsx::launch_copies(unpack, stream), "unpack forces");
        }
        enqueue_reverse(stream);
        const unsigned st = read_status(stream);
        if (st & dsx::kStatusCopyTimeout)
            fail(DSX_E_RUNTIME, "a bulk copy of particle records did not complete within 1 s");
        if (st & dsx::kStatusMigrationMismatch) fail(DSX_E_RUNTIME, "migration count mismatch");
        if (st & dsx::kStatusCutsInvalid)
            fail(DSX_E_INVALID, "dynamic cuts must be strictly increasing and span the domain");
        if (st & dsx::kStatusGhostOverflow) fail(DSX_E_RUNTIME, "ghost region overflow in a planned step");
        // every subdomain's new count (retained + immigrants, from the sums)
        // for the next fused step's rebalance
        shard_counts.assign(static_cast<std::size_t>(P), 0.0);
        for (int t = 0; t < P; ++t)
            shard_counts[static_cast<std::size_t>(t)] =
                static_cast<double>(sum[static_cast<std::size_t>(t)] + imm_total[t]);
        shard_counts_version = layout_version;
        if (status_out) *status_out = st;
    }

    void upload(const long long* counts, const void* const* arrays, cudaStream_t stream) {
        long long sum = 0;
        for (int s = 0; s < P; ++s) {
            if (counts[s] < 0) fail(DSX_E_INVALID, "negative particle count");
            sum += counts[s];
        }
        if (sum > ncap) fail(DSX_E_LENGTH, "particle storage is smaller than the supplied counts");
        total = sum;
        parity = 0;
        cur = 0;
        ++layout_version;
        pairs_valid = false;
        plan_valid = false;
        ghosts_valid = false;
        std::fill(last_ghosts.begin(), last_ghosts.end(), 0);
        const std::size_t n = static_cast<std::size_t>(sum);
        for (int a = 0; a < 13; ++a) {
            void* dst = a < 11 ? static_cast<void*>(A.d[a]) : a == 11 ? static_cast<void*>(A.type) : A.gid;
            const std::size_t bytes = n * (a < 11 ? sizeof(double) : sizeof(int));
            if (arrays && arrays[a])
                cuda_check(cudaMemcpyAsync(dst, arrays[a], bytes, cudaMemcpyDefault, stream), "upload");
            else
                cuda_check(cudaMemsetAsync(dst, 0, bytes, stream), "upload");
        }
        for (std::size_t f = 0; f < fields.size(); ++f) {
            const void* src = arrays ? arrays[13 + f] : nullptr;
            if (src)
                cuda_check(cudaMemcpyAsync(A.f.base[f], src, n * fields[f].bytes, cudaMemcpyDefault, stream), "upload");
            else
                cuda_check(cudaMemsetAsync(A.f.base[f], 0, n * fields[f].bytes, stream), "upload");
        }
        std::vector<int> c(static_cast<std::size_t>(P) + 1, 0);
        for (int s = 0; s < P; ++s) c[static_cast<std::size_t>(s)] = static_cast<int>(counts[s]);
        cuda_check(cudaMemcpyAsync(layout[cur][0], c.data(), sizeof(int) * (P + 1), cudaMemcpyHostToDevice, stream),
                   "upload counts");
        dsx::launch_layout(params(), layout[cur][0], layout[cur][1], layout[cur][2], layout_tiles[cur],
                           stream);
        cuda_check(cudaMemsetAsync(S.g, 0, sizeof(int) * (P + 1), stream), "memset");
        cuda_check(cudaMemsetAsync(S.gbase, 0, sizeof(int) * (P + 1), stream), "memset");
        cuda_check(cudaMemsetAsync(S.halo_info, 0, sizeof(int) * 4, stream), "memset");
        cuda_check(cudaStreamSynchronize(stream), "upload");
    }

    // slot range of one rank -> device index ranges in the owned/ghost regions
    void access(int rank, int array, long long start, long long count, void* host, bool write,
                cudaStream_t stream) {
        if (rank < 0 || rank >= P) fail(DSX_E_INVALID, "rank out of range");
        std::size_t element = 0;
        unsigned char* base = nullptr;
        if (array >= 0 && array < 11) { element = 8; base = reinterpret_cast<unsigned char*>(A.d[array]); }
        else if (array == 11) { element = 4; base = reinterpret_cast<unsigned char*>(A.type); }
        else if (array == 12) { element = 4; base = reinterpret_cast<unsigned char*>(A.gid); }
        else if (array >= 13 && array < 13 + static_cast<int>(fields.size())) {
            element = static_cast<std::size_t>(fields[static_cast<std::size_t>(array - 13)].bytes);
            base = A.f.base[array - 13];
        } else fail(DSX_E_INVALID, "bad array id");
        const std::vector<int> n = read_ints(layout[cur][0], P, stream);
        const std::vector<int> ob = read_ints(layout[cur][1], P, stream);
        std::vector<int> g(static_cast<std::size_t>(P), 0), gb(static_cast<std::size_t>(P), 0);
        if (ghosts_valid || sharded_ghosts) {
            g = read_ints(S.g, P, stream);
            gb = read_ints(S.gbase, P, stream);
        }
        const long long owned = n[static_cast<std::size_t>(rank)];
        const long long ghosts = g[static_cast<std::size_t>(rank)];
        if (start < 0 || count < 0 || start + count > owned + ghosts)
            fail(DSX_E_INVALID, "slot range outside the subdomain's particles");
        auto copy = [&](long long device_index, long long slots, unsigned char* h) {
            if (slots <= 0) return;
            unsigned char* d = base + static_cast<std::size_t>(device_index) * element;
            if (write)
                cuda_check(cudaMemcpyAsync(d, h, static_cast<std::size_t>(slots) * element, cudaMemcpyHostToDevice, stream), "write");
            else
                cuda_check(cudaMemcpyAsync(h, d, static_cast<std::size_t>(slots) * element, cudaMemcpyDeviceToHost, stream), "read");
        };
        unsigned char* h = static_cast<unsigned char*>(host);
        const long long owned_part = std::max<long long>(0, std::min(start + count, owned) - start);
        copy(owned_off() + ob[static_cast<std::size_t>(rank)] + start, owned_part, h);
        const long long ghost_start = std::max(start, owned) - owned;
        const long long ghost_part = count - owned_part;
        copy(ghost_off() + gb[static_cast<std::size_t>(rank)] + ghost_start, ghost_part,
             h + static_cast<std::size_t>(owned_part) * element);
        cuda_check(cudaStreamSynchronize(stream), "synchronize");
    }
};

extern "C" {

const char* dsx_last_error(void) { return g_error.c_str(); }
const char* dsx_version(void) { return "dsdecompx-b200 1.0.0 (sm_100a)"; }

int dsx_rank_migrate(double* x, double* y, double* z, long long owned, const dsx_domain* domain,
                     void* stream, dsx_migration_result* result) {
    return guarded([&] {
        if (!domain) fail(DSX_E_INVALID, "missing domain");
        if (!stream) fail(DSX_E_INVALID, "CUDA migration requires an explicit communication stream");
        if (owned < 0) fail(DSX_E_INVALID, "negative owned count");
        if (owned && (!x || !y || !z)) fail(DSX_E_INVALID, "incomplete CUDA migration view");
        double extent[3];
        for (int a = 0; a < 3; ++a) {
            if (!(domain->upper[a] > domain->lower[a])) fail(DSX_E_INVALID, "global-domain extent must be positive");
            extent[a] = domain->upper[a] - domain->lower[a];
        }
        dsx::launch_wrap_inplace(x, y, z, owned, domain->lower, extent, domain->periodic,
                                 static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch migrate");
        if (result) {
            result->ownership_changed = 0;
            result->previous_owned_count = owned;
            result->retained_count = owned;
            result->sent_count = 0;
            result->received_count = 0;
            result->new_owned_count = owned;
        }
    });
}

int dsx_plan_topology(const dsx_grid_desc* desc, int rank, int* dims, int* count, int* info,
                      double* shifts) {
    return guarded([&] {
        if (!desc) fail(DSX_E_INVALID, "null argument");
        const int P = desc->nranks;
        if (P < 1 || P > dsx::kMaxRanks) fail(DSX_E_INVALID, "nranks must be in 1..1024");
        if (rank < 0 || rank >= P) fail(DSX_E_INVALID, "rank out of range");
        int d[3];
        if (desc->policy != DSX_MANUAL) {
            const double len[3] = {desc->upper[0] - desc->lower[0], desc->upper[1] - desc->lower[1],
                                   desc->upper[2] - desc->lower[2]};
            for (double l : len) if (!(l > 0.0)) fail(DSX_E_INVALID, "domain lengths must be positive");
            choose_grid(P, len, desc->periodic, desc->policy, d);
        } else {
            for (int a = 0; a < 3; ++a) d[a] = desc->dims[a];
        }
        if (!fill_dims(P, d)) fail(DSX_E_INVALID, "process-grid dimensions do not match communicator size");
        const int c[3] = {rank / (d[1] * d[2]), (rank / d[2]) % d[1], rank % d[2]};
        const auto list = neighbors_of(c, d, *desc);
        for (int a = 0; a < 3; ++a) dims[a] = d[a];
        *count = static_cast<int>(list.size());
        for (std::size_t n = 0; n < list.size(); ++n) {
            info[5 * n + 0] = list[n].rank;
            for (int a = 0; a < 3; ++a) {
                info[5 * n + 1 + a] = list[n].dir[a];
                shifts[3 * n + a] = list[n].shift[a];
            }
            info[5 * n + 4] = list[n].slot;
        }
    });
}

int dsx_grid_create(const dsx_grid_desc* desc, const dsx_field_desc* fields, int nfields,
                    long long particles, long long ghost_capacity, dsx_grid** out) {
    return guarded([&] {
        if (!desc || !out) fail(DSX_E_INVALID, "null argument");
        if (nfields && !fields) fail(DSX_E_INVALID, "custom field array is null");
        auto* g = new dsx_grid();
        try {
            g->setup(*desc, fields, nfields, particles, ghost_capacity);
        } catch (...) {
            delete g;
            throw;
        }
        *out = g;
    });
}

int dsx_grid_destroy(dsx_grid* grid) {
    return guarded([&] { delete grid; });
}

int dsx_grid_topology(dsx_grid* grid, int rank, int* dims, int* coords, double* local) {
    return guarded([&] {
        if (!grid || rank < 0 || rank >= grid->P) fail(DSX_E_INVALID, "rank out of range");
        std::vector<double> cuts;
        int total = 0;
        for (int a = 0; a < 3; ++a) total += grid->dims[a] + 1;
        cuts.resize(static_cast<std::size_t>(total));
        cuda_check(cudaMemcpy(cuts.data(), grid->cuts, sizeof(double) * total, cudaMemcpyDeviceToHost), "read cuts");
        const auto& c = grid->coords[static_cast<std::size_t>(rank)];
        for (int a = 0; a < 3; ++a) {
            dims[a] = grid->dims[a];
            coords[a] = c[static_cast<std::size_t>(a)];
            local[a] = cuts[static_cast<std::size_t>(grid->cut_offset[a] + c[static_cast<std::size_t>(a)])];
            local[3 + a] = cuts[static_cast<std::size_t>(grid->cut_offset[a] + c[static_cast<std::size_t>(a)] + 1)];
        }
    });
}

int dsx_grid_neighbors(dsx_grid* grid, int rank, int* count, int* info, double* shifts) {
    return guarded([&] {
        if (!grid || rank < 0 || rank >= grid->P) fail(DSX_E_INVALID, "rank out of range");
        const auto& list = grid->topo[static_cast<std::size_t>(rank)];
        *count = static_cast<int>(list.size());
        for (std::size_t n = 0; n < list.size(); ++n) {
            info[5 * n + 0] = list[n].rank;
            info[5 * n + 1] = list[n].dir[0];
            info[5 * n + 2] = list[n].dir[1];
            info[5 * n + 3] = list[n].dir[2];
            info[5 * n + 4] = list[n].slot;
            for (int a = 0; a < 3; ++a) shifts[3 * n + a] = list[n].shift[a];
        }
    });
}

int dsx_grid_cuts(dsx_grid* grid, double* out, void* stream) {
    return guarded([&] {
        grid->settle_async();
        int total = 0;
        for (int a = 0; a < 3; ++a) total += grid->dims[a] + 1;
        cuda_check(cudaMemcpyAsync(out, grid->cuts, sizeof(double) * total, cudaMemcpyDeviceToHost,
                                   static_cast<cudaStream_t>(stream)), "read cuts");
        cuda_check(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "synchronize");
    });
}

int dsx_grid_upload(dsx_grid* grid, const long long* counts, const void* const* arrays, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !counts) fail(DSX_E_INVALID, "null argument");
        grid->upload(counts, arrays, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_download(dsx_grid* grid, long long* counts, void* const* arrays, void* stream) {
    return guarded([&] {
        grid->settle_async();
        const auto s = static_cast<cudaStream_t>(stream);
        const std::vector<int> n = grid->read_ints(grid->layout[grid->cur][0], grid->P, s);
        for (int r = 0; r < grid->P; ++r) if (counts) counts[r] = n[static_cast<std::size_t>(r)];
        const std::size_t total = static_cast<std::size_t>(grid->total);
        const long long off = grid->owned_off();
        for (int a = 0; a < 13 + static_cast<int>(grid->fields.size()); ++a) {
            if (!arrays || !arrays[a]) continue;
            const void* src;
            std::size_t element;
            if (a < 11) { src = grid->A.d[a] + off; element = 8; }
            else if (a == 11) { src = grid->A.type + off; element = 4; }
            else if (a == 12) { src = grid->A.gid + off; element = 4; }
            else {
                element = static_cast<std::size_t>(grid->fields[static_cast<std::size_t>(a - 13)].bytes);
                src = grid->A.f.base[a - 13] + off * static_cast<long long>(element);
            }
            cuda_check(cudaMemcpyAsync(arrays[a], src, total * element, cudaMemcpyDefault, s), "download");
        }
        cuda_check(cudaStreamSynchronize(s), "download");
    });
}

int dsx_grid_totals(dsx_grid* grid, long long* out4, void* stream) {
    return guarded([&] {
        grid->settle_async();
        const auto s = static_cast<cudaStream_t>(stream);
        const std::vector<int> e = grid->read_ints(grid->S.emig_info, 1, s);
        const std::vector<int> h = grid->read_ints(grid->S.halo_info, 2, s);
        out4[0] = grid->total;
        out4[1] = e[0];
        out4[2] = h[0];
        out4[3] = h[1];
    });
}

int dsx_grid_counts(dsx_grid* grid, long long* owned, long long* ghosts, void* stream) {
    return guarded([&] {
        grid->settle_async();
        const auto s = static_cast<cudaStream_t>(stream);
        const std::vector<int> n = grid->read_ints(grid->layout[grid->cur][0], grid->P, s);
        std::vector<int> g(static_cast<std::size_t>(grid->P), 0);
        if (grid->ghosts_valid || grid->sharded_ghosts) g = grid->read_ints(grid->S.g, grid->P, s);
        for (int r = 0; r < grid->P; ++r) {
            if (owned) owned[r] = n[static_cast<std::size_t>(r)];
            if (ghosts) ghosts[r] = g[static_cast<std::size_t>(r)];
        }
    });
}

int dsx_grid_read(dsx_grid* grid, int rank, int array, long long start, long long count, void* host_out,
                  void* stream) {
    return guarded([&] {
        grid->settle_async();
        grid->access(rank, array, start, count, host_out, false, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_write(dsx_grid* grid, int rank, int array, long long start, long long count, const void* host_in,
                   void* stream) {
    return guarded([&] {
        grid->settle_async();
        grid->access(rank, array, start, count, const_cast<void*>(host_in), true, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_view_get(dsx_grid* grid, dsx_grid_view* out) {
    return guarded([&] { *out = grid->view(); });
}

int dsx_grid_migrate(dsx_grid* grid, void* stream, long long* results) {
    return guarded([&] {
        grid->settle_async();
        grid->migrate(static_cast<cudaStream_t>(stream), results);
        cuda_check(cudaGetLastError(), "launch migrate");
    });
}

int dsx_grid_exchange_halo(dsx_grid* grid, int rebuild, int positions_only, void* stream, long long* results) {
    return guarded([&] {
        grid->settle_async();
        grid->exchange_halo(rebuild != 0, positions_only != 0, static_cast<cudaStream_t>(stream), results);
        cuda_check(cudaGetLastError(), "launch halo");
    });
}

int dsx_grid_reverse_halo(dsx_grid* grid, void* stream) {
    return guarded([&] {
        grid->settle_async();
        grid->reverse_halo(static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch reverse halo");
    });
}

int dsx_grid_reverse_exchange(dsx_grid* grid, int nfields, const int* field_ids, const int* ops, void* stream) {
    return guarded([&] {
        grid->settle_async();
        grid->reverse_exchange(nfields, field_ids, ops, static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch reverse exchange");
    });
}

int dsx_grid_forward_exchange(dsx_grid* grid, int nfields, const int* field_ids, void* stream) {
    return guarded([&] {
        grid->settle_async();
        grid->forward_exchange(nfields, field_ids, static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch forward exchange");
    });
}

int dsx_grid_rebalance(dsx_grid* grid, const double* work, int force, void* stream, long long* results,
                       double* imbalance) {
    return guarded([&] {
        grid->settle_async();
        grid->rebalance(work, force != 0, static_cast<cudaStream_t>(stream), results, imbalance);
    });
}

int dsx_grid_set_halo_width(dsx_grid* grid, double width) {
    return guarded([&] {
        grid->settle_async();
        if (width < 0.0) fail(DSX_E_INVALID, "halo width cannot be negative");
        grid->not_pending("set_halo_width");
        if (grid->halo_width != width) {
            grid->halo_width = width;
            grid->plan_valid = false;
            grid->destroy_graphs();   // captured kernels hold the old width
        }
    });
}

int dsx_grid_set_refresh_kind(dsx_grid* grid, int kind) {
    return guarded([&] {
        if (!grid) fail(DSX_E_INVALID, "null grid");
        grid->settle_async();
        grid->not_pending("set_refresh_kind");
        if (kind < 0 || kind > 3) fail(DSX_E_INVALID, "refresh kind must be 0, 1, 2 or 3");
        if (grid->S.refresh_kind != kind) {
            grid->S.refresh_kind = kind;
            grid->destroy_graphs();
        }
    });
}

int dsx_grid_set_split_share(dsx_grid* grid, int ctas_per_sm) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        if (ctas_per_sm < 0) fail(DSX_E_INVALID, "CTAs per SM cannot be negative");
        grid->not_pending("set_split_share");
        if (grid->split_ctas_per_sm != ctas_per_sm) {
            grid->split_ctas_per_sm = ctas_per_sm;
            grid->destroy_graphs();
        }
    });
}

int dsx_grid_invalidate_halo(dsx_grid* grid) {
    return guarded([&] {
        grid->settle_async();
        grid->plan_valid = false;
    });
}

int dsx_grid_halo_backward(dsx_grid* grid, const double* cx, const double* cy, const double* cz,
                           double* gx, double* gy, double* gz, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (grid->P == 1 || !grid->ghosts_valid) return;
        dsx::launch_reverse_sum3(grid->params(), gx, gy, gz, cx, cy, cz, grid->S,
                                 static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch halo backward");
    });
}

int dsx_grid_step(dsx_grid* grid, dsx_step_callback callback, void* user, int capture, void* stream,
                  unsigned* status) {
    return guarded([&] {
        grid->settle_async();
        if (grid->P == 1) fail(DSX_E_INVALID, "the batched step needs at least two subdomains");
        if (capture && (stream == nullptr || static_cast<cudaStream_t>(stream) == cudaStreamLegacy ||
                        static_cast<cudaStream_t>(stream) == cudaStreamPerThread))
            fail(DSX_E_INVALID, "capturing the step in a CUDA graph needs a created stream, not the default stream");
        grid->step(callback, user, capture != 0, static_cast<cudaStream_t>(stream), status);
        cuda_check(cudaGetLastError(), "launch step");
    });
}

int dsx_grid_step_async(dsx_grid* grid, dsx_step_callback callback, void* user, void* stream) {
    return guarded([&] {
        if (grid->P == 1) fail(DSX_E_INVALID, "the batched step needs at least two subdomains");
        if (stream == nullptr || static_cast<cudaStream_t>(stream) == cudaStreamLegacy ||
            static_cast<cudaStream_t>(stream) == cudaStreamPerThread)
            fail(DSX_E_INVALID, "asynchronous steps need a created stream, not the default stream");
        grid->step_async(callback, user, static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch step");
    });
}

int dsx_grid_step_wait(dsx_grid* grid, unsigned* status) {
    return guarded([&] {
        const unsigned st = grid->step_wait();
        if (status) *status = st;
    });
}

int dsx_grid_sharded_step(dsx_grid* grid, const int* owners, int shard, int nshards,
                          const dsx_transport* transport, dsx_step_callback callback, void* user,
                          void* stream, unsigned* status) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !owners || !transport) fail(DSX_E_INVALID, "null argument");
        if (grid->P == 1) fail(DSX_E_INVALID, "the sharded step needs at least two subdomains");
        grid->sharded_step(owners, shard, nshards, *transport, callback, user,
                           static_cast<cudaStream_t>(stream), status);
        cuda_check(cudaGetLastError(), "launch sharded step");
    });
}

int dsx_shard_plan_step(const dsx_grid_desc* desc, const int* owners, int shard, int nshards,
                        const long long* sums, long long nsums, long long* out) {
    return guarded([&] {
        if (!desc || !owners || !sums || !out) fail(DSX_E_INVALID, "null argument");
        const int P = desc->nranks;
        if (P < 2 || P > dsx::kMaxRanks) fail(DSX_E_INVALID, "nranks must be in 2..1024");
        if (nshards < 1 || shard < 0 || shard >= nshards) fail(DSX_E_INVALID, "shard out of range");
        const long long want = 58LL * P + static_cast<long long>(P) * P + nshards;
        if (nsums != want) fail(DSX_E_INVALID, "sums must hold 58 P + P * P + nshards values");
        std::vector<int> own(owners, owners + P);
        for (int t = 0; t < P; ++t)
            if (own[t] < 0 || own[t] >= nshards) fail(DSX_E_INVALID, "subdomain owner out of range");
        int d[3];
        if (desc->policy != DSX_MANUAL) {
            const double len[3] = {desc->upper[0] - desc->lower[0], desc->upper[1] - desc->lower[1],
                                   desc->upper[2] - desc->lower[2]};
            choose_grid(P, len, desc->periodic, desc->policy, d);
        } else {
            for (int a = 0; a < 3; ++a) d[a] = desc->dims[a];
        }
        if (!fill_dims(P, d)) fail(DSX_E_INVALID, "process-grid dimensions do not match nranks");
        std::vector<std::vector<Neighbor>> topo(static_cast<std::size_t>(P));
        for (int r = 0; r < P; ++r) {
            const int c[3] = {r / (d[1] * d[2]), (r / d[2]) % d[1], r % d[2]};
            topo[static_cast<std::size_t>(r)] = neighbors_of(c, d, *desc);
        }
        const std::vector<long long> sum(sums, sums + nsums);
        const ShardPlan pl = plan_shard_layout(P, topo, sum, own, shard, nshards, 0);
        out[0] = pl.own_total;
        out[1] = pl.out_total;
        out[2] = pl.ghosts;
        out[3] = pl.own_ghosts;
        out[4] = pl.boundary;
        out[5] = pl.images;
        for (int p = 0; p < nshards; ++p) {
            long long* o = out + 6 + 4 * p;
            o[0] = pl.out_end[p] - pl.out_start[p];
            o[1] = pl.recv_particles[p];
            o[2] = pl.gout_end[p] - pl.gout_start[p];
            o[3] = pl.recv_ghosts[p];
        }
    });
}

int dsx_grid_autotune(dsx_grid* grid, void* stream, dsx_tune_report* report) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        grid->autotune(static_cast<cudaStream_t>(stream), report);
    });
}

int dsx_grid_begin_halo_exchange(dsx_grid* grid, int rebuild, int positions_only, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        grid->begin_halo(rebuild != 0, positions_only != 0, static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch halo exchange");
    });
}

int dsx_grid_end_halo_exchange(dsx_grid* grid, void* stream, long long* results) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        grid->end_halo(static_cast<cudaStream_t>(stream), results);
    });
}

int dsx_grid_owner_rank(dsx_grid* grid, const double* x, const double* y, const double* z,
                        long long n, int* out, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || n < 0 || (n > 0 && (!x || !y || !z || !out))) fail(DSX_E_INVALID, "null argument");
        dsx::launch_owner_rank(grid->params(), x, y, z, n, out, static_cast<cudaStream_t>(stream));
        cuda_check(cudaGetLastError(), "launch owner_rank");
    });
}

int dsx_grid_out_of_domain(dsx_grid* grid, int* flags, int* any, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        const long long o = grid->owned_off();
        dsx::launch_out_of_domain(grid->params(), grid->A.d[0] + o, grid->A.d[1] + o,
                                  grid->A.d[2] + o, grid->S.out_flags, s);
        std::vector<int> f = grid->read_ints(grid->S.out_flags, grid->P, s);
        int hit = 0;
        for (int v : f) hit |= v;
        if (flags) std::copy(f.begin(), f.end(), flags);
        if (any) *any = hit;
    });
}

int dsx_grid_set_cuts(dsx_grid* grid, const double* cuts, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !cuts) fail(DSX_E_INVALID, "null argument");
        grid->set_cuts(cuts, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_rescale_domain(dsx_grid* grid, const double* lower, const double* upper,
                            int invalidate_plan, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !lower || !upper) fail(DSX_E_INVALID, "null argument");
        grid->rescale_domain(lower, upper, invalidate_plan != 0, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_migration_pairs(dsx_grid* grid, long long* pairs, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !pairs) fail(DSX_E_INVALID, "null argument");
        grid->migration_pairs(pairs, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_send_lists(dsx_grid* grid, int* length, int* first_slot, void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !length || !first_slot) fail(DSX_E_INVALID, "null argument");
        grid->send_lists(length, first_slot, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_assemble(dsx_grid* grid, const long long* counts, int nsources,
                      const void* const* sources, long long nsegments, const dsx_segment* segments,
                      void* stream) {
    return guarded([&] {
        grid->settle_async();
        if (!grid || !counts || (nsegments > 0 && !segments) || (nsources > 0 && !sources) ||
            nsources < 0 || nsegments < 0)
            fail(DSX_E_INVALID, "null argument");
        grid->assemble(counts, nsources, sources, nsegments, segments, static_cast<cudaStream_t>(stream));
    });
}

int dsx_grid_set_rebalance_work(dsx_grid* grid, const double* work) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        grid->set_rebalance_work(work);
    });
}

int dsx_copy_segments(const dsx_copy* copies, long long n, void* stream) {
    return guarded([&] {
        if (n < 0 || (n > 0 && !copies)) fail(DSX_E_INVALID, "null argument");
        std::vector<dsx::CopyPiece> list;
        list.reserve(static_cast<std::size_t>(n));
        for (long long k = 0; k < n; ++k) {
            if (copies[k].bytes < 0) fail(DSX_E_INVALID, "negative copy size");
            if (copies[k].bytes && (!copies[k].src || !copies[k].dst)) fail(DSX_E_INVALID, "null copy address");
            list.push_back({static_cast<const unsigned char*>(copies[k].src),
                            static_cast<unsigned char*>(copies[k].dst), copies[k].bytes});
        }
        cuda_check(dsx::launch_copies(list, static_cast<cudaStream_t>(stream)), "copy segments");
    });
}

int dsx_grid_set_tuning(dsx_grid* grid, int classify_threads, int move_kind,
                        int reverse_ctas_per_sm, int classify_combine) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        if (classify_threads != 64 && classify_threads != 128 && classify_threads != 256)
            fail(DSX_E_INVALID, "classify threads must be 64, 128 or 256");
        if (move_kind < 0 || move_kind > 3) fail(DSX_E_INVALID, "move kind must be 0..3");
        if (reverse_ctas_per_sm < 0 || reverse_ctas_per_sm > 32)
            fail(DSX_E_INVALID, "reverse CTAs per SM must be 0..32");
        grid->not_pending("set_tuning");
        grid->S.classify_threads = classify_threads;
        grid->S.classify_combine = classify_combine != 0;
        grid->S.move_staged = move_kind;
        grid->S.reverse_per_sm = reverse_ctas_per_sm;
        grid->destroy_graphs();   // captured steps hold the old launch shapes
    });
}

int dsx_grid_set_plain(dsx_grid* grid, int plain) {
    return guarded([&] {
        grid->settle_async();
        if (!grid) fail(DSX_E_INVALID, "null grid");
        grid->plain = plain != 0;
        grid->plain_bounds.clear();
    });
}

int dsx_grid_profile(dsx_grid* grid, int enable) {
    return guarded([&] {
        grid->settle_async();
        if (enable && !grid->marks.ev[0])
            for (auto& e : grid->marks.ev) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        if ((enable != 0) != grid->marks.on) grid->destroy_graphs();
        grid->marks.on = enable != 0;
        grid->marks.count = 0;
    });
}

int dsx_grid_kernel_times(dsx_grid* grid, int max, const char** names, float* ms) {
    int n = 0;
    const int status = guarded([&] {
        grid->settle_async();
        const dsx::Marks& m = grid->marks;
        if (!m.on || m.count < 2) return;
        cuda_check(cudaEventSynchronize(m.ev[m.count - 1]), "event synchronize");
        for (int k = 1; k < m.count && n < max; ++k, ++n) {
            float t = 0.0f;
            cuda_check(cudaEventElapsedTime(&t, m.ev[k - 1], m.ev[k]), "event elapsed");
            if (names) names[n] = m.name[k];
            if (ms) ms[n] = t;
        }
    });
    return status == DSX_OK ? n : status;
}

int dsx_grid_step_kernel_count(dsx_grid* grid) {
    // rebalance (Dynamic only); classify, counter scan, layout, tile bases,
    // move; emigrant histogram, column scan, placement; immigrants' classify,
    // scan, scatter; reverse sum
    return (grid->desc.policy == DSX_DYNAMIC ? 1 : 0) + 5 + 3 + 3 + 1;
}

}  // extern "C"
