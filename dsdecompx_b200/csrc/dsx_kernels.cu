// Hand-written sm_100a kernels of the particle-bookkeeping hot path.
//
// All of this work is HBM-bound integer/FP64 bookkeeping (no contraction, so
// no tensor cores): every kernel streams SoA arrays with coalesced accesses,
// compacts with warp ballots + popc, and orders its output with per-tile
// counters and prefix sums so that the result is deterministic and identical
// to the reference's Host path order (dsDecompX src/migration.cpp:437-518,
// src/halo.cpp:164-238, 1476-1531).
//
// Built with -fmad=false: the few FP64 expressions (periodic wrap, shift add,
// force sums) must round exactly like the reference's.
#include "dsx_kernels.cuh"

#include <cstdio>
#include <mutex>
#include <utility>

namespace dsx {
namespace {

constexpr int NT = 256;           // threads per CTA of the tile kernels
constexpr int ITEMS = 2;          // consecutive 32-particle groups per warp
constexpr int TILE = NT * ITEMS;  // particles per tile
constexpr int NW = NT / 32;

static_assert(TILE == kTile, "engine tile size");

// Exclusive block scan; `total` gets the block sum.  ws: 33 ints of shared.
template <int THREADS>
__device__ __forceinline__ int block_scan_excl(int v, int& total, int* ws) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < THREADS / 32 ? ws[lane] : 0;
        int winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= o) winc += u;
        }
        ws[lane] = winc - w;
        if (lane == 31) ws[32] = winc;
    }
    __syncthreads();
    const int excl = inc - v + ws[warp];
    total = ws[32];
    __syncthreads();
    return excl;
}

__device__ __forceinline__ int warp_inclusive_sum(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

// One subdomain's cell: its grid coordinates and cut planes.
struct Cell {
    int c[3];
    double lo[3], hi[3];
};

__device__ __forceinline__ bool inside_cell(const Cell& cell, double px, double py, double pz) {
    return cell.lo[0] <= px && px < cell.hi[0] && cell.lo[1] <= py && py < cell.hi[1] &&
           cell.lo[2] <= pz && pz < cell.hi[2];
}

// With every periodic axis starting at 0, a coordinate inside its own cell
// needs no wrap arithmetic: both Host wraps return it (a -0 as +0).
__device__ __forceinline__ bool simple_wrap(const Grid& G) {
    return (!G.periodic[0] || G.lower[0] == 0.0) && (!G.periodic[1] || G.lower[1] == 0.0) &&
           (!G.periodic[2] || G.lower[2] == 0.0);
}

__device__ __forceinline__ Cell cell_of(const Grid& G, int s) {
    Cell cell;
    const int packed = G.coord[s];
    cell.c[0] = packed >> 20;
    cell.c[1] = (packed >> 10) & 1023;
    cell.c[2] = packed & 1023;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double* cuts = G.cuts + G.cut_offset[a];
        cell.lo[a] = cuts[cell.c[a]];
        cell.hi[a] = cuts[cell.c[a] + 1];
    }
    return cell;
}

// Host-path destination of one owned particle: wrapped_record wraps the
// position once, owner_rank wraps it again and bisects the cuts
// (dsDecompX src/migration.cpp:437-441, 74-98).  Returns the rank and the
// once-wrapped position that the migrated record carries.  `cell` is where
// the particle most likely still is: inside its cut planes upper_bound's
// answer is the cell's own coordinate (the cuts are strictly increasing), so
// the bisection runs only for particles that left it.
__device__ __forceinline__ int destination_near(const Grid& G, const Cell& cell, double px,
                                                double py, double pz, double& wx, double& wy,
                                                double& wz) {
    const double p[3] = {px, py, pz};
    double w[3];
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double v = p[a];
        if (G.periodic[a]) {
            w[a] = wrap_axis(p[a], G.lower[a], G.extent[a]);
            v = wrap_axis(w[a], G.lower[a], G.extent[a]);
        } else {
            w[a] = p[a];
        }
        c[a] = (cell.lo[a] <= v && v < cell.hi[a])
                   ? cell.c[a]
                   : axis_coordinate(G.cuts + G.cut_offset[a], G.dims[a], v);
    }
    wx = w[0];
    wy = w[1];
    wz = w[2];
    return (c[0] * G.dims[1] + c[1]) * G.dims[2] + c[2];
}

__device__ __forceinline__ void move_record(const Arrays& A, long long src, long long dst,
                                            double wx, double wy, double wz) {
    double v[8];
#pragma unroll
    for (int a = 3; a < 11; ++a) v[a - 3] = ro(A.d[a] + src);
    const int ty = ro(A.type + src), id = ro(A.gid + src);
    A.d[0][dst] = wx;
    A.d[1][dst] = wy;
    A.d[2][dst] = wz;
#pragma unroll
    for (int a = 3; a < 11; ++a) A.d[a][dst] = v[a - 3];
    A.type[dst] = ty;
    A.gid[dst] = id;
    copy_fields(A.f, src, dst);
}

// End of the tile window of a launch: the window's own end in plain mode
// (one launch per subdomain), else the tile count on the device.
__device__ __forceinline__ int tile_limit(const Grid& G, const int* ntiles) {
    return G.tile_end >= 0 ? G.tile_end : *ntiles;
}

// ------------------------------------------------------------------ layout

// Writes the per-tile descriptors {s, begin, end, first tile of s} of a
// layout whose counts, bases and tile starts sit in shared memory.
__device__ __forceinline__ void fill_tiles(int P, int tile, const int* s_n, const int* s_ob,
                                           const int* s_ts, int4* tiles) {
    const int total = s_ts[P];
    for (int g = threadIdx.x; g < total; g += blockDim.x) {
        int lo = 0, hi = P;   // largest s with s_ts[s] <= g
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_ts[mid] <= g) lo = mid;
            else hi = mid;
        }
        const int begin = s_ob[lo] + (g - s_ts[lo]) * tile;
        const int end = min(begin + tile, s_ob[lo] + s_n[lo]);
        tiles[g] = make_int4(lo, begin, end, s_ts[lo]);
    }
}

__global__ void __launch_bounds__(1024) k_layout(int P, int tile, const int* n, int* obase,
                                                  int* tile_start, int4* tiles) {
    pdl_begin();
    __shared__ int ws[33];
    __shared__ int s_n[kMaxRanks + 1], s_ob[kMaxRanks + 1], s_ts[kMaxRanks + 1];
    const int t = threadIdx.x;
    const int a = t < P ? n[t] : 0;
    const int b = t < P ? (a + tile - 1) / tile : 0;
    int ta, tb;
    const int ea = block_scan_excl<1024>(a, ta, ws);
    const int eb = block_scan_excl<1024>(b, tb, ws);
    if (t < P) {
        obase[t] = ea;
        tile_start[t] = eb;
        s_n[t] = a;
        s_ob[t] = ea;
        s_ts[t] = eb;
    }
    if (t == 0) {
        obase[P] = ta;
        tile_start[P] = tb;
        s_ob[P] = ta;
        s_ts[P] = tb;
    }
    __syncthreads();
    fill_tiles(P, tile, s_n, s_ob, s_ts, tiles);
}

// Exclusive prefix of counter k (= blockIdx.x) over the tiles of the layout.
// cnt/pre are counter-major: [k * stride + tile]; pre[k*stride + ntiles] = total.
__device__ __forceinline__ void scan_counter(const int* cnt, int* pre, int stride,
                                             const int* tile_start_end);

__global__ void __launch_bounds__(1024) k_scan_counters(const int* cnt, int* pre, int stride,
                                                         const int* tile_start_end) {
    pdl_begin();
    scan_counter(cnt, pre, stride, tile_start_end);
}

__device__ __forceinline__ void scan_counter(const int* cnt, int* pre, int stride,
                                             const int* tile_start_end) {
    constexpr int PER = 8;
    constexpr int CHUNK = 1024 * PER;
    __shared__ int ws[33];
    // a chunk of the counter, padded one word per 32 so that thread t's PER
    // consecutive entries sit in distinct banks
    __shared__ int buf[CHUNK + CHUNK / 32];
    const int k = blockIdx.x;
    const int ntiles = *tile_start_end;
    const int* src = cnt + static_cast<long long>(k) * stride;
    int* dst = pre + static_cast<long long>(k) * stride;
    auto at = [](int i) { return i + (i >> 5); };
    int carry = 0;
    for (int base = 0; base < ntiles; base += CHUNK) {
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = j * 1024 + threadIdx.x;
            buf[at(i)] = base + i < ntiles ? src[base + i] : 0;
        }
        __syncthreads();
        int v[PER];
        int sum = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            v[j] = buf[at(threadIdx.x * PER + j)];
            sum += v[j];
        }
        int total;
        int run = block_scan_excl<1024>(sum, total, ws) + carry;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            buf[at(threadIdx.x * PER + j)] = run;
            run += v[j];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = j * 1024 + threadIdx.x;
            if (base + i < ntiles) dst[base + i] = buf[at(i)];
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) dst[ntiles] = carry;
}

// ----------------------------------------------------------------- migrate

// K1: destination of every owned particle; per-tile stay/emigrant counts and
// per-destination immigrant totals.
__global__ void __launch_bounds__(NT, 4) k_mig_classify(Grid G, const double* __restrict__ x,
                                                     const double* __restrict__ y,
                                                     const double* __restrict__ z, int* cnt,
                                                     int stride, int* imm_total) {
    pdl_begin();
    __shared__ int ws[33];
    const int g = G.tile_first + blockIdx.x;
    const int P = G.P;
    if (g >= tile_limit(G, G.tile_start + P)) return;
    const int4 td = G.tiles[g];
    const int s = td.x, begin = td.y, end = td.z;
    int stay = 0, emig = 0;
    const Cell cell = cell_of(G, s);
    double px[ITEMS], py[ITEMS], pz[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = begin + threadIdx.x + j * NT;
        if (i < end) {
            px[j] = ro(x + i);
            py[j] = ro(y + i);
            pz[j] = ro(z + i);
        }
    }
    const bool simple = simple_wrap(G);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = begin + threadIdx.x + j * NT;
        const bool valid = i < end;
        // a group that stays inside its cell needs no wrap arithmetic
        if (__all_sync(0xffffffffu, !valid || (simple && inside_cell(cell, px[j], py[j], pz[j])))) {
            stay += valid ? 1 : 0;
            continue;
        }
        int key = -1;   // destination of an emigrant
        if (valid) {
            double wx, wy, wz;
            const int d = destination_near(G, cell, px[j], py[j], pz[j], wx, wy, wz);
            if (d == s) {
                ++stay;
            } else {
                ++emig;
                key = d;
            }
        }
        // one atomic per destination and warp: after the cut planes moved,
        // most of a group can leave for the same few subdomains
        if (__any_sync(0xffffffffu, key >= 0)) {
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            if (key >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1)
                atomicAdd(&imm_total[key], __popc(peers));
        }
    }
    int stays, emigs;
    block_scan_excl<NT>(stay, stays, ws);
    block_scan_excl<NT>(emig, emigs, ws);
    if (threadIdx.x == 0) {
        cnt[g] = stays;
        cnt[stride + g] = emigs;
    }
}

// S1: the next layout (retained + immigrants per subdomain) and the migration
// result of every subdomain.  One CTA, one thread per subdomain.
__global__ void __launch_bounds__(1024) k_mig_layout(Grid G, const int* pre, int stride,
                                                      const int* imm_total, int* imm_base,
                                                      int* emig_info, long long* results) {
    pdl_begin();
    __shared__ int ws[33];
    const int P = G.P;
    const int t = threadIdx.x;
    const int ntiles = G.tile_start[P];
    int retained = 0, received = 0, old = 0, next = 0;
    if (t < P) {
        retained = pre[G.tile_start[t + 1]] - pre[G.tile_start[t]];
        received = imm_total[t];
        old = G.n[t];
        next = retained + received;
    }
    __shared__ int s_n[kMaxRanks + 1], s_ob[kMaxRanks + 1], s_ts[kMaxRanks + 1];
    int total_next, total_tiles;
    const int ob = block_scan_excl<1024>(next, total_next, ws);
    const int tiles = t < P ? (next + G.tile - 1) / G.tile : 0;
    const int ts = block_scan_excl<1024>(tiles, total_tiles, ws);
    if (t < P) {
        s_n[t] = next;
        s_ob[t] = ob;
        s_ts[t] = ts;
        G.n_next[t] = next;
        G.obase_next[t] = ob;
        G.tile_start_next[t] = ts;
        imm_base[t] = ob + retained;
        long long* o = results + 6 * t;
        o[1] = old;
        o[2] = retained;
        o[3] = old - retained;
        o[4] = received;
        o[5] = next;
        o[0] = (o[3] != 0 || o[4] != 0) ? 1 : 0;
    }
    if (t == 0) {
        s_ob[P] = total_next;
        s_ts[P] = total_tiles;
        G.obase_next[P] = total_next;
        G.tile_start_next[P] = total_tiles;
        const int E = pre[stride + ntiles];
        emig_info[0] = E;
        emig_info[1] = (E + TILE - 1) / TILE;
        if (total_next != G.obase[P]) atomicOr(G.status, kStatusMigrationMismatch);
    }
    __syncthreads();
    fill_tiles(P, G.tile, s_n, s_ob, s_ts, G.tiles_next);
}

// K2: retained particles move (stably) to the next layout; emigrants are
// listed in (source subdomain, source order), which is the order the
// reference's receivers append them in.
__global__ void __launch_bounds__(NT, 4) k_mig_move(Grid G, Arrays A, long long src_off,
                                                 long long dst_off, const int* pre, int stride,
                                                 int* emig_src, int* emig_dst) {
    pdl_begin();
    __shared__ int s_stay[NW], s_emig[NW];
    const int g = G.tile_first + blockIdx.x;
    const int P = G.P;
    if (g >= tile_limit(G, G.tile_start + P)) return;
    const int4 td = G.tiles[g];
    const int s = td.x, begin = td.y, end = td.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * ITEMS;
    const unsigned lt = lanemask_lt();

    int dest[ITEMS];
    double wx[ITEMS], wy[ITEMS], wz[ITEMS];
    int nstay = 0, nemig = 0;
    const Cell cell = cell_of(G, s);
    const bool simple = simple_wrap(G);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        const bool valid = i < end;
        dest[j] = -1;
        double px = 0.0, py = 0.0, pz = 0.0;
        if (valid) {
            const long long src = src_off + i;
            px = ro(A.d[0] + src);
            py = ro(A.d[1] + src);
            pz = ro(A.d[2] + src);
        }
        if (__all_sync(0xffffffffu, !valid || (simple && inside_cell(cell, px, py, pz)))) {
            // the whole group stays: both Host wraps return the coordinate (a -0 as +0)
            if (valid) {
                dest[j] = s;
                wx[j] = G.periodic[0] && px == 0.0 ? 0.0 : px;
                wy[j] = G.periodic[1] && py == 0.0 ? 0.0 : py;
                wz[j] = G.periodic[2] && pz == 0.0 ? 0.0 : pz;
            }
        } else if (valid) {
            dest[j] = destination_near(G, cell, px, py, pz, wx[j], wy[j], wz[j]);
        }
        nstay += __popc(__ballot_sync(0xffffffffu, dest[j] == s));
        nemig += __popc(__ballot_sync(0xffffffffu, dest[j] >= 0 && dest[j] != s));
    }
    if (lane == 0) {
        s_stay[warp] = nstay;
        s_emig[warp] = nemig;
    }
    __syncthreads();
    int stay_base = G.obase_next[s] + (pre[g] - pre[td.w]);
    int emig_base = pre[stride + g];
    for (int w = 0; w < warp; ++w) {
        stay_base += s_stay[w];
        emig_base += s_emig[w];
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        const unsigned bs = __ballot_sync(0xffffffffu, dest[j] == s);
        const unsigned be = __ballot_sync(0xffffffffu, dest[j] >= 0 && dest[j] != s);
        if (dest[j] == s) {
            move_record(A, src_off + i, dst_off + stay_base + __popc(bs & lt), wx[j], wy[j], wz[j]);
        } else if (dest[j] >= 0) {
            const int e = emig_base + __popc(be & lt);
            emig_src[e] = i;
            emig_dst[e] = dest[j];
        }
        stay_base += __popc(bs);
        emig_base += __popc(be);
    }
}

// K3a: per chunk of the emigrant list, how many go to each destination.
__global__ void __launch_bounds__(NT) k_emig_hist(int P, const int* emig_info,
                                                  const int* __restrict__ emig_dst, int* hist) {
    pdl_begin();
    extern __shared__ int sm[];  // [NW][P]
    const int E = emig_info[0], nchunks = emig_info[1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        for (int k = threadIdx.x; k < NW * P; k += NT) sm[k] = 0;
        __syncthreads();
        const int base = c * TILE + warp * 32 * ITEMS;
        for (int j = 0; j < ITEMS; ++j) {
            const int e = base + j * 32 + lane;
            const int d = e < E ? emig_dst[e] : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (d >= 0 && lane == __ffs(peers) - 1) sm[warp * P + d] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        for (int d = threadIdx.x; d < P; d += NT) {
            int sum = 0;
            for (int w = 0; w < NW; ++w) sum += sm[w * P + d];
            hist[static_cast<long long>(c) * P + d] = sum;
        }
        __syncthreads();
    }
}

// K3b: per destination, exclusive prefix of its chunk counts.
__global__ void __launch_bounds__(NT) k_emig_colscan(int P, const int* emig_info, int* hist,
                                                     const int* imm_total, unsigned* status) {
    pdl_begin();
    __shared__ int ws[33];
    const int d = blockIdx.x;
    const int nchunks = emig_info[1];
    int carry = 0;
    for (int base = 0; base < nchunks; base += NT) {
        const int c = base + threadIdx.x;
        const long long at = static_cast<long long>(c) * P + d;
        const int v = c < nchunks ? hist[at] : 0;
        int total;
        const int excl = block_scan_excl<NT>(v, total, ws);
        if (c < nchunks) hist[at] = carry + excl;
        carry += total;
    }
    if (threadIdx.x == 0 && carry != imm_total[d]) atomicOr(status, kStatusMigrationMismatch);
}

// K3c: every emigrant lands after its destination's retained particles, in
// (source subdomain, source order) -- a stable multi-split of the list.
__global__ void __launch_bounds__(NT) k_emig_place(Grid G, Arrays A, long long src_off,
                                                   long long dst_off, const int* emig_info,
                                                   const int* __restrict__ emig_src,
                                                   const int* __restrict__ emig_dst,
                                                   const int* hist, const int* imm_base,
                                                   const int* __restrict__ gap) {
    pdl_begin();
    extern __shared__ int sm[];  // [NW][P]
    const int P = G.P;
    const int E = emig_info[0], nchunks = emig_info[1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        for (int k = threadIdx.x; k < NW * P; k += NT) sm[k] = 0;
        __syncthreads();
        const int base = c * TILE + warp * 32 * ITEMS;
        int dj[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const int e = base + j * 32 + lane;
            dj[j] = e < E ? emig_dst[e] : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, dj[j]);
            if (dj[j] >= 0 && lane == __ffs(peers) - 1) sm[warp * P + dj[j]] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // per destination: exclusive prefix over warps, in place
        for (int d = threadIdx.x; d < P; d += NT) {
            int run = 0;
            for (int w = 0; w < NW; ++w) {
                const int v = sm[w * P + d];
                sm[w * P + d] = run;
                run += v;
            }
        }
        __syncthreads();
        // every emigrant's slot first (the counters step group by group),
        // then both records gathered before either is written
        int pos[ITEMS];
        long long src[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const int e = base + j * 32 + lane;
            const int d = dj[j];
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            pos[j] = 0;
            src[j] = 0;
            if (d >= 0) {
                pos[j] = imm_base[d] + hist[static_cast<long long>(c) * P + d] + sm[warp * P + d] +
                         __popc(peers & lt);
                const int i = emig_src[e];
                if (gap) {
                    // a sharded step: other shards' groups of immigrants of
                    // d that come before this emigrant's source q
                    int lo = 0, hi = P;   // largest q with obase[q] <= i
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (G.obase[mid] <= i) lo = mid;
                        else hi = mid;
                    }
                    pos[j] += gap[d * P + lo];
                }
                src[j] = src_off + i;
            }
            __syncwarp();
            if (d >= 0 && lane == __ffs(peers) - 1) sm[warp * P + d] += __popc(peers);
            __syncwarp();
        }
        double v[ITEMS][11];
        int ty[ITEMS], id[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (dj[j] < 0) continue;
#pragma unroll
            for (int a = 0; a < 11; ++a) v[j][a] = ro(A.d[a] + src[j]);
            ty[j] = ro(A.type + src[j]);
            id[j] = ro(A.gid + src[j]);
        }
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (dj[j] < 0) continue;
            const long long dst = dst_off + pos[j];
#pragma unroll
            for (int a = 0; a < 3; ++a)
                A.d[a][dst] = G.periodic[a] ? wrap_axis(v[j][a], G.lower[a], G.extent[a]) : v[j][a];
#pragma unroll
            for (int a = 3; a < 11; ++a) A.d[a][dst] = v[j][a];
            A.type[dst] = ty[j];
            A.gid[dst] = id[j];
            copy_fields(A.f, src[j], dst);
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------------- halo

struct TileBounds {
    double lo[3], hi[3];  // local.lower + width, local.upper - width
};

__device__ __forceinline__ TileBounds halo_bounds(const Grid& G, int s) {
    TileBounds b;
    const int packed = G.coord[s];
    const int c[3] = {packed >> 20, (packed >> 10) & 1023, packed & 1023};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double* cuts = G.cuts + G.cut_offset[a];
        b.lo[a] = __dadd_rn(cuts[c[a]], G.width);
        b.hi[a] = __dsub_rn(cuts[c[a] + 1], G.width);
    }
    return b;
}

// Host halo classification (dsDecompX src/halo.cpp:200-221): six strict
// comparisons, then the neighbor mask from the subdomain's lookup table.
__device__ __forceinline__ unsigned halo_mask(const TileBounds& b, const unsigned* lut, double px,
                                              double py, double pz) {
    const unsigned flags = (px < b.lo[0] ? 1u : 0u) | (px > b.hi[0] ? 2u : 0u) |
                           (py < b.lo[1] ? 4u : 0u) | (py > b.hi[1] ? 8u : 0u) |
                           (pz < b.lo[2] ? 16u : 0u) | (pz > b.hi[2] ? 32u : 0u);
    return flags ? lut[flags] : 0u;   // shared or global table
}

// Adds this warp's contribution of one 32-particle group to the per-lane
// counters (lane n < 26: send list n, lane 26: boundary owners, lane 27: images).
__device__ __forceinline__ void count_group(unsigned m, int nn, int lane, int& acc) {
    (void)nn;
    const unsigned any = __ballot_sync(0xffffffffu, m != 0);
    if (!any) return;
    // only the neighbors some lane of the warp sends to (a face particle of a
    // warp rarely touches more than a few of the 26)
    const unsigned used = __reduce_or_sync(0xffffffffu, m);
    for (unsigned rest = used; rest; rest &= rest - 1) {
        const int n = __ffs(rest) - 1;
        const unsigned b = __ballot_sync(0xffffffffu, (m >> n) & 1u);
        if (lane == n) acc += __popc(b);
    }
    const int total_images = __reduce_add_sync(0xffffffffu, __popc(m));
    if (lane == kBoundaryCounter) acc += __popc(any);
    if (lane == kImageCounter) acc += total_images;
}

// count_group over K groups at once (lane holds one particle of each): the
// same sums, one warp reduction per neighbor instead of one ballot per group.
template <int K>
__device__ __forceinline__ void count_groups(const unsigned (&m)[K], int lane, int& acc) {
    unsigned all = 0;
    int boundary = 0, images = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        all |= m[j];
        boundary += m[j] != 0u;
        images += __popc(m[j]);
    }
    const unsigned used = __reduce_or_sync(0xffffffffu, all);
    if (!used) return;
    for (unsigned rest = used; rest; rest &= rest - 1) {
        const int n = __ffs(rest) - 1;
        unsigned c = 0;
#pragma unroll
        for (int j = 0; j < K; ++j) c += (m[j] >> n) & 1u;
        const int total = static_cast<int>(__reduce_add_sync(0xffffffffu, c));
        if (lane == n) acc += total;
    }
    const int total_boundary = __reduce_add_sync(0xffffffffu, boundary);
    const int total_images = __reduce_add_sync(0xffffffffu, images);
    if (lane == kBoundaryCounter) acc += total_boundary;
    if (lane == kImageCounter) acc += total_images;
}

// Immigrant totals of one 32-particle group: a lane with key >= 0 holds an
// emigrant bound for subdomain `key` (-1: none) with the new owner's
// neighbor mask `me`, counted into the owner's total, boundary, image and
// per-list counters with one atomic per distinct destination of the warp.
// Every lane of the warp calls it.  It pays where the emigrants of a step are
// many and share few destinations (per-lane atomics on the same counters
// serialise); with a few emigrants per warp the match costs more than it
// saves, and the autotuner chooses.
__device__ __forceinline__ void add_immigrants(int key, unsigned me, int lane, int* total,
                                               int* bnd, int* img, int* list) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key < 0) return;
    const bool leader = lane == __ffs(peers) - 1;
    const int boundary = __reduce_add_sync(peers, me != 0u ? 1 : 0);
    const int images = __reduce_add_sync(peers, __popc(me));
    if (leader) {
        atomicAdd(&total[key], __popc(peers));
        if (boundary) {
            atomicAdd(&bnd[key], boundary);
            atomicAdd(&img[key], images);
        }
    }
    for (unsigned r = __reduce_or_sync(peers, me); r; r &= r - 1) {
        const int n = __ffs(r) - 1;
        const int c = __popc(__ballot_sync(peers, (me >> n) & 1u));
        if (leader) atomicAdd(&list[key * kMaxNeighbors + n], c);
    }
}

// H1: neighbor mask of every owned particle and per-tile list counts.
// `tiles`/`ntiles`: the tiles to classify (all owned particles of a layout,
// or the immigrant segments of a fused step).
__device__ __forceinline__ void halo_classify_tile(int g, const Grid& G,
                                                   const int4* __restrict__ tiles,
                                                   const double* __restrict__ x,
                                                   const double* __restrict__ y,
                                                   const double* __restrict__ z, unsigned* mask,
                                                   int* cnt, int stride) {
    __shared__ int s_cnt[NW][32];
    const int4 td = tiles[g];
    const int s = td.x, begin = td.y, end = td.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * ITEMS;
    const TileBounds b = halo_bounds(G, s);
    const unsigned* lut = G.lut + s * 64;
    const int nn = G.nn[s];
    int acc = 0;
    double px[ITEMS], py[ITEMS], pz[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        if (i < end) {
            px[j] = ro(x + i);
            py[j] = ro(y + i);
            pz[j] = ro(z + i);
        }
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        unsigned m = 0;
        if (i < end) {
            m = halo_mask(b, lut, px[j], py[j], pz[j]);
            mask[i] = m;
        }
        count_group(m, nn, lane, acc);
    }
    s_cnt[warp][lane] = acc;
    __syncthreads();
    if (threadIdx.x < kHaloCounters) {
        int sum = 0;
        for (int w = 0; w < NW; ++w) sum += s_cnt[w][threadIdx.x];
        cnt[threadIdx.x * stride + g] = sum;
    }
}

// The blocks stride over the tiles, so a launch may be smaller than the tile
// count (the immigrant segments of a step are few and counted on the device).
__global__ void __launch_bounds__(NT) k_halo_classify(Grid G, const int4* __restrict__ tiles,
                                                      const int* ntiles,
                                                      const double* __restrict__ x,
                                                      const double* __restrict__ y,
                                                      const double* __restrict__ z,
                                                      unsigned* mask, int* cnt, int stride) {
    pdl_begin();
    const int nt = tile_limit(G, ntiles);
    for (int g = G.tile_first + blockIdx.x; g < nt; g += gridDim.x) {
        halo_classify_tile(g, G, tiles, x, y, z, mask, cnt, stride);
        __syncthreads();
    }
}

// S2b: send-list lengths, receiver ghost layout (blocks in the receiver's
// neighbor order, dsDecompX src/halo.cpp:609-649) and the first ghost slot of
// every send list.  One CTA, one thread per receiver.
__global__ void __launch_bounds__(1024) k_halo_layout(Grid G, const int* pre, int stride,
                                                       int* list_len, int* send_base, int* gq,
                                                       int* gbase, int* boff, int* info,
                                                       int* cbase) {
    pdl_begin();
    __shared__ int ws[33];
    __shared__ int s_rcv[kMaxRanks + 1];
    const int P = G.P;
    const int ntiles = G.tile_start[P];
    for (int idx = threadIdx.x; idx < P * kMaxNeighbors; idx += blockDim.x) {
        const int r = idx / kMaxNeighbors, n = idx % kMaxNeighbors;
        int len = 0;
        if (n < G.nn[r] && G.nbr[idx] >= 0)
            len = pre[n * stride + G.tile_start[r + 1]] - pre[n * stride + G.tile_start[r]];
        list_len[idx] = len;
    }
    __syncthreads();
    // receivers, one warp each: lane m reads the block of neighbor m
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int r = warp; r < P; r += nwarps) {
        int len = 0;
        if (lane < G.nn[r]) {
            const int e = G.sender_of[r * kMaxNeighbors + lane];
            len = e >= 0 ? list_len[e] : 0;
        }
        const int sum = __reduce_add_sync(0xffffffffu, len);
        if (lane == 0) s_rcv[r] = sum;
    }
    __syncthreads();
    const int q = threadIdx.x;
    const int mine = q < P ? s_rcv[q] : 0;
    int total;
    const int excl = block_scan_excl<1024>(mine, total, ws);
    if (q < P) {
        gq[q] = mine;
        gbase[q] = excl;
        s_rcv[q] = excl;
    }
    __syncthreads();
    for (int r = warp; r < P; r += nwarps) {
        int len = 0, e = -1;
        if (lane < G.nn[r]) {
            e = G.sender_of[r * kMaxNeighbors + lane];
            len = e >= 0 ? list_len[e] : 0;
        }
        const int incl = warp_inclusive_sum(len);
        if (e >= 0) send_base[e] = s_rcv[r] + incl - len;
    }
    if (q == 0) {
        gbase[P] = total;
        const int B = pre[kBoundaryCounter * stride + ntiles];
        const int images = pre[kImageCounter * stride + ntiles];
        info[0] = total;
        info[1] = B;
        if (static_cast<long long>(total) > G.gcap) {
            atomicOr(G.status, kStatusGhostOverflow);
        } else {
            boff[B] = images;
        }
    }
    __syncthreads();
    // per subdomain and counter, the value that turns a tile prefix into the
    // global index: first slot of each send list, boundary/image prefixes
    for (int idx = threadIdx.x; idx < P * kHaloCounters; idx += blockDim.x) {
        const int r = idx / kHaloCounters, k = idx % kHaloCounters;
        int v;
        if (k < kMaxNeighbors) v = (k < G.nn[r] && G.nbr[r * kMaxNeighbors + k] >= 0) ? send_base[r * kMaxNeighbors + k] : 0;
        else v = pre[k * stride + G.tile_start[r]];
        cbase[idx] = v;
    }
}

// Ghost images a tile stages in shared memory before writing them out; a tile
// with more images (only possible with a halo wider than half a cell) writes
// them directly instead.
constexpr int kStageCap = 3072;

__device__ __forceinline__ void write_ghost(const Arrays& A, long long src, long long gi,
                                            const double* sh) {
    const double px = ro(A.d[0] + src), py = ro(A.d[1] + src), pz = ro(A.d[2] + src);
    const double vx = ro(A.d[3] + src), vy = ro(A.d[4] + src), vz = ro(A.d[5] + src);
    const double ms = ro(A.d[9] + src), ch = ro(A.d[10] + src);
    const int ty = ro(A.type + src), id = ro(A.gid + src);
    A.d[0][gi] = __dadd_rn(px, sh[0]);
    A.d[1][gi] = __dadd_rn(py, sh[1]);
    A.d[2][gi] = __dadd_rn(pz, sh[2]);
    A.d[3][gi] = vx; A.d[4][gi] = vy; A.d[5][gi] = vz;
    A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
    A.d[9][gi] = ms; A.d[10][gi] = ch;
    A.type[gi] = ty; A.gid[gi] = id;
    copy_fields(A.f, src, gi);
}

// H2: every (owner, neighbor) hit becomes a ghost in the receiver's block --
// x + shift, v, f = 0, mass, charge, type, id and the registered fields, as
// the reference's make_record + copy_record leave it (dsDecompX
// src/halo.cpp:37-55, src/runtime.cpp:82-96) -- plus the ghost -> owner map
// and the owner -> ghosts CSR that reverse_halo sums in neighbor order.
//
// The warps first rank every hit (ballot + popc) and stage the tile's images
// in shared memory list by list; the whole CTA then writes each list's slice
// of the ghost region with consecutive threads on consecutive slots, so every
// array is written with full, coalesced runs.
__device__ __forceinline__ void halo_scatter_tile(int g, const Grid& G, const Arrays& A,
                                                  long long owned_off, long long ghost_off,
                                                  const int4* __restrict__ tiles,
                                                  const unsigned* __restrict__ mask,
                                                  const int* pre, int stride, const int* cbase,
                                                  int* ghost_owner, int* ghost_entry,
                                                  int* bowner, int* boff, int* bslot,
                                                  int* bfirst) {
    __shared__ int s_cnt[NW][32];
    __shared__ int s_base[32];
    __shared__ int s_off[kMaxNeighbors + 1];
    __shared__ unsigned short s_own[kStageCap];
    const int4 td = tiles[g];
    const int s = td.x, begin = td.y, end = td.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * ITEMS;
    const int nn = G.nn[s];
    const unsigned lt = lanemask_lt();

    unsigned m[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        m[j] = i < end ? mask[i] : 0u;
    }
    int acc = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) count_group(m[j], nn, lane, acc);
    s_cnt[warp][lane] = acc;
    if (threadIdx.x < kHaloCounters) {
        const int k = threadIdx.x;
        s_base[k] = cbase[s * kHaloCounters + k] + pre[k * stride + g] - pre[k * stride + td.w];
    }
    __syncthreads();
    if (warp == 0) {
        // staging offsets of the lists: lane n sums its list over the warps,
        // then an exclusive scan over the lanes
        int tot = 0;
        if (lane < nn)
            for (int w = 0; w < NW; ++w) tot += s_cnt[w][lane];
        const int incl = warp_inclusive_sum(tot);
        if (lane < nn) s_off[lane] = incl - tot;
        if (lane == 31) s_off[nn] = incl;
    }
    __syncthreads();
    const int Q = s_off[nn];
    const bool staged = Q <= kStageCap;
    // lane k carries counter k's running offset for this warp: the global
    // slot (run) and, for lists, the position in the staged array (lrun)
    int run = 0, lrun = 0;
    if (lane < kHaloCounters) {
        run = s_base[lane];
        if (lane < nn) lrun = s_off[lane];
        for (int w = 0; w < warp; ++w) {
            run += s_cnt[w][lane];
            lrun += s_cnt[w][lane];
        }
    }
    const double* shift = G.shift + static_cast<long long>(s) * kMaxNeighbors * 3;
#pragma unroll 1
    for (int j = 0; j < ITEMS; ++j) {
        const unsigned mj = m[j];
        const unsigned any = __ballot_sync(0xffffffffu, mj != 0);
        if (!any) continue;
        const int i = wbegin + j * 32 + lane;
        const int b = __shfl_sync(0xffffffffu, run, kBoundaryCounter) + __popc(any & lt);
        const int pm = __popc(mj);
        const int incl = warp_inclusive_sum(pm);
        const int img = __shfl_sync(0xffffffffu, run, kImageCounter) + incl - pm;
        if (mj) {
            bowner[b] = i;
            boff[b] = img;
        }
        int k = 0;
        const unsigned used = __reduce_or_sync(0xffffffffu, mj);
        for (unsigned rest = used; rest; rest &= rest - 1) {
            const int n = __ffs(rest) - 1;
            const unsigned hit = __ballot_sync(0xffffffffu, (mj >> n) & 1u);
            const int list_base = __shfl_sync(0xffffffffu, run, n);
            const int stage_base = __shfl_sync(0xffffffffu, lrun, n);
            if ((mj >> n) & 1u) {
                const int rank = __popc(hit & lt);
                const int slot = list_base + rank;
                bslot[img + k] = slot;
                if (k == 0) bfirst[b] = slot;
                ++k;
                if (staged) {
                    s_own[stage_base + rank] = static_cast<unsigned short>(i - begin);
                } else {
                    write_ghost(A, owned_off + i, ghost_off + slot, shift + 3 * n);
                    ghost_owner[slot] = i;
                    ghost_entry[slot] = s * kMaxNeighbors + n;
                }
            }
            if (lane == n) {
                run += __popc(hit);
                lrun += __popc(hit);
            }
        }
        const int group_images = __shfl_sync(0xffffffffu, incl, 31);
        if (lane == kBoundaryCounter) run += __popc(any);
        if (lane == kImageCounter) run += group_images;
    }
    if (!staged) return;
    __syncthreads();
    for (int q = threadIdx.x; q < Q; q += NT) {
        int lo = 0, hi = nn;   // largest n with s_off[n] <= q
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_off[mid] <= q) lo = mid;
            else hi = mid;
        }
        const int n = lo;
        const int slot = s_base[n] + (q - s_off[n]);
        const int i = begin + s_own[q];
        write_ghost(A, owned_off + i, ghost_off + slot, shift + 3 * n);
        ghost_owner[slot] = i;
        ghost_entry[slot] = s * kMaxNeighbors + n;
    }
}

__global__ void __launch_bounds__(NT) k_halo_scatter(Grid G, Arrays A, long long owned_off,
                                                     long long ghost_off,
                                                     const int4* __restrict__ tiles,
                                                     const int* ntiles,
                                                     const unsigned* __restrict__ mask,
                                                     const int* pre, int stride,
                                                     const int* cbase, int* ghost_owner,
                                                     int* ghost_entry, int* bowner, int* boff,
                                                     int* bslot, int* bfirst) {
    pdl_begin();
    if (*G.status & kStatusGhostOverflow) return;
    const int nt = tile_limit(G, ntiles);
    for (int g = G.tile_first + blockIdx.x; g < nt; g += gridDim.x) {
        halo_scatter_tile(g, G, A, owned_off, ghost_off, tiles, mask, pre, stride, cbase,
                          ghost_owner, ghost_entry, bowner, boff, bslot, bfirst);
        __syncthreads();
    }
}

// ------------------------------------------------------------- fused step
//
// A batched step runs migrate and the plan build as one pipeline, so each
// owned record is read once: the classify pass already knows every
// particle's destination and its halo mask there (the mask of the particle's
// NEW owner, computed from its wrapped position), the move pass writes a
// retained particle to its new slot and, from the same registers, its ghost
// images; the few immigrants get theirs in a small pass over their segments.
// The result is the same as migrate followed by a rebuild: a send list
// L(r, n) is r's retained particles with bit n (old order, which is their new
// order) followed by r's immigrants with bit n (immigrant order).

// counters per tile of the old layout: 0..25 retained send lists, 26 retained
// boundary owners, 27 retained images, 28 stays, 29 emigrants
constexpr int kStepCounters = 30;
constexpr int kStepStay = 28;
constexpr int kStepEmig = 29;

__device__ __forceinline__ double wrap_if(const Grid& G, int a, double v) {
    return G.periodic[a] ? wrap_axis(v, G.lower[a], G.extent[a]) : v;
}

// F1: destination and new-owner halo mask of every owned particle; per-tile
// counters; per-destination totals of the emigrants (atomics: only sums;
// COMBINE: one per destination and warp, add_immigrants).
template <int CT, int MINB, bool COMBINE>
__global__ void __launch_bounds__(CT, MINB) k_step_classify(Grid G, const double* __restrict__ x,
                                                      const double* __restrict__ y,
                                                      const double* __restrict__ z, int* cnt,
                                                      int stride, int* imm_total, int* imm_list,
                                                      int* imm_bnd, int* imm_img,
                                                      unsigned short* __restrict__ dest_out,
                                                      unsigned* __restrict__ mask_out,
                                                      int* pairs) {
    pdl_begin();
    constexpr int CI = TILE / CT;   // 32-particle groups per warp
    constexpr int CW = CT / 32;
    static_assert(CI * CT == TILE && CW >= 1, "tile split");
    __shared__ int s_cnt[CW][32];
    __shared__ unsigned s_lut[64];   // the subdomain's halo flags -> neighbor mask
    __shared__ unsigned short s_queue[TILE];   // tile slots left to the general path
    __shared__ int s_qn;
    const int g = blockIdx.x;
    // the descriptor is read together with the tile count (the table has a
    // row for every block of the launch)
    const int4 td = G.tiles[g];
    if (g >= G.tile_start[G.P]) return;
    const int s = td.x, begin = td.y, end = td.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * CI;
    double px[CI], py[CI], pz[CI];
#pragma unroll
    for (int j = 0; j < CI; ++j) {
        const int i = wbegin + j * 32 + lane;
        if (i < end) {
            px[j] = ro(x + i);
            py[j] = ro(y + i);
            pz[j] = ro(z + i);
        }
    }
    const TileBounds bs = halo_bounds(G, s);
    const Cell cell = cell_of(G, s);
    for (int f = threadIdx.x; f < 64; f += CT) s_lut[f] = G.lut[s * 64 + f];
    if (threadIdx.x == 0) s_qn = 0;
    __syncthreads();
    const unsigned* lut = s_lut;
    const int nn = G.nn[s];
    // with every periodic axis starting at 0, a coordinate inside its own
    // cell needs no wrap arithmetic: both Host wraps return it (a -0 as +0)
    const bool simple = (!G.periodic[0] || G.lower[0] == 0.0) &&
                        (!G.periodic[1] || G.lower[1] == 0.0) &&
                        (!G.periodic[2] || G.lower[2] == 0.0);
    int acc = 0;
    unsigned m[CI];
    int fast = 0;   // this lane's particles that stay inside their own cell
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < CI; ++j) {
        const int i = wbegin + j * 32 + lane;
        const bool valid = i < end;
        const bool own = valid && simple && cell.lo[0] <= px[j] && px[j] < cell.hi[0] &&
                         cell.lo[1] <= py[j] && py[j] < cell.hi[1] && cell.lo[2] <= pz[j] &&
                         pz[j] < cell.hi[2];
        m[j] = 0;
        if (own) {
            // stays: destination s, mask of the own subdomain
            const double wx = G.periodic[0] && px[j] == 0.0 ? 0.0 : px[j];
            const double wy = G.periodic[1] && py[j] == 0.0 ? 0.0 : py[j];
            const double wz = G.periodic[2] && pz[j] == 0.0 ? 0.0 : pz[j];
            m[j] = halo_mask(bs, lut, wx, wy, wz);
            dest_out[static_cast<long long>(g) * TILE + (i - begin)] = static_cast<unsigned short>(s);
            mask_out[static_cast<long long>(g) * TILE + (i - begin)] = m[j];
            ++fast;
        }
        // every other particle of the tile waits in a queue for the
        // general path (one slot per particle; one shared atomic per group)
        const unsigned queued = __ballot_sync(0xffffffffu, valid && !own);
        if (queued) {
            int at = 0;
            if (lane == 0) at = atomicAdd(&s_qn, __popc(queued));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (valid && !own) s_queue[at + __popc(queued & lt)] = static_cast<unsigned short>(i - begin);
        }
    }
    count_groups<CI>(m, lane, acc);
    const int fast_stays = __reduce_add_sync(0xffffffffu, fast);
    if (lane == kStepStay) acc += fast_stays;
    __syncthreads();
    // The general path, 32 queued particles per warp and pass (a group with
    // one leaver no longer runs it for all 32 lanes); it re-reads the
    // positions, still in L1.
    const int nq = s_qn;
#pragma unroll 1
    for (int q0 = warp * 32; q0 < nq; q0 += CW * 32) {
        const int q = q0 + lane;
        const int i = q < nq ? begin + s_queue[q] : end;
        int d = -1;
        unsigned mg = 0, me = 0;
        if (i < end) {
            double wx, wy, wz;
            d = destination_near(G, cell, ro(x + i), ro(y + i), ro(z + i), wx, wy, wz);
            dest_out[static_cast<long long>(g) * TILE + (i - begin)] = static_cast<unsigned short>(d);
            if (d == s) {
                mg = halo_mask(bs, lut, wx, wy, wz);
                mask_out[static_cast<long long>(g) * TILE + (i - begin)] = mg;
            } else {
                me = halo_mask(halo_bounds(G, d), G.lut + d * 64, wx, wy, wz);
                // emigrants per (destination, source), for a sharded step
                if (pairs) atomicAdd(&pairs[d * G.P + s], 1);
                if constexpr (!COMBINE) {
                    atomicAdd(&imm_total[d], 1);
                    if (me) {
                        atomicAdd(&imm_bnd[d], 1);
                        atomicAdd(&imm_img[d], __popc(me));
                        for (unsigned r = me; r; r &= r - 1)
                            atomicAdd(&imm_list[d * kMaxNeighbors + __ffs(r) - 1], 1);
                    }
                }
            }
        }
        if constexpr (COMBINE)
            add_immigrants(d >= 0 && d != s ? d : -1, me, lane, imm_total, imm_bnd, imm_img, imm_list);
        count_group(mg, nn, lane, acc);
        const int stays = __popc(__ballot_sync(0xffffffffu, d == s));
        const int emigs = __popc(__ballot_sync(0xffffffffu, d >= 0 && d != s));
        if (lane == kStepStay) acc += stays;
        if (lane == kStepEmig) acc += emigs;
    }
    s_cnt[warp][lane] = acc;
    __syncthreads();
    if (threadIdx.x < kStepCounters) {
        int sum = 0;
        for (int w = 0; w < CW; ++w) sum += s_cnt[w][threadIdx.x];
        cnt[threadIdx.x * stride + g] = sum;
    }
}

// F3: the new owned layout, the ghost layout of the whole plan (retained +
// immigrant parts of every send list), the CSR bases and the immigrant
// segments.  One CTA, one thread per subdomain.
struct StepTables {
    int* imm_total;
    int* imm_list;
    int* imm_bnd;
    int* imm_img;
    int* imm_base;
    int* emig_info;
    long long* results;
    int* list_ret;
    int* list_len;
    int* send_base;
    int* gq;
    int* gbase;
    int* boff;
    int* info;
    int* cbase_ret;
    int* cbase_imm;
    int* imm_tile_start;
    int4* imm_tiles;
};

__device__ __forceinline__ void step_layout_body(const Grid& G, const int* pre, int stride,
                                                 const StepTables& T);

// The counter scan (one CTA per counter) and, in the CTA that finishes
// last, the layout: one launch instead of two.  The last CTA reads the
// prefixes the others wrote through L2 (after the fence that orders them
// before its ticket) and puts the ticket back to 0 for the next launch.
__global__ void __launch_bounds__(1024) k_step_scan_layout(Grid G, const int* cnt, int* pre,
                                                            int stride, StepTables T,
                                                            unsigned* ticket) {
    pdl_begin();
    __shared__ bool s_last;
    scan_counter(cnt, pre, stride, G.tile_start + G.P);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    step_layout_body(G, pre, stride, T);
    if (threadIdx.x == 0) *ticket = 0u;
}

__device__ __forceinline__ void step_layout_body(const Grid& G, const int* pre, int stride,
                                                 const StepTables& T) {
    __shared__ int ws[33];
    __shared__ int s_rcv[kMaxRanks + 1];
    __shared__ int s_ts[kMaxRanks + 1];   // the current layout's tile starts, staged once
    const int P = G.P;
    const int t = threadIdx.x;
    for (int k = t; k <= P; k += blockDim.x) s_ts[k] = G.tile_start[k];
    __syncthreads();
    const int ntiles = s_ts[P];
    const int* ts_old = s_ts;
    auto tile_sum = [&](int k, int r) {
        return __ldcg(pre + k * stride + ts_old[r + 1]) - __ldcg(pre + k * stride + ts_old[r]);
    };
    // new owned layout and migration results
    int retained = 0, received = 0, old = 0, next = 0;
    if (t < P) {
        retained = tile_sum(kStepStay, t);
        received = T.imm_total[t];
        old = G.n[t];
        next = retained + received;
    }
    int total_next, total_tiles, total_imm_tiles;
    const int ob = block_scan_excl<1024>(next, total_next, ws);
    const int ntl = t < P ? (next + G.tile - 1) / G.tile : 0;
    const int ts = block_scan_excl<1024>(ntl, total_tiles, ws);
    const int itl = t < P ? (received + G.tile - 1) / G.tile : 0;
    const int its = block_scan_excl<1024>(itl, total_imm_tiles, ws);
    if (t < P) {
        G.n_next[t] = next;
        G.obase_next[t] = ob;
        G.tile_start_next[t] = ts;
        T.imm_base[t] = ob + retained;
        T.imm_tile_start[t] = its;
        long long* o = T.results + 6 * t;
        o[1] = old;
        o[2] = retained;
        o[3] = old - retained;
        o[4] = received;
        o[5] = next;
        o[0] = (o[3] != 0 || o[4] != 0) ? 1 : 0;
    }
    if (t == 0) {
        G.obase_next[P] = total_next;
        G.tile_start_next[P] = total_tiles;
        T.imm_tile_start[P] = total_imm_tiles;
        const int E = __ldcg(pre + kStepEmig * stride + ntiles);
        T.emig_info[0] = E;
        T.emig_info[1] = (E + TILE - 1) / TILE;
        if (total_next != G.obase[P]) atomicOr(G.status, kStatusMigrationMismatch);
    }
    // send-list lengths: retained part from the tile prefixes, immigrant part
    // from the atomics of F1
    for (int idx = t; idx < P * kMaxNeighbors; idx += blockDim.x) {
        const int r = idx / kMaxNeighbors, n = idx % kMaxNeighbors;
        const bool active = n < G.nn[r] && G.nbr[idx] >= 0;
        const int ret = active ? tile_sum(n, r) : 0;
        T.list_ret[idx] = ret;
        T.list_len[idx] = active ? ret + T.imm_list[idx] : 0;
    }
    __syncthreads();
    // (the tile descriptors of the next layout and of the immigrant segments
    // are written by k_tile_bases, over the whole grid)
    // receivers: blocks in the receiver's neighbor order, one warp per
    // receiver (lane m reads the block of neighbor m)
    const int warp = t >> 5, lane = t & 31, nwarps = blockDim.x >> 5;
    for (int q = warp; q < P; q += nwarps) {
        int len = 0;
        if (lane < G.nn[q]) {
            const int e = G.sender_of[q * kMaxNeighbors + lane];
            len = e >= 0 ? T.list_len[e] : 0;
        }
        const int sum = __reduce_add_sync(0xffffffffu, len);
        if (lane == 0) s_rcv[q] = sum;
    }
    __syncthreads();
    const int mine = t < P ? s_rcv[t] : 0;
    int total_ghosts;
    const int gb = block_scan_excl<1024>(mine, total_ghosts, ws);
    if (t < P) {
        T.gq[t] = mine;
        T.gbase[t] = gb;
        s_rcv[t] = gb;
    }
    __syncthreads();
    for (int q = warp; q < P; q += nwarps) {
        int len = 0, e = -1;
        if (lane < G.nn[q]) {
            e = G.sender_of[q * kMaxNeighbors + lane];
            len = e >= 0 ? T.list_len[e] : 0;
        }
        const int incl = warp_inclusive_sum(len);
        if (e >= 0) T.send_base[e] = s_rcv[q] + incl - len;
    }
    // boundary owners and images: retained part first, then the immigrants
    int bret = 0, bimm = 0, iret = 0, iimm = 0;
    if (t < P) {
        bret = tile_sum(kBoundaryCounter, t);
        bimm = T.imm_bnd[t];
        iret = tile_sum(kImageCounter, t);
        iimm = T.imm_img[t];
    }
    int total_b, total_i;
    const int bb = block_scan_excl<1024>(bret + bimm, total_b, ws);
    const int ib = block_scan_excl<1024>(iret + iimm, total_i, ws);   // syncs: send_base complete
    for (int e = t; e < P * kMaxNeighbors; e += blockDim.x) {
        const int r = e / kMaxNeighbors, n = e % kMaxNeighbors;
        const bool active = n < G.nn[r] && G.nbr[e] >= 0;
        T.cbase_ret[r * kHaloCounters + n] = active ? T.send_base[e] : 0;
        T.cbase_imm[r * kHaloCounters + n] = active ? T.send_base[e] + T.list_ret[e] : 0;
    }
    if (t < P) {
        int* cr = T.cbase_ret + t * kHaloCounters;
        int* ci = T.cbase_imm + t * kHaloCounters;
        cr[kBoundaryCounter] = bb;
        ci[kBoundaryCounter] = bb + bret;
        cr[kImageCounter] = ib;
        ci[kImageCounter] = ib + iret;
    }
    if (t == 0) {
        T.gbase[P] = total_ghosts;
        T.info[0] = total_ghosts;
        T.info[1] = total_b;
        if (static_cast<long long>(total_ghosts) > G.gcap) atomicOr(G.status, kStatusGhostOverflow);
        else T.boff[total_b] = total_i;
    }
}

__device__ __forceinline__ void write_ghost_wrapped(const Grid& G, const Arrays& A, long long src,
                                                    long long gi, const double* sh) {
    const double px = wrap_if(G, 0, ro(A.d[0] + src));
    const double py = wrap_if(G, 1, ro(A.d[1] + src));
    const double pz = wrap_if(G, 2, ro(A.d[2] + src));
    const double vx = ro(A.d[3] + src), vy = ro(A.d[4] + src), vz = ro(A.d[5] + src);
    const double ms = ro(A.d[9] + src), ch = ro(A.d[10] + src);
    const int ty = ro(A.type + src), id = ro(A.gid + src);
    A.d[0][gi] = __dadd_rn(px, sh[0]);
    A.d[1][gi] = __dadd_rn(py, sh[1]);
    A.d[2][gi] = __dadd_rn(pz, sh[2]);
    A.d[3][gi] = vx; A.d[4][gi] = vy; A.d[5][gi] = vz;
    A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
    A.d[9][gi] = ms; A.d[10][gi] = ch;
    A.type[gi] = ty; A.gid[gi] = id;
    copy_fields(A.f, src, gi);
}

// F4: retained particles move to their new slots (stable) and write their
// ghost images (staged per tile, then written list by list with coalesced
// stores); emigrants are listed for the multi-split.  On a ghost overflow the
// move still completes (the engine grows the ghost region and rebuilds).
__global__ void __launch_bounds__(NT, 4) k_step_move(Grid G, Arrays A, long long src_off,
                                                  long long dst_off, long long ghost_off,
                                                  const int* pre, int stride, const int* cbase_ret,
                                                  const unsigned short* __restrict__ dest_in,
                                                  const unsigned* __restrict__ mask_in,
                                                  int* emig_src, int* emig_dst, int* ghost_owner,
                                                  int* ghost_entry, int* bowner, int* boff,
                                                  int* bslot, int* bfirst) {
    pdl_begin();
    __shared__ int s_cnt[NW][32];
    __shared__ int s_base[32];
    __shared__ int s_off[kMaxNeighbors + 1];
    __shared__ unsigned short s_own[kStageCap];
    __shared__ int s_ni[TILE];
    const int g = blockIdx.x;
    if (g >= G.tile_start[G.P]) return;
    const bool ghosts = !(*G.status & kStatusGhostOverflow);
    const int4 td = G.tiles[g];
    const int s = td.x, begin = td.y, end = td.z, first = td.w;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * ITEMS;
    const int nn = G.nn[s];
    const unsigned lt = lanemask_lt();

    int dest[ITEMS];
    unsigned msk[ITEMS];
    int acc = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        dest[j] = -1;
        msk[j] = 0;
        if (i < end) {
            dest[j] = dest_in[static_cast<long long>(g) * TILE + (i - begin)];
            if (dest[j] == s) msk[j] = mask_in[static_cast<long long>(g) * TILE + (i - begin)];
        }
        count_group(msk[j], nn, lane, acc);
        const int stays = __popc(__ballot_sync(0xffffffffu, dest[j] == s));
        const int emigs = __popc(__ballot_sync(0xffffffffu, dest[j] >= 0 && dest[j] != s));
        if (lane == kStepStay) acc += stays;
        if (lane == kStepEmig) acc += emigs;
    }
    s_cnt[warp][lane] = acc;
    if (threadIdx.x < kStepCounters) {
        const int k = threadIdx.x;
        int base;
        if (k < kHaloCounters) base = cbase_ret[s * kHaloCounters + k] + pre[k * stride + g] - pre[k * stride + first];
        else if (k == kStepStay) base = G.obase_next[s] + pre[k * stride + g] - pre[k * stride + first];
        else base = pre[k * stride + g];
        s_base[k] = base;
    }
    __syncthreads();
    if (warp == 0) {
        // staging offsets of the lists: lane n sums its list over the warps,
        // then an exclusive scan over the lanes
        int tot = 0;
        if (lane < nn)
            for (int w = 0; w < NW; ++w) tot += s_cnt[w][lane];
        const int incl = warp_inclusive_sum(tot);
        if (lane < nn) s_off[lane] = incl - tot;
        if (lane == 31) s_off[nn] = incl;
    }
    __syncthreads();
    const int Q = s_off[nn];
    const bool staged = Q <= kStageCap;
    int run = 0, lrun = 0;
    if (lane < kStepCounters) {
        run = s_base[lane];
        if (lane < nn) lrun = s_off[lane];
        for (int w = 0; w < warp; ++w) {
            run += s_cnt[w][lane];
            lrun += s_cnt[w][lane];
        }
    }
    const double* shift = G.shift + static_cast<long long>(s) * kMaxNeighbors * 3;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        const bool stay = dest[j] == s;
        const bool emig = dest[j] >= 0 && !stay;
        const unsigned bs_ = __ballot_sync(0xffffffffu, stay);
        const unsigned be = __ballot_sync(0xffffffffu, emig);
        const int ni = __shfl_sync(0xffffffffu, run, kStepStay) + __popc(bs_ & lt);
        const int eb = __shfl_sync(0xffffffffu, run, kStepEmig) + __popc(be & lt);
        if (stay) {
            const long long src = src_off + i;
            move_record(A, src, dst_off + ni, wrap_if(G, 0, ro(A.d[0] + src)),
                        wrap_if(G, 1, ro(A.d[1] + src)), wrap_if(G, 2, ro(A.d[2] + src)));
            s_ni[i - begin] = ni;
        } else if (emig) {
            emig_src[eb] = i;
            emig_dst[eb] = dest[j];
        }
        const unsigned mj = ghosts ? msk[j] : 0u;
        const unsigned any = __ballot_sync(0xffffffffu, mj != 0);
        if (any) {
            const int b = __shfl_sync(0xffffffffu, run, kBoundaryCounter) + __popc(any & lt);
            const int pm = __popc(mj);
            const int incl = warp_inclusive_sum(pm);
            const int img = __shfl_sync(0xffffffffu, run, kImageCounter) + incl - pm;
            if (mj) {
                bowner[b] = ni;
                boff[b] = img;
            }
            int k = 0;
            const unsigned used = __reduce_or_sync(0xffffffffu, mj);
            for (unsigned rest = used; rest; rest &= rest - 1) {
                const int n = __ffs(rest) - 1;
                const unsigned hit = __ballot_sync(0xffffffffu, (mj >> n) & 1u);
                const int list_base = __shfl_sync(0xffffffffu, run, n);
                const int stage_base = __shfl_sync(0xffffffffu, lrun, n);
                if ((mj >> n) & 1u) {
                    const int rank = __popc(hit & lt);
                    const int slot = list_base + rank;
                    bslot[img + k] = slot;
                    if (k == 0) bfirst[b] = slot;
                    ++k;
                    if (staged) {
                        s_own[stage_base + rank] = static_cast<unsigned short>(i - begin);
                    } else {
                        write_ghost_wrapped(G, A, src_off + i, ghost_off + slot, shift + 3 * n);
                        ghost_owner[slot] = ni;
                        ghost_entry[slot] = s * kMaxNeighbors + n;
                    }
                }
                if (lane == n) {
                    run += __popc(hit);
                    lrun += __popc(hit);
                }
            }
            const int group_images = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == kBoundaryCounter) run += __popc(any);
            if (lane == kImageCounter) run += group_images;
        }
        if (lane == kStepStay) run += __popc(bs_);
        if (lane == kStepEmig) run += __popc(be);
    }
    if (!ghosts || !staged) return;
    __syncthreads();
    for (int q = threadIdx.x; q < Q; q += NT) {
        int lo = 0, hi = nn;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_off[mid] <= q) lo = mid;
            else hi = mid;
        }
        const int n = lo;
        const int slot = s_base[n] + (q - s_off[n]);
        const int l = s_own[q];
        write_ghost_wrapped(G, A, src_off + begin + l, ghost_off + slot, shift + 3 * n);
        ghost_owner[slot] = s_ni[l];
        ghost_entry[slot] = s * kMaxNeighbors + n;
    }
}

// ------------------------------------------------------------ bulk staging
// The staged move brings a tile's records into shared memory with the TMA
// unit (cp.async.bulk, completion counted in bytes on an mbarrier) while the
// block reads the destinations and combines its counts; the move and the ghost
// images then read shared memory, so each record crosses HBM once and the
// copies are in flight from the block's first instruction.

constexpr int kStagedArrays = 13 + kMaxFields;
constexpr int kStagedMaxBytes = 100 * 1024;         // dynamic shared memory cap
constexpr unsigned long long kBulkWaitNs = 1000000000ull;   // 1 s: a copy counts as lost

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes,
                                          unsigned bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

// Polls the mbarrier's phase `parity` for at most kBulkWaitNs; false if it
// never completed.
__device__ __forceinline__ bool bulk_wait_parity(unsigned bar, unsigned parity) {
    const unsigned long long start = global_ns();
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
        if (global_ns() - start > kBulkWaitNs) return false;
    }
}

// Phase 0 (a barrier that completes once).
__device__ __forceinline__ bool bulk_wait(unsigned bar) { return bulk_wait_parity(bar, 0u); }

// Array k of the record (0..10 doubles, 11 type, 12 id, 13.. fields).
__device__ __forceinline__ int array_bytes(const Arrays& A, int k) {
    return k < 11 ? 8 : k < 13 ? 4 : A.f.bytes[k - 13];
}
__device__ __forceinline__ const unsigned char* array_base(const Arrays& A, int k) {
    if (k < 11) return reinterpret_cast<const unsigned char*>(A.d[k]);
    if (k == 11) return reinterpret_cast<const unsigned char*>(A.type);
    if (k == 12) return reinterpret_cast<const unsigned char*>(A.gid);
    return A.f.base[k - 13];
}

__device__ __forceinline__ double srd(const unsigned char* rec, int seg, int l) {
    return *reinterpret_cast<const double*>(rec + seg + l * 8);
}
__device__ __forceinline__ int sri(const unsigned char* rec, int seg, int l) {
    return *reinterpret_cast<const int*>(rec + seg + l * 4);
}

// Words of one field, four at a time: the four shared-memory loads are
// issued before the four stores (the generic pointers could otherwise alias,
// which would order every store before the next load).
template <class W>
__device__ __forceinline__ void copy_words_staged(const W* __restrict__ src, W* __restrict__ out,
                                                  int n) {
    for (int w0 = 0; w0 < n; w0 += 4) {
        W t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (w0 + u < n) t[u] = src[w0 + u];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (w0 + u < n) out[w0 + u] = t[u];
    }
}

__device__ __forceinline__ void fields_from_stage(const FieldSet& f, const unsigned char* rec,
                                                  const int* seg, int l, long long dst) {
    for (int k = 0; k < f.count; ++k) {
        const int b = f.bytes[k];
        const unsigned char* src = rec + seg[k] + l * b;
        unsigned char* out = f.base[k] + dst * b;
        if ((b & 7) == 0)
            copy_words_staged(reinterpret_cast<const unsigned long long*>(src),
                              reinterpret_cast<unsigned long long*>(out), b >> 3);
        else
            copy_words_staged(reinterpret_cast<const unsigned*>(src), reinterpret_cast<unsigned*>(out),
                              b >> 2);
    }
}

// Owned record l of the staged tile to slot dst, positions wrapped.  `sg`:
// where element 0 of each core array sits in `rec`, `fseg` the same for the
// fields (every value is read before the first store, so the reads overlap).
__device__ __forceinline__ void move_from_stage(const Grid& G, const Arrays& A,
                                                const unsigned char* rec, const int* sg,
                                                const int* fseg, int l, long long dst) {
    double v[11];
#pragma unroll
    for (int a = 0; a < 11; ++a) v[a] = srd(rec, sg[a], l);
    const int ty = sri(rec, sg[11], l), id = sri(rec, sg[12], l);
#pragma unroll
    for (int a = 0; a < 3; ++a) A.d[a][dst] = wrap_if(G, a, v[a]);
#pragma unroll
    for (int a = 3; a < 11; ++a) A.d[a][dst] = v[a];
    A.type[dst] = ty;
    A.gid[dst] = id;
    fields_from_stage(A.f, rec, fseg, l, dst);
}

// move_from_stage for a tile staged without its force arrays: the owner's
// forces come from HBM (fx, fy, fz), everything else from the stage.
__device__ __forceinline__ void move_from_stage_forces(const Grid& G, const Arrays& A,
                                                       const unsigned char* rec, const int* sg,
                                                       const int* fseg, int l, long long dst,
                                                       double fx, double fy, double fz) {
    double v[11];
#pragma unroll
    for (int a = 0; a < 11; ++a)
        if (a < 6 || a > 8) v[a] = srd(rec, sg[a], l);
    v[6] = fx;
    v[7] = fy;
    v[8] = fz;
    const int ty = sri(rec, sg[11], l), id = sri(rec, sg[12], l);
#pragma unroll
    for (int a = 0; a < 3; ++a) A.d[a][dst] = wrap_if(G, a, v[a]);
#pragma unroll
    for (int a = 3; a < 11; ++a) A.d[a][dst] = v[a];
    A.type[dst] = ty;
    A.gid[dst] = id;
    fields_from_stage(A.f, rec, fseg, l, dst);
}

// Ghost image of record l of the staged tile (plan-build semantics: wrapped
// position + shift, velocities, zero force, mass, charge, type, id, fields).
__device__ __forceinline__ void ghost_from_stage(const Grid& G, const Arrays& A,
                                                 const unsigned char* rec, const int* sg,
                                                 const int* fseg, int l, long long gi,
                                                 const double* sh) {
    double v[11];
#pragma unroll
    for (int a = 0; a < 11; ++a)
        if (a < 6 || a > 8) v[a] = srd(rec, sg[a], l);
    const int ty = sri(rec, sg[11], l), id = sri(rec, sg[12], l);
    const double s0 = sh[0], s1 = sh[1], s2 = sh[2];
    A.d[0][gi] = __dadd_rn(wrap_if(G, 0, v[0]), s0);
    A.d[1][gi] = __dadd_rn(wrap_if(G, 1, v[1]), s1);
    A.d[2][gi] = __dadd_rn(wrap_if(G, 2, v[2]), s2);
#pragma unroll
    for (int a = 3; a < 6; ++a) A.d[a][gi] = v[a];
    A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
    A.d[9][gi] = v[9];
    A.d[10][gi] = v[10];
    A.type[gi] = ty;
    A.gid[gi] = id;
    fields_from_stage(A.f, rec, fseg, l, gi);
}

// Warp 0 issues the bulk copies of elements [first, last) of a tile into a
// shared-memory buffer: each lane copies one array k of [a0, a1) (skipping
// the force arrays when asked) and stores in seg[k - a0] where element 0
// landed.  Lane 0 announces the byte total on the
// mbarrier before any copy starts.
__device__ __forceinline__ void stage_issue(const Arrays& A, long long src_off, int first,
                                            int last, unsigned char* stage, unsigned bar,
                                            int* seg, int lane, int a0, int a1,
                                            bool skip_forces = false) {
    // lane -> array: a0 + lane, stepping over the force arrays (6..8) when
    // they are read directly instead
    const int k = a0 + lane + (skip_forces && a0 + lane >= 6 ? 3 : 0);
    int b = 0;
    const unsigned char* base = nullptr;
    if (k < a1) {
        b = array_bytes(A, k);
        base = array_base(A, k);
    }
    const int size = b ? TILE * b + 32 : 0;
    const int soff = warp_inclusive_sum(size) - size;
    long long gl = 0, lo = 0, hi = 0;
    if (b) {
        gl = (src_off + first) * b;
        lo = gl & ~15LL;
        hi = ((src_off + last) * b + 15) & ~15LL;
    }
    const unsigned bytes = static_cast<unsigned>(hi - lo);
    const unsigned total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total)
                     : "memory");
    __syncwarp();
    if (b) {
        bulk_load(smem_u32(stage + soff), base + lo, bytes, bar);
        seg[k - a0] = soff + static_cast<int>(gl - lo);
    }
}

// Value of step counter k at tile g (the global running index of the tile's
// first entry): send-list slots, boundary/image offsets, new owned slots,
// emigrant slots.
__device__ __forceinline__ int tile_base(const Grid& G, const int* pre, int stride,
                                         const int* cbase_ret, int g, int4 td, int k) {
    const int s = td.x, first = td.w;
    if (k < kHaloCounters)
        return cbase_ret[s * kHaloCounters + k] + pre[k * stride + g] - pre[k * stride + first];
    if (k == kStepStay) return G.obase_next[s] + pre[k * stride + g] - pre[k * stride + first];
    return pre[k * stride + g];
}

// Array k of staged record l to owned slot dst (positions wrapped): the
// per-array form of move_from_stage for a move split into several passes.
__device__ __forceinline__ void move_array_from_stage(const Grid& G, const Arrays& A,
                                                      const unsigned char* rec, int seg, int k,
                                                      int l, long long dst) {
    if (k < 11) {
        const double v = srd(rec, seg, l);
        A.d[k][dst] = k < 3 ? wrap_if(G, k, v) : v;
    } else if (k < 13) {
        (k == 11 ? A.type : A.gid)[dst] = sri(rec, seg, l);
    } else {
        const int b = A.f.bytes[k - 13];
        const unsigned* src = reinterpret_cast<const unsigned*>(rec + seg + l * b);
        unsigned* out = reinterpret_cast<unsigned*>(A.f.base[k - 13] + dst * b);
        for (int w = 0; w < (b >> 2); ++w) out[w] = src[w];
    }
}

// Array k of the ghost image of staged record l (position + shift, zero
// force, the rest copied).
__device__ __forceinline__ void ghost_array_from_stage(const Grid& G, const Arrays& A,
                                                       const unsigned char* rec, int seg, int k,
                                                       int l, long long gi, const double* sh) {
    if (k < 3) {
        A.d[k][gi] = __dadd_rn(wrap_if(G, k, srd(rec, seg, l)), sh[k]);
    } else if (k >= 6 && k < 9) {
        A.d[k][gi] = 0.0;
    } else {
        move_array_from_stage(G, A, rec, seg, k, l, gi);
    }
}

// Ghost image of staged record l for a plan rebuild: the position as it is
// (the rebuild copies it without a wrap, like write_ghost) + shift,
// velocities, zero force, mass, charge, type, id, fields.
__device__ __forceinline__ void ghost_from_stage_unwrapped(const Arrays& A, const unsigned char* rec,
                                                           const int* sg, const int* fseg, int l,
                                                           long long gi, const double* sh) {
    double v[11];
#pragma unroll
    for (int a = 0; a < 11; ++a)
        if (a < 6 || a > 8) v[a] = srd(rec, sg[a], l);
    const int ty = sri(rec, sg[11], l), id = sri(rec, sg[12], l);
    A.d[0][gi] = __dadd_rn(v[0], sh[0]);
    A.d[1][gi] = __dadd_rn(v[1], sh[1]);
    A.d[2][gi] = __dadd_rn(v[2], sh[2]);
#pragma unroll
    for (int a = 3; a < 6; ++a) A.d[a][gi] = v[a];
    A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
    A.d[9][gi] = v[9];
    A.d[10][gi] = v[10];
    A.type[gi] = ty;
    A.gid[gi] = id;
    fields_from_stage(A.f, rec, fseg, l, gi);
}

// The plan build's scatter (same outputs as k_halo_scatter, one tile per
// block) with the tile's records brought into shared memory by bulk copies
// (every array but the forces, which a ghost does not carry) while the block
// ranks the tile's hits from the masks.  The images are then written list by
// list from shared memory, consecutive threads on consecutive ghost slots:
// the records cross HBM once, as whole tiles, instead of as one 32-byte
// sector per array and image.  A tile with more images than the staging
// list holds writes them from HBM reads during the ranking, as k_halo_scatter
// does.
__global__ void __launch_bounds__(NT, 4) k_halo_scatter_staged(
    Grid G, Arrays A, long long owned_off, long long ghost_off, const int4* __restrict__ tiles,
    const int* ntiles, const unsigned* __restrict__ mask, const int* pre, int stride,
    const int* cbase, int* ghost_owner, int* ghost_entry, int* bowner, int* boff, int* bslot,
    int* bfirst) {
    pdl_begin();
    extern __shared__ __align__(16) unsigned char s_rec[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ int s_seg[kStagedArrays];
    __shared__ int s_cnt[NW][32];
    __shared__ int s_base[32];
    __shared__ int s_off[kMaxNeighbors + 1];
    __shared__ unsigned short s_own[kStageCap];
    const int g = G.tile_first + blockIdx.x;
    if (g >= tile_limit(G, ntiles) || (*G.status & kStatusGhostOverflow)) return;
    const int4 td = tiles[g];
    const int s = td.x, begin = td.y, end = td.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * ITEMS;
    const unsigned bar = smem_u32(&s_bar);
    if (warp == 0) {
        if (lane == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
        stage_issue(A, owned_off, begin, end, s_rec, bar, s_seg, lane, 0, 13 + A.f.count, true);
    }
    const int nn = G.nn[s];
    const unsigned lt = lanemask_lt();
    unsigned m[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        m[j] = i < end ? mask[i] : 0u;
    }
    int acc = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) count_group(m[j], nn, lane, acc);
    s_cnt[warp][lane] = acc;
    if (threadIdx.x < kHaloCounters) {
        const int k = threadIdx.x;
        s_base[k] = cbase[s * kHaloCounters + k] + pre[k * stride + g] - pre[k * stride + td.w];
    }
    __syncthreads();
    if (warp == 0) {
        int tot = 0;
        if (lane < nn)
            for (int w = 0; w < NW; ++w) tot += s_cnt[w][lane];
        const int incl = warp_inclusive_sum(tot);
        if (lane < nn) s_off[lane] = incl - tot;
        if (lane == 31) s_off[nn] = incl;
    }
    __syncthreads();
    const int Q = s_off[nn];
    const bool staged = Q <= kStageCap;
    int run = 0, lrun = 0;
    if (lane < kHaloCounters) {
        run = s_base[lane];
        if (lane < nn) lrun = s_off[lane];
        for (int w = 0; w < warp; ++w) {
            run += s_cnt[w][lane];
            lrun += s_cnt[w][lane];
        }
    }
    const double* shift = G.shift + static_cast<long long>(s) * kMaxNeighbors * 3;
#pragma unroll 1
    for (int j = 0; j < ITEMS; ++j) {
        const unsigned mj = m[j];
        const unsigned any = __ballot_sync(0xffffffffu, mj != 0);
        if (!any) continue;
        const int i = wbegin + j * 32 + lane;
        const int b = __shfl_sync(0xffffffffu, run, kBoundaryCounter) + __popc(any & lt);
        const int pm = __popc(mj);
        const int incl = warp_inclusive_sum(pm);
        const int img = __shfl_sync(0xffffffffu, run, kImageCounter) + incl - pm;
        if (mj) {
            bowner[b] = i;
            boff[b] = img;
        }
        int k = 0;
        const unsigned used = __reduce_or_sync(0xffffffffu, mj);
        for (unsigned rest = used; rest; rest &= rest - 1) {
            const int n = __ffs(rest) - 1;
            const unsigned hit = __ballot_sync(0xffffffffu, (mj >> n) & 1u);
            const int list_base = __shfl_sync(0xffffffffu, run, n);
            const int stage_base = __shfl_sync(0xffffffffu, lrun, n);
            if ((mj >> n) & 1u) {
                const int rank = __popc(hit & lt);
                const int slot = list_base + rank;
                bslot[img + k] = slot;
                if (k == 0) bfirst[b] = slot;
                ++k;
                if (staged) {
                    s_own[stage_base + rank] = static_cast<unsigned short>(i - begin);
                } else {
                    write_ghost(A, owned_off + i, ghost_off + slot, shift + 3 * n);
                    ghost_owner[slot] = i;
                    ghost_entry[slot] = s * kMaxNeighbors + n;
                }
            }
            if (lane == n) {
                run += __popc(hit);
                lrun += __popc(hit);
            }
        }
        const int group_images = __shfl_sync(0xffffffffu, incl, 31);
        if (lane == kBoundaryCounter) run += __popc(any);
        if (lane == kImageCounter) run += group_images;
    }
    // the records must have landed (and every warp's staging list be
    // visible) before the images are written from shared memory
    const bool lost = !bulk_wait(bar);
    if (__syncthreads_or(lost)) {
        if (lost) bulk_wait(bar);   // copies still in flight get one more bounded wait
        if (threadIdx.x == 0) atomicOr(G.status, kStatusCopyTimeout);
        return;
    }
    if (!staged) return;
    int sg[13];
#pragma unroll
    for (int a = 0; a < 13; ++a) sg[a] = s_seg[a];
    const int* fseg = s_seg + 13;
    for (int q = threadIdx.x; q < Q; q += NT) {
        int lo = 0, hi = nn;   // largest n with s_off[n] <= q
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_off[mid] <= q) lo = mid;
            else hi = mid;
        }
        const int n = lo;
        const int slot = s_base[n] + (q - s_off[n]);
        const int l = s_own[q];
        ghost_from_stage_unwrapped(A, s_rec, sg, fseg, l, ghost_off + slot, shift + 3 * n);
        ghost_owner[slot] = begin + l;
        ghost_entry[slot] = s * kMaxNeighbors + n;
    }
}

// First boundary owner of every tile of the current layout (tile_b0[g]; the
// boundary owners are in owned order in every plan) and tile_b0[ntiles] = B.
__global__ void __launch_bounds__(NT) k_tile_boundary_starts(Grid G, const int* info,
                                                             const int* __restrict__ bowner,
                                                             int* tile_b0) {
    pdl_begin();
    const int ntiles = G.tile_start[G.P];
    const int B = info[1];
    for (int g = blockIdx.x * NT + threadIdx.x; g <= ntiles; g += gridDim.x * NT) {
        if (g == ntiles) {
            tile_b0[g] = B;
            continue;
        }
        const int begin = G.tiles[g].y;
        int lo = 0, hi = B;   // first b with bowner[b] >= begin
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ro(bowner + mid) < begin) lo = mid + 1;
            else hi = mid;
        }
        tile_b0[g] = lo;
    }
}

// Refresh along the plan, one tile of owners at a time: the arrays the
// refresh copies (x, y, z; with velocities and the registered fields for a
// full refresh) come into shared memory by bulk copies of the whole tile,
// while the block sorts the tile's images by ghost slot from the CSR (the
// images of one send list from one tile are a run of consecutive slots,
// every list being in owned order); then consecutive threads write
// consecutive ghost slots from shared memory.  Owned data crosses HBM once,
// as whole tiles, instead of one sector per array and ghost.  A tile whose
// images do not fit the staging list, or break the run order, writes each
// image straight to its slot from shared memory.
__global__ void __launch_bounds__(NT) k_halo_refresh_staged(Grid G, Arrays A, long long owned_off,
                                                           long long ghost_off, int positions_only,
                                                           const int* __restrict__ bowner,
                                                           const int* __restrict__ boff,
                                                           const int* __restrict__ bslot,
                                                           const int* __restrict__ bfirst,
                                                           const int* __restrict__ ghost_entry,
                                                           const int* __restrict__ tile_b0) {
    pdl_begin();
    extern __shared__ __align__(16) unsigned char s_rec[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ int s_seg[6 + kMaxFields];
    __shared__ int s_min[kMaxNeighbors];
    __shared__ int s_cnt[kMaxNeighbors];
    __shared__ int s_off[kMaxNeighbors + 1];
    __shared__ int s_bad;
    __shared__ unsigned short s_own[kStageCap];
    if (*G.status & kStatusGhostOverflow) return;
    const int ntiles = G.tile_start[G.P];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int narr = positions_only ? 3 : 6 + A.f.count;
    const unsigned bar = smem_u32(&s_bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned phase = 0;
    for (int g = blockIdx.x; g < ntiles; g += gridDim.x) {
        const int b0 = tile_b0[g], b1 = tile_b0[g + 1];
        if (b0 == b1) continue;   // uniform: no owner of this tile has an image
        const int4 td = G.tiles[g];
        const int s = td.x, begin = td.y, end = td.z;
        if (warp == 0) {
            // lane -> array: x, y, z, then vx, vy, vz and the fields
            const int k = lane < 6 ? lane : 13 + (lane - 6);
            int b = 0;
            const unsigned char* base = nullptr;
            if (lane < narr) {
                b = array_bytes(A, k);
                base = array_base(A, k);
            }
            const int size = b ? TILE * b + 32 : 0;
            const int soff = warp_inclusive_sum(size) - size;
            long long gl = 0, lo = 0, hi = 0;
            if (b) {
                gl = (owned_off + begin) * b;
                lo = gl & ~15LL;
                hi = ((owned_off + end) * b + 15) & ~15LL;
            }
            const unsigned bytes = static_cast<unsigned>(hi - lo);
            const unsigned total = __reduce_add_sync(0xffffffffu, bytes);
            if (lane == 0)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                             "r"(total) : "memory");
            __syncwarp();
            if (b) {
                bulk_load(smem_u32(s_rec + soff), base + lo, bytes, bar);
                s_seg[lane] = soff + static_cast<int>(gl - lo);
            }
        }
        if (threadIdx.x < kMaxNeighbors) {
            s_min[threadIdx.x] = INT_MAX;
            s_cnt[threadIdx.x] = 0;
        }
        if (threadIdx.x == 0) s_bad = 0;
        __syncthreads();
        // pass 1: each list's first slot and image count in this tile
        for (int b = b0 + threadIdx.x; b < b1; b += NT) {
            const int k0 = boff[b], k1 = boff[b + 1];
            for (int k = k0; k < k1; ++k) {
                const int slot = k == k0 ? bfirst[b] : bslot[k];
                const int n = ghost_entry[slot] - s * kMaxNeighbors;
                if (n < 0 || n >= kMaxNeighbors) {   // not this tile's sender: direct writes
                    s_bad = 1;
                    continue;
                }
                atomicMin(&s_min[n], slot);
                atomicAdd(&s_cnt[n], 1);
            }
        }
        __syncthreads();
        if (warp == 0) {
            const int c = lane < kMaxNeighbors ? s_cnt[lane] : 0;
            const int incl = warp_inclusive_sum(c);
            if (lane < kMaxNeighbors) s_off[lane] = incl - c;
            if (lane == 31) s_off[kMaxNeighbors] = incl;
        }
        __syncthreads();
        const int Q = s_off[kMaxNeighbors];
        const bool listed = Q <= kStageCap && !s_bad;
        // pass 2: every image's place in its list's run (a run that is not
        // one block of slots sends the tile to the direct writes)
        if (listed) {
            for (int b = b0 + threadIdx.x; b < b1; b += NT) {
                const int l = bowner[b] - begin;
                const int k0 = boff[b], k1 = boff[b + 1];
                for (int k = k0; k < k1; ++k) {
                    const int slot = k == k0 ? bfirst[b] : bslot[k];
                    const int n = ghost_entry[slot] - s * kMaxNeighbors;
                    const int rel = slot - s_min[n];
                    if (rel >= 0 && rel < s_cnt[n]) s_own[s_off[n] + rel] = static_cast<unsigned short>(l);
                    else s_bad = 1;
                }
            }
        }
        const bool lost = !bulk_wait_parity(bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(lost)) {
            if (lost) bulk_wait_parity(bar, phase ^ 1u);
            if (threadIdx.x == 0) atomicOr(G.status, kStatusCopyTimeout);
            return;
        }
        const double* shift = G.shift;
        auto write_image = [&](int l, long long gi, int entry) {
            const double* sh = shift + 3ll * entry;
            A.d[0][gi] = __dadd_rn(srd(s_rec, s_seg[0], l), sh[0]);
            A.d[1][gi] = __dadd_rn(srd(s_rec, s_seg[1], l), sh[1]);
            A.d[2][gi] = __dadd_rn(srd(s_rec, s_seg[2], l), sh[2]);
            A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
            if (!positions_only) {
                A.d[3][gi] = srd(s_rec, s_seg[3], l);
                A.d[4][gi] = srd(s_rec, s_seg[4], l);
                A.d[5][gi] = srd(s_rec, s_seg[5], l);
                fields_from_stage(A.f, s_rec, s_seg + 6, l, gi);
            }
        };
        if (listed && !s_bad) {
            for (int q = threadIdx.x; q < Q; q += NT) {
                int lo = 0, hi = kMaxNeighbors;   // largest n with s_off[n] <= q
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_off[mid] <= q) lo = mid;
                    else hi = mid;
                }
                const int n = lo;
                write_image(s_own[q], ghost_off + s_min[n] + (q - s_off[n]), s * kMaxNeighbors + n);
            }
        } else {
            for (int b = b0 + threadIdx.x; b < b1; b += NT) {
                const int l = bowner[b] - begin;
                const int k0 = boff[b], k1 = boff[b + 1];
                for (int k = k0; k < k1; ++k) {
                    const int slot = k == k0 ? bfirst[b] : bslot[k];
                    write_image(l, ghost_off + slot, ghost_entry[slot]);
                }
            }
        }
        __syncthreads();   // the stage and the lists are reused by the next tile
    }
}

// Tile descriptors {s, begin, end, first tile of s} of a layout given by its
// global counts, bases and tile starts (P + 1 entries each), the tiles
// strided over the threads of the grid.
__device__ __forceinline__ void fill_tiles_grid(int P, int tile, const int* n, const int* ob,
                                                const int* ts, int4* tiles) {
    const int total = ts[P];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = P;   // largest s with ts[s] <= g
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (ts[mid] <= g) lo = mid;
            else hi = mid;
        }
        const int begin = ob[lo] + (g - ts[lo]) * tile;
        const int end = min(begin + tile, ob[lo] + n[lo]);
        tiles[g] = make_int4(lo, begin, end, ts[lo]);
    }
}

// Counter bases of every tile of the layout (30 per tile, row stride 32), so
// that the move reads them with one load per tile; and the tile descriptors
// of the next layout and of its immigrant segments (imm_in: immigrants per
// subdomain, imm_base: where they start, imm_ts: their tile starts).
__global__ void __launch_bounds__(NT) k_tile_bases(Grid G, const int* pre, int stride,
                                                   const int* cbase_ret, int* tile_bases,
                                                   const int* imm_in, const int* imm_base,
                                                   const int* imm_ts, int4* imm_tiles) {
    pdl_begin();
    const int ntiles = G.tile_start[G.P];
    for (long long idx = blockIdx.x * static_cast<long long>(NT) + threadIdx.x;
         idx < static_cast<long long>(ntiles) * 32; idx += static_cast<long long>(gridDim.x) * NT) {
        const int g = static_cast<int>(idx >> 5), k = static_cast<int>(idx & 31);
        if (k < kStepCounters) tile_bases[idx] = tile_base(G, pre, stride, cbase_ret, g, G.tiles[g], k);
    }
    fill_tiles_grid(G.P, G.tile, G.n_next, G.obase_next, G.tile_start_next, G.tiles_next);
    fill_tiles_grid(G.P, G.tile, imm_in, imm_base, imm_ts, imm_tiles);
}

// The tile prefixes of the step's counters summed per subdomain, for a
// sharded step whose layout is planned on the host from the counts of every
// shard: out[0, P) retained particles, [P, 2P) boundary owners and [2P, 3P)
// their images (the retained parts), [3P, 3P + 26P) the retained part of
// every send list, and out[29P] the emigrants of this shard.
__global__ void __launch_bounds__(1024) k_step_export(Grid G, const int* pre, int stride, int* out) {
    pdl_begin();
    const int P = G.P;
    const int* ts = G.tile_start;
    auto tile_sum = [&](int k, int r) {
        return pre[k * stride + ts[r + 1]] - pre[k * stride + ts[r]];
    };
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
        out[t] = tile_sum(kStepStay, t);
        out[P + t] = tile_sum(kBoundaryCounter, t);
        out[2 * P + t] = tile_sum(kImageCounter, t);
    }
    for (int idx = threadIdx.x; idx < P * kMaxNeighbors; idx += blockDim.x) {
        const int r = idx / kMaxNeighbors, n = idx % kMaxNeighbors;
        const bool active = n < G.nn[r] && G.nbr[idx] >= 0;
        out[3 * P + idx] = active ? tile_sum(n, r) : 0;
    }
    if (threadIdx.x == 0) out[29 * P] = pre[kStepEmig * stride + ts[P]];
}

// F4 with the tile's records staged in shared memory (same output as
// k_step_move).  Dynamic shared memory: sum over the arrays of TILE x element
// bytes + 32.
//
// FULL: one pass over the whole record.  Otherwise the pass moves arrays
// [a0, a1) only (a record too wide for three staged tiles per SM is moved in
// several passes); every pass redoes the index work from the destinations
// and masks, and only the pass with index_outputs writes its results.
template <bool FULL, bool DIRECT_FORCES>
__global__ void __launch_bounds__(NT, 3) k_step_move_staged(
    Grid G, Arrays A, long long src_off, long long dst_off, long long ghost_off, const int* pre,
    int stride, const int* cbase_ret, const unsigned short* __restrict__ dest_in,
    const unsigned* __restrict__ mask_in, const int* __restrict__ tile_bases, int* emig_src,
    int* emig_dst, int* ghost_owner, int* ghost_entry, int* bowner, int* boff, int* bslot, int* bfirst, int a0,
    int a1, int index_outputs) {
    pdl_begin();
    extern __shared__ __align__(16) unsigned char s_rec[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ int s_seg[kStagedArrays];
    __shared__ int s_cnt[NW][32];
    __shared__ int s_base[32];
    __shared__ int s_off[kMaxNeighbors + 1];
    __shared__ unsigned short s_own[kStageCap];
    __shared__ int s_ni[TILE];
    const int g = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // destinations, masks (per tile slot) and the counter bases (per tile)
    // need only the tile index: they are read together with the descriptor
    const int4 td = G.tiles[g];
    const long long slot0 = static_cast<long long>(g) * TILE + warp * 32 * ITEMS + lane;
    unsigned short d16[ITEMS];
    unsigned mraw[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        d16[j] = dest_in[slot0 + j * 32];
        mraw[j] = mask_in[slot0 + j * 32];
    }
    const int base = threadIdx.x < kStepCounters ? tile_bases[static_cast<long long>(g) * 32 + threadIdx.x] : 0;
    if (g >= G.tile_start[G.P]) return;
    const int s = td.x, begin = td.y, end = td.z;
    const unsigned bar = smem_u32(&s_bar);
    const int wbegin = begin + warp * 32 * ITEMS;
    // the tile's records go out as soon as the descriptor is known
    if (warp == 0) {
        if (lane == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
        stage_issue(A, src_off, begin, end, s_rec, bar, s_seg, lane, a0, a1, DIRECT_FORCES);
    }
    // (slots past the tile's end hold stale values: masked here; the mask
    // is only meaningful for a stay)
    int dest[ITEMS];
    unsigned msk[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const bool in = wbegin + j * 32 + lane < end;
        dest[j] = in ? static_cast<int>(d16[j]) : -1;
        msk[j] = in ? mraw[j] : 0u;
    }
    const bool ghosts = !(*G.status & kStatusGhostOverflow);
    const int nn = G.nn[s];
    const unsigned lt = lanemask_lt();
    int acc = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (dest[j] != s) msk[j] = 0;
        count_group(msk[j], nn, lane, acc);
        const int stays = __popc(__ballot_sync(0xffffffffu, dest[j] == s));
        const int emigs = __popc(__ballot_sync(0xffffffffu, dest[j] >= 0 && dest[j] != s));
        if (lane == kStepStay) acc += stays;
        if (lane == kStepEmig) acc += emigs;
    }
    s_cnt[warp][lane] = acc;
    if (threadIdx.x < kStepCounters) s_base[threadIdx.x] = base;
    __syncthreads();
    // staging offsets of the lists: lane n sums its list over the warps, then
    // an exclusive scan over the lanes (every warp computes them; warp 0
    // keeps them for the ghost pass)
    int tot = 0;
    if (lane < nn)
        for (int w = 0; w < NW; ++w) tot += s_cnt[w][lane];
    const int sincl = warp_inclusive_sum(tot);
    const int Q = __shfl_sync(0xffffffffu, sincl, 31);
    if (warp == 0) {
        if (lane < nn) s_off[lane] = sincl - tot;
        if (lane == 31) s_off[nn] = sincl;
    }
    const bool staged = Q <= kStageCap;
    int run = 0, lrun = 0;
    if (lane < kStepCounters) {
        run = s_base[lane];
        if (lane < nn) lrun = sincl - tot;
        for (int w = 0; w < warp; ++w) {
            run += s_cnt[w][lane];
            lrun += s_cnt[w][lane];
        }
    }
    const int run0 = run;
    // the index work needs only destinations and masks, so it runs while the
    // record copies are still landing: new slots, emigrant list, boundary
    // owners and their image slots, and the ghost images staged by list
    int nis[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        const int l = i - begin;
        const bool stay = dest[j] == s;
        const bool emig = dest[j] >= 0 && !stay;
        const unsigned bs_ = __ballot_sync(0xffffffffu, stay);
        const unsigned be = __ballot_sync(0xffffffffu, emig);
        const int ni = __shfl_sync(0xffffffffu, run, kStepStay) + __popc(bs_ & lt);
        const int eb = __shfl_sync(0xffffffffu, run, kStepEmig) + __popc(be & lt);
        nis[j] = ni;
        if (stay) {
            s_ni[l] = ni;
        } else if (emig && index_outputs) {
            emig_src[eb] = i;
            emig_dst[eb] = dest[j];
        }
        const unsigned mj = ghosts ? msk[j] : 0u;
        const unsigned any = __ballot_sync(0xffffffffu, mj != 0);
        if (any) {
            const int b = __shfl_sync(0xffffffffu, run, kBoundaryCounter) + __popc(any & lt);
            const int pm = __popc(mj);
            const int incl = warp_inclusive_sum(pm);
            const int img = __shfl_sync(0xffffffffu, run, kImageCounter) + incl - pm;
            if (mj && index_outputs) {
                bowner[b] = ni;
                boff[b] = img;
            }
            int k = 0;
            const unsigned used = __reduce_or_sync(0xffffffffu, mj);
            for (unsigned rest = used; rest; rest &= rest - 1) {
                const int n = __ffs(rest) - 1;
                const unsigned hit = __ballot_sync(0xffffffffu, (mj >> n) & 1u);
                const int list_base = __shfl_sync(0xffffffffu, run, n);
                const int stage_base = __shfl_sync(0xffffffffu, lrun, n);
                if ((mj >> n) & 1u) {
                    const int rank = __popc(hit & lt);
                    if (index_outputs) {
                        bslot[img + k] = list_base + rank;
                        if (k == 0) bfirst[b] = list_base + rank;
                    }
                    ++k;
                    if (staged) s_own[stage_base + rank] = static_cast<unsigned short>(l);
                }
                if (lane == n) {
                    run += __popc(hit);
                    lrun += __popc(hit);
                }
            }
            const int group_images = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == kBoundaryCounter) run += __popc(any);
            if (lane == kImageCounter) run += group_images;
        }
        if (lane == kStepStay) run += __popc(bs_);
        if (lane == kStepEmig) run += __popc(be);
    }
    // forces of the stays read from HBM (not staged), in flight with the copies
    double fstay[ITEMS][3];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        fstay[j][0] = fstay[j][1] = fstay[j][2] = 0.0;
        if (DIRECT_FORCES && dest[j] == s) {
            const long long src = src_off + wbegin + j * 32 + lane;
            fstay[j][0] = ro(A.d[6] + src);
            fstay[j][1] = ro(A.d[7] + src);
            fstay[j][2] = ro(A.d[8] + src);
        }
    }
    // the records must have landed before anything reads them; after this
    // barrier every warp's staging is visible too
    const bool lost = !bulk_wait(bar);
    if (__syncthreads_or(lost)) {
        if (lost) bulk_wait(bar);   // copies still in flight get one more bounded wait
        if (threadIdx.x == 0) atomicOr(G.status, kStatusCopyTimeout);
        return;
    }
    int sg[13];
#pragma unroll
    for (int a = 0; a < 13; ++a) sg[a] = FULL ? s_seg[a] : 0;
    const int* fseg = s_seg + 13;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (dest[j] != s) continue;
        const int l = wbegin + j * 32 + lane - begin;
        if (FULL && DIRECT_FORCES) {
            move_from_stage_forces(G, A, s_rec, sg, fseg, l, dst_off + nis[j], fstay[j][0],
                                   fstay[j][1], fstay[j][2]);
        } else if (FULL) {
            move_from_stage(G, A, s_rec, sg, fseg, l, dst_off + nis[j]);
        } else {
            for (int c = a0; c < a1; ++c)
                move_array_from_stage(G, A, s_rec, s_seg[c - a0], c, l, dst_off + nis[j]);
        }
    }
    if (!ghosts) return;
    const double* shift = G.shift + static_cast<long long>(s) * kMaxNeighbors * 3;
    if (staged) {
        // list by list: consecutive threads write consecutive ghost slots
        for (int q = threadIdx.x; q < Q; q += NT) {
            int lo = 0, hi = nn;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (s_off[mid] <= q) lo = mid;
                else hi = mid;
            }
            const int n = lo;
            const int slot = s_base[n] + (q - s_off[n]);
            const int l = s_own[q];
            if (FULL) {
                ghost_from_stage(G, A, s_rec, sg, fseg, l, ghost_off + slot, shift + 3 * n);
            } else {
                for (int c = a0; c < a1; ++c)
                    ghost_array_from_stage(G, A, s_rec, s_seg[c - a0], c, l, ghost_off + slot,
                                           shift + 3 * n);
            }
            if (index_outputs) {
                ghost_owner[slot] = s_ni[l];
                ghost_entry[slot] = s * kMaxNeighbors + n;
            }
        }
        return;
    }
    // a tile with more images than the staging holds (a halo wider than
    // half a cell) writes them from the hitting lanes directly
    run = run0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int l = wbegin + j * 32 + lane - begin;
        const unsigned mj = msk[j];
        const unsigned used = __reduce_or_sync(0xffffffffu, mj);
        for (unsigned rest = used; rest; rest &= rest - 1) {
            const int n = __ffs(rest) - 1;
            const unsigned hit = __ballot_sync(0xffffffffu, (mj >> n) & 1u);
            const int list_base = __shfl_sync(0xffffffffu, run, n);
            if ((mj >> n) & 1u) {
                const int slot = list_base + __popc(hit & lt);
                if (FULL) {
                    ghost_from_stage(G, A, s_rec, sg, fseg, l, ghost_off + slot, shift + 3 * n);
                } else {
                    for (int c = a0; c < a1; ++c)
                        ghost_array_from_stage(G, A, s_rec, s_seg[c - a0], c, l, ghost_off + slot,
                                               shift + 3 * n);
                }
                if (index_outputs) {
                    ghost_owner[slot] = nis[j];
                    ghost_entry[slot] = s * kMaxNeighbors + n;
                }
            }
            if (lane == n) run += __popc(hit);
        }
    }
}

// Refresh along the existing plan (Host semantics, dsDecompX
// src/halo.cpp:256-289 + 687): positions (+ shift) and velocities and every
// registered field; forces of the ghosts become 0 again; mass, charge, type
// and id keep the values of the plan build.  positions_only moves x, y, z.
__global__ void __launch_bounds__(NT) k_halo_refresh(Grid G, Arrays A, long long owned_off,
                                                     long long ghost_off, int positions_only,
                                                     const int* info,
                                                     const int* __restrict__ ghost_owner,
                                                     const int* __restrict__ ghost_entry) {
    pdl_begin();
    if (*G.status & kStatusGhostOverflow) return;
    const int total = info[0];
    // four ghosts per thread and pass: their owner indices, then their
    // owners' positions, are all in flight before the first store (two per
    // thread at 40 registers ran slower: 0.155 against 0.148 ms)
    constexpr int U = 4;
    const int step = gridDim.x * NT;
    for (int s0 = blockIdx.x * NT + threadIdx.x; s0 < total; s0 += U * step) {
        int own[U], ent[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int slot = s0 + u * step;
            own[u] = slot < total ? ro(ghost_owner + slot) : 0;
            ent[u] = slot < total ? ro(ghost_entry + slot) : 0;
        }
        double p[U][3];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (s0 + u * step < total) {
                const long long src = owned_off + own[u];
                p[u][0] = A.d[0][src];
                p[u][1] = A.d[1][src];
                p[u][2] = A.d[2][src];
            }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int slot = s0 + u * step;
            if (slot >= total) continue;
            const long long src = owned_off + own[u];
            const double* sh = G.shift + 3ll * ent[u];
            const long long gi = ghost_off + slot;
            A.d[0][gi] = __dadd_rn(p[u][0], sh[0]);
            A.d[1][gi] = __dadd_rn(p[u][1], sh[1]);
            A.d[2][gi] = __dadd_rn(p[u][2], sh[2]);
            A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
            if (!positions_only) {
                A.d[3][gi] = A.d[3][src];
                A.d[4][gi] = A.d[4][src];
                A.d[5][gi] = A.d[5][src];
                copy_fields(A.f, src, gi);
            }
        }
    }
}

// Refresh along the plan, owner by owner: every boundary owner's record is
// read once (the reverse sum's CSR lists its images in neighbor order) and
// written to each of its images with that image's periodic shift.  The
// owners' reads then touch each sector of the owned arrays once, where a
// ghost-by-ghost gather reads a sector per image (the owners of one send
// list are sparse in the owned order).  Two owners per thread and pass keep
// their loads in flight together.
__global__ void __launch_bounds__(NT) k_halo_refresh_owners(Grid G, Arrays A, long long owned_off,
                                                            long long ghost_off, int positions_only,
                                                            const int* info,
                                                            const int* __restrict__ bowner,
                                                            const int* __restrict__ boff,
                                                            const int* __restrict__ bslot,
                                                            const int* __restrict__ bfirst,
                                                            const int* __restrict__ ghost_entry) {
    pdl_begin();
    if (*G.status & kStatusGhostOverflow) return;
    const int B = info[1];
    constexpr int U = 2;
    const int step = gridDim.x * NT;
    for (int b0 = blockIdx.x * NT + threadIdx.x; b0 < B; b0 += U * step) {
        long long src[U];
        int k0[U], k1[U], first[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int b = b0 + u * step;
            const bool in = b < B;
            src[u] = owned_off + (in ? ro(bowner + b) : 0);
            first[u] = in ? ro(bfirst + b) : 0;
            k0[u] = in ? ro(boff + b) : 0;
            k1[u] = in ? ro(boff + b + 1) : 0;
        }
        // the owner's record and its first image's list entry in one round trip
        double p[U][6];
        int entry[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (k0[u] >= k1[u]) continue;
            entry[u] = ro(ghost_entry + first[u]);
#pragma unroll
            for (int a = 0; a < 3; ++a) p[u][a] = ro(A.d[a] + src[u]);
            if (!positions_only)
#pragma unroll
                for (int a = 3; a < 6; ++a) p[u][a] = ro(A.d[a] + src[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            for (int k = k0[u]; k < k1[u]; ++k) {
                const int slot = k == k0[u] ? first[u] : ro(bslot + k);
                const double* sh = G.shift + 3ll * (k == k0[u] ? entry[u] : ro(ghost_entry + slot));
                const long long gi = ghost_off + slot;
                A.d[0][gi] = __dadd_rn(p[u][0], sh[0]);
                A.d[1][gi] = __dadd_rn(p[u][1], sh[1]);
                A.d[2][gi] = __dadd_rn(p[u][2], sh[2]);
                A.d[6][gi] = 0.0; A.d[7][gi] = 0.0; A.d[8][gi] = 0.0;
                if (!positions_only) {
                    A.d[3][gi] = p[u][3];
                    A.d[4][gi] = p[u][4];
                    A.d[5][gi] = p[u][5];
                    copy_fields(A.f, src[u], gi);
                }
            }
        }
    }
}

__global__ void __launch_bounds__(NT) k_forward_fields(Arrays A, long long owned_off,
                                                       long long ghost_off, FieldOps F,
                                                       const int* info,
                                                       const int* __restrict__ ghost_owner,
                                                       const unsigned* status) {
    pdl_begin();
    if (*status & kStatusGhostOverflow) return;
    const int total = info[0];
    for (int slot = blockIdx.x * NT + threadIdx.x; slot < total; slot += gridDim.x * NT) {
        const long long src = owned_off + ghost_owner[slot];
        const long long dst = ghost_off + slot;
        for (int t = 0; t < F.count; ++t) {
            const int f = F.index[t];
            const int b = A.f.bytes[f];
            unsigned char* base = A.f.base[f];
            if ((b & 7) == 0) {
                const unsigned long long* s = reinterpret_cast<const unsigned long long*>(base + src * b);
                unsigned long long* d = reinterpret_cast<unsigned long long*>(base + dst * b);
                for (int w = 0; w < (b >> 3); ++w) d[w] = s[w];
            } else {
                const unsigned* s = reinterpret_cast<const unsigned*>(base + src * b);
                unsigned* d = reinterpret_cast<unsigned*>(base + dst * b);
                for (int w = 0; w < (b >> 2); ++w) d[w] = s[w];
            }
        }
    }
}

// Owner-centric deterministic sum: owner += ghost images in the order the
// reference's Host reverse_exchange visits them (neighbor n ascending,
// dsDecompX src/halo.cpp:1507-1530).  No atomics.  The first image's slot is
// read beside the owner index (bfirst), so the owner's force and its first
// image arrive in one round trip; further images (edges, corners) follow
// from the CSR.
__global__ void __launch_bounds__(NT) k_reverse_sum3(const int* info, const int* __restrict__ bowner,
                                                     const int* __restrict__ boff,
                                                     const int* __restrict__ bslot,
                                                     const int* __restrict__ bfirst,
                                                     double* __restrict__ ox,
                                                     double* __restrict__ oy,
                                                     double* __restrict__ oz,
                                                     const double* __restrict__ gx,
                                                     const double* __restrict__ gy,
                                                     const double* __restrict__ gz,
                                                     const unsigned* status, int b_first,
                                                     int b_end) {
    pdl_begin();
    if (*status & kStatusGhostOverflow) return;
    const int B = b_end >= 0 ? b_end : info[1];
    for (int b = b_first + blockIdx.x * NT + threadIdx.x; b < B; b += gridDim.x * NT) {
        const int i = bowner[b];
        const int s0 = bfirst[b];
        const int k0 = boff[b], k1 = boff[b + 1];
        double fx = ox[i], fy = oy[i], fz = oz[i];
        fx = __dadd_rn(fx, gx[s0]);
        fy = __dadd_rn(fy, gy[s0]);
        fz = __dadd_rn(fz, gz[s0]);
        for (int k = k0 + 1; k < k1; ++k) {
            const int slot = bslot[k];
            fx = __dadd_rn(fx, gx[slot]);
            fy = __dadd_rn(fy, gy[slot]);
            fz = __dadd_rn(fz, gz[slot]);
        }
        ox[i] = fx;
        oy[i] = fy;
        oz[i] = fz;
    }
}

// std::min / std::max / += / = exactly as reduce_field_values applies them
// (dsDecompX src/halo.cpp:1351-1372).
template <class T>
__device__ __forceinline__ T reduce_one(T d, T v, int op) {
    switch (op) {
    case 0: return static_cast<T>(d + v);
    case 1: return v < d ? v : d;
    case 2: return d < v ? v : d;
    default: return v;
    }
}
template <>
__device__ __forceinline__ double reduce_one<double>(double d, double v, int op) {
    switch (op) {
    case 0: return __dadd_rn(d, v);
    case 1: return v < d ? v : d;
    case 2: return d < v ? v : d;
    default: return v;
    }
}
template <>
__device__ __forceinline__ float reduce_one<float>(float d, float v, int op) {
    switch (op) {
    case 0: return __fadd_rn(d, v);
    case 1: return v < d ? v : d;
    case 2: return d < v ? v : d;
    default: return v;
    }
}
template <>
__device__ __forceinline__ int reduce_one<int>(int d, int v, int op) {
    switch (op) {
    case 0: return static_cast<int>(static_cast<unsigned>(d) + static_cast<unsigned>(v));
    case 1: return v < d ? v : d;
    case 2: return d < v ? v : d;
    default: return v;
    }
}
template <>
__device__ __forceinline__ long long reduce_one<long long>(long long d, long long v, int op) {
    switch (op) {
    case 0: return static_cast<long long>(static_cast<unsigned long long>(d) + static_cast<unsigned long long>(v));
    case 1: return v < d ? v : d;
    case 2: return d < v ? v : d;
    default: return v;
    }
}

template <class T>
__device__ __forceinline__ void reduce_images(unsigned char* base, int comps, int op, long long owner,
                                              long long ghost_off, const int* bslot, int k0, int k1) {
    T* o = reinterpret_cast<T*>(base) + owner * comps;
    for (int c = 0; c < comps; ++c) {
        T acc = o[c];
        for (int k = k0; k < k1; ++k)
            acc = reduce_one<T>(acc, reinterpret_cast<const T*>(base)[(ghost_off + bslot[k]) * comps + c], op);
        o[c] = acc;
    }
}

__global__ void __launch_bounds__(NT) k_reverse_fields(Arrays A, long long owned_off,
                                                       long long ghost_off, FieldOps F,
                                                       const int* info,
                                                       const int* __restrict__ bowner,
                                                       const int* __restrict__ boff,
                                                       const int* __restrict__ bslot,
                                                       const unsigned* status) {
    pdl_begin();
    if (*status & kStatusGhostOverflow) return;
    const int B = info[1];
    for (int b = blockIdx.x * NT + threadIdx.x; b < B; b += gridDim.x * NT) {
        const long long owner = owned_off + bowner[b];
        const int k0 = boff[b], k1 = boff[b + 1];
        for (int t = 0; t < F.count; ++t) {
            unsigned char* base = A.f.base[F.index[t]];
            const int comps = F.components[t];
            const int op = F.op[t];
            switch (F.type[t]) {
            case 0: reduce_images<int>(base, comps, op, owner, ghost_off, bslot, k0, k1); break;
            case 1: reduce_images<long long>(base, comps, op, owner, ghost_off, bslot, k0, k1); break;
            case 2: reduce_images<unsigned>(base, comps, op, owner, ghost_off, bslot, k0, k1); break;
            case 3: reduce_images<unsigned long long>(base, comps, op, owner, ghost_off, bslot, k0, k1); break;
            case 4: reduce_images<float>(base, comps, op, owner, ghost_off, bslot, k0, k1); break;
            default: reduce_images<double>(base, comps, op, owner, ghost_off, bslot, k0, k1); break;
            }
        }
    }
}

// ---------------------------------------------------------------- rebalance

// Dynamic cut planes (dsDecompX src/runtime.cpp:345-447) evaluated by one
// warp, every value with the reference's operations in the reference's
// order, on the device so that it can sit inside a captured step.
//
// The serial sums run in one loop over the subdomains in index order, each
// on its own lane: lane 31 the total and the maximum, lanes 0..30 one
// (axis, slab) sum each (more slabs take further passes).  Every lane adds
// its terms in the order the reference's single loop does, so each sum has
// the reference's bits; the lanes only run side by side.
__global__ void __launch_bounds__(32) k_rebalance(Grid G, const double* work_in,
                                                  RebalanceParams p, long long* call_counter,
                                                  double* result) {
    pdl_begin();
    __shared__ double s_work[kMaxRanks];
    __shared__ int s_coord[kMaxRanks];         // packed grid coordinates, staged once
    __shared__ double s_old[kMaxRanks + 4];    // current cuts, axis a at G.cut_offset[a]
    __shared__ double s_next[kMaxRanks + 4];   // next cuts, same places
    __shared__ double s_slab[kMaxRanks + 3];   // slab work, axis a at slab_off[a]
    __shared__ double s_total, s_max;
    __shared__ int s_go, s_bad;
    const int lane = threadIdx.x;
    if (blockIdx.x != 0) return;
    if (p.clear_status && lane == 0) *G.status = 0u;
    for (int k = lane; k < p.nzero; k += 32) p.zero[k] = 0;
    const int P = G.P;
    const int ncuts = G.cut_offset[2] + G.dims[2] + 1;
    // everything the warp reads, in one round trip
    for (int s = lane; s < P; s += 32) {
        s_work[s] = work_in ? work_in[s] : static_cast<double>(G.n[s]);
        s_coord[s] = G.coord[s];
    }
    for (int k = lane; k < ncuts; k += 32) {
        const double c = G.cuts[k];
        s_old[k] = c;
        s_next[k] = c;
    }
    if (lane == 0) {
        result[0] = 0.0;
        result[1] = 0.0;
        result[2] = 1.0;
        int go = 1;
        if (p.automatic) {
            const long long calls = ++(*call_counter);
            if (p.interval == 0 || calls % p.interval != 0) go = 0;
        }
        s_go = go;
        s_bad = 0;
    }
    __syncwarp();
    if (!s_go) return;
    const int slab_off[3] = {0, G.dims[0], G.dims[0] + G.dims[1]};
    const int nslabs = G.dims[0] + G.dims[1] + G.dims[2];
    for (int first = 0; first == 0 || first < nslabs; first += 31) {
        // this lane's sum: the total (lane 31, first pass) or slab `pair`
        const int pair = first + lane;
        const bool total_lane = lane == 31 && first == 0;
        const bool slab_lane = lane < 31 && pair < nslabs;
        int slab = 0, shift = 20;
        if (slab_lane) {
            const int axis = pair < slab_off[1] ? 0 : pair < slab_off[2] ? 1 : 2;
            slab = pair - slab_off[axis];
            shift = axis == 0 ? 20 : axis == 1 ? 10 : 0;
        }
        double acc = 0.0, maximum = 0.0;
        for (int s = 0; s < P; ++s) {
            const double w = s_work[s];
            if (total_lane) {
                acc = __dadd_rn(acc, w);
                if (maximum < w) maximum = w;
            } else if (slab_lane && ((s_coord[s] >> shift) & 1023) == slab) {
                acc = __dadd_rn(acc, w);
            }
        }
        if (total_lane) {
            s_total = acc;
            s_max = maximum;
        } else if (slab_lane) {
            s_slab[pair] = acc;
        }
    }
    __syncwarp();
    if (lane == 0) {
        const double total = s_total, maximum = s_max;
        result[0] = 1.0;
        int go = 1;
        if (total <= 0.0 || P <= 1) {
            go = 0;
        } else {
            const double imbalance = __ddiv_rn(maximum, __ddiv_rn(total, static_cast<double>(P)));
            result[2] = imbalance;
            if (!p.force && imbalance < p.threshold) go = 0;
        }
        s_go = go;
    }
    __syncwarp();
    if (!s_go) return;
    const double total = s_total;
    for (int a = 0; a < 3; ++a) {
        const int slabs = G.dims[a];
        if (slabs <= 1) continue;
        const double* old = s_old + G.cut_offset[a];
        const double* sw = s_slab + slab_off[a];
        double* next = s_next + G.cut_offset[a];
        const double target = __ddiv_rn(total, static_cast<double>(slabs));
        if (lane == 0) {
            next[0] = G.lower[a];
            next[slabs] = G.upper[a];
        }
        for (int b = 1 + lane; b < slabs; b += 32) {
            const double desired = __dmul_rn(target, static_cast<double>(b));
            double cumulative = 0.0;
            int slab = 0;
            while (slab < slabs - 1 && __dadd_rn(cumulative, sw[slab]) < desired)
                cumulative = __dadd_rn(cumulative, sw[slab++]);
            const double weight = sw[slab];
            double fraction = 0.5;
            if (weight > 0.0) {
                const double v = __ddiv_rn(__dsub_rn(desired, cumulative), weight);
                fraction = v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v);
            }
            const double proposed =
                __dadd_rn(old[slab], __dmul_rn(fraction, __dsub_rn(old[slab + 1], old[slab])));
            const double o = old[b];
            next[b] = __dadd_rn(o, __dmul_rn(p.relaxation, __dsub_rn(proposed, o)));
        }
    }
    __syncwarp();
    if (lane < 3 && G.dims[lane] > 1) {
        const int a = lane, slabs = G.dims[a];
        double* next = s_next + G.cut_offset[a];
        const double extent = __dsub_rn(G.upper[a], G.lower[a]);
        const double uniform = __ddiv_rn(extent, static_cast<double>(slabs));
        double bound = __dmul_rn(uniform, p.minimum_fraction);
        if (bound < p.halo_width) bound = p.halo_width;
        const double minimum_width = bound < uniform ? bound : uniform;
        for (int i = 1; i < slabs; ++i) {
            const double floor_value = __dadd_rn(next[i - 1], minimum_width);
            if (next[i] < floor_value) next[i] = floor_value;
        }
        for (int i = slabs - 1; i > 0; --i) {
            const double ceiling = __dsub_rn(next[i + 1], minimum_width);
            if (ceiling < next[i]) next[i] = ceiling;
        }
    }
    __syncwarp();
    bool moved = false;
    for (int k = lane; k < ncuts; k += 32)
        if (fabs(__dsub_rn(s_next[k], s_old[k])) > 1.0e-12) moved = true;
    if (!__any_sync(0xffffffffu, moved)) return;
    // Decomposition::set_axis_cuts validation (dsDecompX src/decomp.cpp:146-163)
    if (lane < 3) {
        const int a = lane, slabs = G.dims[a];
        const double* next = s_next + G.cut_offset[a];
        bool valid = next[0] == G.lower[a] && next[slabs] == G.upper[a];
        for (int i = 0; i < slabs; ++i) valid = valid && next[i] < next[i + 1];
        if (!valid) atomicOr(&s_bad, 1);
    }
    __syncwarp();
    if (s_bad) {
        if (lane == 0) atomicOr(G.status, kStatusCutsInvalid);
        return;
    }
    for (int k = lane; k < ncuts; k += 32) G.cuts[k] = s_next[k];
    if (lane == 0) result[1] = 1.0;
}


// upper_bound(cuts, cuts + dims + 1, v) - cuts - 1 clamped to [0, dims - 1],
// as a count of the cuts that v is not below: the cuts increase strictly, so
// !(v < cut) holds on a prefix of them (on all of them for a NaN, where the
// bisection of axis_coordinate also ends past the last cut).
// Axes of at most kCountedCells cells; the loop is unrolled and predicated
// (no branches).
constexpr int kCountedCells = 8;
__device__ __forceinline__ int axis_coordinate_count(const double* cuts, int dims, double v) {
    int c = -1;
#pragma unroll
    for (int k = 0; k <= kCountedCells; ++k)
        if (k <= dims) c += !(v < cuts[k]);
    c = c > dims - 1 ? dims - 1 : c;
    return c < 0 ? 0 : c;
}

// Decomposition::owner_rank (dsDecompX src/migration.cpp:74-98) of arbitrary
// positions: one periodic wrap, then the cut search, with the cut planes in
// shared memory.  The search goes through a coarse table: each axis is split
// into kGuessBins equal bins, and the table holds the cell of every bin's
// lower edge (found with the exact rule).  A position starts at its bin's cell and steps
// forward while it is not below the next cut, backward while it is below its
// cell's own cut: the cuts increase strictly, so the steps end at the cell
// the full search returns (clamped at both ends; a NaN, below no cut, ends
// in the last cell as there), whatever the bin arithmetic rounded to.
// Usually no step or one step is taken, against one comparison per cut.
constexpr int kGuessBins = 64;

struct CellGuess {
    double lower[3], inv[3];   // kGuessBins / extent per axis
};

__device__ __forceinline__ CellGuess cell_guess(const Grid& G) {
    CellGuess g;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        g.lower[a] = G.lower[a];
        g.inv[a] = static_cast<double>(kGuessBins) / G.extent[a];
    }
    return g;
}

// s_bins[a * kGuessBins + b]: the cell of bin b's lower edge on axis a
// (every thread of the CTA takes part; ends with a barrier).
__device__ __forceinline__ void stage_bins(const Grid& G, const double* s_cuts,
                                           unsigned short* s_bins) {
    for (int k = threadIdx.x; k < 3 * kGuessBins; k += blockDim.x) {
        const int a = k / kGuessBins, b = k % kGuessBins;
        const double edge = G.lower[a] + G.extent[a] * (static_cast<double>(b) / kGuessBins);
        const double* cuts = s_cuts + G.cut_offset[a];
        s_bins[k] = static_cast<unsigned short>(
            G.dims[a] <= kCountedCells ? axis_coordinate_count(cuts, G.dims[a], edge)
                                       : axis_coordinate(cuts, G.dims[a], edge));
    }
    __syncthreads();
}

__device__ __forceinline__ int owner_of_binned(const Grid& G, const CellGuess& g,
                                               const double* s_cuts,
                                               const unsigned short* s_bins, double px, double py,
                                               double pz) {
    const double p[3] = {px, py, pz};
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double v = wrap_if(G, a, p[a]);
        const double* cuts = s_cuts + G.cut_offset[a];
        const int dims = G.dims[a];
        // the bin, rounded to nearest by the 1.5 x 2^52 shift (its low word
        // is the integer; any value, NaN's included, is clamped, and a guess
        // one bin off is stepped away like any other)
        int b = __double2loint(__fma_rn(v - g.lower[a], g.inv[a], 6755399441055744.0));
        b = b < 0 ? 0 : (b > kGuessBins - 1 ? kGuessBins - 1 : b);
        int k = s_bins[a * kGuessBins + b];
        // one step either way without a branch; a position two or more
        // cells from the guess (cuts closer than a bin) keeps stepping
        const bool up = k < dims - 1 && !(v < cuts[k + 1]);
        const bool down = k > 0 && v < cuts[k];
        k += up ? 1 : 0;
        k -= down ? 1 : 0;
        if ((up && k < dims - 1 && !(v < cuts[k + 1])) || (down && k > 0 && v < cuts[k])) {
            while (k < dims - 1 && !(v < cuts[k + 1])) ++k;
            while (k > 0 && v < cuts[k]) --k;
        }
        c[a] = k;
    }
    return (c[0] * G.dims[1] + c[1]) * G.dims[2] + c[2];
}

__device__ __forceinline__ void stage_cuts(const Grid& G, double* s_cuts) {
    const int total = G.dims[0] + G.dims[1] + G.dims[2] + 3;
    for (int k = threadIdx.x; k < total; k += blockDim.x) s_cuts[k] = G.cuts[k];
    __syncthreads();
}

// One position per thread and pass, the next pass's position loaded before
// this one is searched (software pipelining: the loads stay in flight while
// the search runs).
__global__ void __launch_bounds__(NT) k_owner_rank(Grid G, const double* __restrict__ x,
                                                   const double* __restrict__ y,
                                                   const double* __restrict__ z, long long n,
                                                   int* out) {
    pdl_begin();
    __shared__ double s_cuts[kMaxRanks + 16];   // cut_offset[a] + kCountedCells <= 1036
    __shared__ unsigned short s_bins[3 * kGuessBins];
    stage_cuts(G, s_cuts);
    stage_bins(G, s_cuts, s_bins);
    const CellGuess guess = cell_guess(G);
    const long long step = static_cast<long long>(gridDim.x) * NT;
    long long i = blockIdx.x * static_cast<long long>(NT) + threadIdx.x;
    double px = 0.0, py = 0.0, pz = 0.0;
    if (i < n) {
        px = ro(x + i);
        py = ro(y + i);
        pz = ro(z + i);
    }
    for (; i < n; i += step) {
        const long long j = i + step;
        double qx = 0.0, qy = 0.0, qz = 0.0;
        if (j < n) {
            qx = ro(x + j);
            qy = ro(y + j);
            qz = ro(z + j);
        }
        out[i] = owner_of_binned(G, guess, s_cuts, s_bins, px, py, pz);
        px = qx;
        py = qy;
        pz = qz;
    }
}

// Decomp::has_out_of_domain_particles (dsDecompX src/runtime.cpp:828-840) for
// every subdomain at once: flags[s] = 1 if an owned particle of s belongs to
// another subdomain.
//
// Each warp takes chunks of 128 consecutive owned particles (four
// coalesced rows of 32, loaded together).  The warp finds the chunk's
// subdomain once (the layout's bases in shared memory) and its cell planes
// once; a position inside its subdomain's own planes is owned there (the wrap
// leaves a position inside the box as it is, -0 aside, which lies in the same
// cell), only the others are searched.  A chunk that runs past the end of
// its subdomain (rare: subdomains hold thousands of particles) finds the
// later particles' subdomains lane by lane.  One flag atomic per chunk for
// the chunk's own subdomain.
__device__ __forceinline__ int subdomain_of_index(const int* s_ob, int lo, int hi, int i) {
    while (hi - lo > 1) {   // largest s in [lo, hi) with s_ob[s] <= i
        const int mid = (lo + hi) >> 1;
        if (s_ob[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool inside_planes(const Grid& G, const double* s_cuts,
                                              const int* s_coord, int s, double px, double py,
                                              double pz) {
    const int packed = s_coord[s];
    const int c[3] = {packed >> 20, (packed >> 10) & 1023, packed & 1023};
    const double p[3] = {px, py, pz};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double* cuts = s_cuts + G.cut_offset[a] + c[a];
        inside = inside && cuts[0] <= p[a] && p[a] < cuts[1];
    }
    return inside;
}

__global__ void __launch_bounds__(NT, 4) k_out_of_domain(Grid G, const double* __restrict__ x,
                                                      const double* __restrict__ y,
                                                      const double* __restrict__ z, int* flags) {
    pdl_begin();
    __shared__ double s_cuts[kMaxRanks + 16];   // cut_offset[a] + kCountedCells <= 1036
    __shared__ unsigned short s_bins[3 * kGuessBins];
    __shared__ int s_ob[kMaxRanks + 1];
    __shared__ int s_coord[kMaxRanks];
    const int P = G.P;
    for (int k = threadIdx.x; k <= P; k += blockDim.x) {
        s_ob[k] = G.obase[k];
        if (k < P) s_coord[k] = G.coord[k];
    }
    stage_cuts(G, s_cuts);
    stage_bins(G, s_cuts, s_bins);
    const CellGuess guess = cell_guess(G);
    const int n = s_ob[P];
    const int lane = threadIdx.x & 31;
    constexpr int U = 4, CHUNK = 32 * U;
    const int warps = gridDim.x * NW;
    const long long nchunks = (static_cast<long long>(n) + CHUNK - 1) / CHUNK;
    for (long long ch = static_cast<long long>(blockIdx.x) * NW + (threadIdx.x >> 5); ch < nchunks;
         ch += warps) {
        const int base = static_cast<int>(ch * CHUNK);
        const int s0 = subdomain_of_index(s_ob, 0, P, base);   // the same on every lane
        const int end = s_ob[s0 + 1];
        double px[U], py[U], pz[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + u * 32 + lane;
            if (i < n) {
                px[u] = ro(x + i);
                py[u] = ro(y + i);
                pz[u] = ro(z + i);
            }
        }
        bool leaves = false;   // a particle of s0 belongs elsewhere
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + u * 32 + lane;
            if (i >= n) continue;
            const int s = i < end ? s0 : subdomain_of_index(s_ob, s0 + 1, P, i);
            if (inside_planes(G, s_cuts, s_coord, s, px[u], py[u], pz[u])) continue;
            if (owner_of_binned(G, guess, s_cuts, s_bins, px[u], py[u], pz[u]) == s) continue;
            if (s == s0) leaves = true;
            else atomicOr(&flags[s], 1);
        }
        if (__any_sync(0xffffffffu, leaves) && lane == 0) atomicOr(&flags[s0], 1);
    }
}

// Emigrants of the last migration counted per (destination, source):
// pairs[t * P + q].  The source of emigrant e is the subdomain of the old
// layout that held index emig_src[e] (obase_old: the old layout's P + 1
// offsets; the largest q with obase_old[q] <= i, so empty subdomains are
// stepped over).  E = info[0].
__global__ void __launch_bounds__(NT) k_pair_counts(int P, const int* __restrict__ info,
                                                    const int* __restrict__ emig_src,
                                                    const int* __restrict__ emig_dst,
                                                    const int* __restrict__ obase_old, int* pairs) {
    pdl_begin();
    const int E = info[0];
    const int lane = threadIdx.x & 31;
    // whole warps walk the list; lanes with the same (destination, source)
    // add once per warp (consecutive emigrants mostly share both)
    for (int base = blockIdx.x * NT + (threadIdx.x & ~31); base < E; base += gridDim.x * NT) {
        const int e = base + lane;
        int key = -1;
        if (e < E) {
            const int i = emig_src[e];
            int lo = 0, hi = P;   // obase_old[lo] <= i < obase_old[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (obase_old[mid] <= i) lo = mid;
                else hi = mid;
            }
            key = emig_dst[e] * P + lo;
        }
        const unsigned same = __match_any_sync(0xffffffffu, key);
        if (key >= 0 && lane == __ffs(same) - 1) atomicAdd(&pairs[key], __popc(same));
    }
}

// Bytes [0, n) of src to dst by the threads of one CTA, in words of W bytes
// between a byte-wise head (up to dst's W alignment) and tail; src and dst
// have the same address modulo W.
template <typename Word>
__device__ __forceinline__ void copy_words(const unsigned char* __restrict__ src,
                                           unsigned char* __restrict__ dst, long long n) {
    constexpr int W = sizeof(Word);
    long long head = static_cast<long long>((W - (reinterpret_cast<uintptr_t>(dst) & (W - 1))) & (W - 1));
    if (head > n) head = n;
    for (long long t = threadIdx.x; t < head; t += blockDim.x) dst[t] = src[t];
    const long long words = (n - head) / W;
    const Word* s = reinterpret_cast<const Word*>(src + head);
    Word* d = reinterpret_cast<Word*>(dst + head);
    // four loads in flight per thread before their stores
    constexpr int U = 4;
    for (long long t = threadIdx.x; t < words; t += U * blockDim.x) {
        Word v[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (t + u * blockDim.x < words) v[u] = s[t + u * blockDim.x];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (t + u * blockDim.x < words) d[t + u * blockDim.x] = v[u];
    }
    for (long long t = head + words * W + threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
}

// Device-to-device copies, one piece per CTA at a time (pieces of at most
// kCopyPiece bytes, so that one long copy spreads over many CTAs): 16-byte
// words when source and destination agree modulo 16, else 8, 4 or 1.
__global__ void __launch_bounds__(NT) k_copy_pieces(const CopyPiece* __restrict__ pieces,
                                                    long long n) {
    pdl_begin();
    for (long long j = blockIdx.x; j < n; j += gridDim.x) {
        const CopyPiece c = pieces[j];
        const uintptr_t mis = reinterpret_cast<uintptr_t>(c.src) ^ reinterpret_cast<uintptr_t>(c.dst);
        if (!(mis & 15)) copy_words<uint4>(c.src, c.dst, c.bytes);
        else if (!(mis & 7)) copy_words<unsigned long long>(c.src, c.dst, c.bytes);
        else if (!(mis & 3)) copy_words<unsigned>(c.src, c.dst, c.bytes);
        else copy_words<unsigned char>(c.src, c.dst, c.bytes);
    }
}

// 1-rank migrate of the drop-in: every particle stays and keeps its slot; its
// position is replaced by the once-wrapped value (dsDecompX
// src/migration.cpp:106-116).  Only changed values are written back.
__global__ void __launch_bounds__(NT) k_wrap_inplace(double* x, double* y, double* z, long long n,
                                                     double3 lower, double3 extent, int3 periodic) {
    pdl_begin();
    for (long long i = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * NT) {
        // all three reads go out before any compare
        const double vx = x[i], vy = y[i], vz = z[i];
        if (periodic.x) {
            const double w = wrap_axis(vx, lower.x, extent.x);
            if (__double_as_longlong(w) != __double_as_longlong(vx)) x[i] = w;
        }
        if (periodic.y) {
            const double w = wrap_axis(vy, lower.y, extent.y);
            if (__double_as_longlong(w) != __double_as_longlong(vy)) y[i] = w;
        }
        if (periodic.z) {
            const double w = wrap_axis(vz, lower.z, extent.z);
            if (__double_as_longlong(w) != __double_as_longlong(vz)) z[i] = w;
        }
    }
}

int g_sm_count = 0;

int sm_count() {
    if (!g_sm_count) {
        int device = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, device);
        if (g_sm_count <= 0) g_sm_count = 148;
    }
    return g_sm_count;
}

// Every kernel launch of the library: programmatic stream serialisation lets
// the kernel's CTAs become resident (and then wait, pdl_begin) while the
// previous kernel on the stream drains, inside captured graphs too; errors
// surface through cudaGetLastError like those of triple-chevron launches.
template <class... Params, class... Args>
void pdl_launch(void (*kernel)(Params...), int grid, int block, std::size_t smem, cudaStream_t s,
                Args&&... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t config = {};
    config.gridDim = dim3(static_cast<unsigned>(grid));
    config.blockDim = dim3(static_cast<unsigned>(block));
    config.dynamicSmemBytes = smem;
    config.stream = s;
    config.attrs = attr;
    config.numAttrs = 1;
    (void)cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

int stream_grid(long long items) {
    const long long want = (items + NT - 1) / NT;
    const long long cap = static_cast<long long>(sm_count()) * 8;
    long long g = want < cap ? want : cap;
    return static_cast<int>(g < 1 ? 1 : g);
}

// Grid of a grid-stride kernel of NT threads: the CTAs that fit on the GPU at
// once (one wave, from the kernel's own occupancy), fewer for small work.
int resident_grid(const void* kernel, long long items) {
    static std::mutex lock;
    static std::vector<std::pair<const void*, int>> cache;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> hold(lock);
        for (const auto& k : cache)
            if (k.first == kernel) per_sm = k.second;
        if (!per_sm) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT, 0) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
            cache.emplace_back(kernel, per_sm);
        }
    }
    const long long want = (items + NT - 1) / NT;
    const long long cap = static_cast<long long>(sm_count()) * per_sm;
    const long long g = want < cap ? want : cap;
    return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace

void launch_layout(const Grid& G, const int* n, int* obase, int* tile_start, int4* tiles,
                   cudaStream_t s) {
    pdl_launch(k_layout, 1, 1024, 0, s, G.P, G.tile, n, obase, tile_start, tiles);
}

// Runs launch(Gs, grid) once over all tiles, or, in plain mode, once per
// subdomain with the tile window of that subdomain.
template <class F>
void per_subdomain(const Grid& G, const PlainLaunch* plain, F&& launch) {
    if (!plain) {
        launch(G, G.max_tiles);
        return;
    }
    for (int r = 0; r < G.P; ++r) {
        const int t0 = plain->tile_start[r], t1 = plain->tile_start[r + 1];
        if (t1 <= t0) continue;
        Grid Gs = G;
        Gs.tile_first = t0;
        Gs.tile_end = t1;
        launch(Gs, t1 - t0);
    }
}

void launch_migrate(const Grid& G, const Arrays& A, long long src_off, long long dst_off,
                    const Scratch& S, cudaStream_t s, const PlainLaunch* plain) {
    cudaMemsetAsync(S.imm_total, 0, sizeof(int) * G.P, s);
    per_subdomain(G, plain, [&](const Grid& Gs, int grid) {
        pdl_launch(k_mig_classify, grid, NT, 0, s, Gs, A.d[0] + src_off, A.d[1] + src_off,
                                           A.d[2] + src_off, S.cnt, S.stride, S.imm_total);
    });
    if (S.marks) S.marks->mark(s, "mig_classify");
    pdl_launch(k_scan_counters, 2, 1024, 0, s, S.cnt, S.pre, S.stride, G.tile_start + G.P);
    if (S.marks) S.marks->mark(s, "mig_scan");
    pdl_launch(k_mig_layout, 1, 1024, 0, s, G, S.pre, S.stride, S.imm_total, S.imm_base, S.emig_info,
                                     S.mig_results);
    if (S.marks) S.marks->mark(s, "mig_layout");
    per_subdomain(G, plain, [&](const Grid& Gs, int grid) {
        pdl_launch(k_mig_move, grid, NT, 0, s, Gs, A, src_off, dst_off, S.pre, S.stride, S.emig_src,
                                       S.emig_dst);
    });
    if (S.marks) S.marks->mark(s, "mig_move");
    const int chunk_grid = S.max_chunks < sm_count() * 4 ? S.max_chunks : sm_count() * 4;
    const size_t smem = sizeof(int) * NW * G.P;
    pdl_launch(k_emig_hist, chunk_grid > 0 ? chunk_grid : 1, NT, smem, s, G.P, S.emig_info, S.emig_dst,
                                                                  S.emig_hist);
    if (S.marks) S.marks->mark(s, "emig_hist");
    pdl_launch(k_emig_colscan, G.P, NT, 0, s, G.P, S.emig_info, S.emig_hist, S.imm_total, G.status);
    if (S.marks) S.marks->mark(s, "emig_colscan");
    pdl_launch(k_emig_place, chunk_grid > 0 ? chunk_grid : 1, NT, smem, s,
        G, A, src_off, dst_off, S.emig_info, S.emig_src, S.emig_dst, S.emig_hist, S.imm_base,
        nullptr);
    if (S.marks) S.marks->mark(s, "emig_place");
}

// Shared memory the staged move needs for one tile of arrays [a0, a1).
int staged_range_bytes(const Arrays& A, int a0, int a1) {
    int bytes = 0;
    for (int k = a0; k < a1; ++k) bytes += TILE * (k < 11 ? 8 : k < 13 ? 4 : A.f.bytes[k - 13]) + 32;
    return bytes;
}

int staged_bytes(const Arrays& A) { return staged_range_bytes(A, 0, 13 + A.f.count); }

// Shared memory of the three force arrays of one staged tile.
constexpr int kForceStageBytes = 3 * (TILE * 8 + 32);

void launch_halo_build(const Grid& G, const Arrays& A, long long owned_off, long long ghost_off,
                       const Scratch& S, cudaStream_t s, const PlainLaunch* plain) {
    per_subdomain(G, plain, [&](const Grid& Gs, int grid) {
        pdl_launch(k_halo_classify, grid, NT, 0, s, Gs, G.tiles, G.tile_start + G.P, A.d[0] + owned_off,
                                            A.d[1] + owned_off, A.d[2] + owned_off, S.mask,
                                            S.cnt, S.stride);
    });
    if (S.marks) S.marks->mark(s, "halo_classify");
    pdl_launch(k_scan_counters, kHaloCounters, 1024, 0, s, S.cnt, S.pre, S.stride, G.tile_start + G.P);
    if (S.marks) S.marks->mark(s, "halo_scan");
    pdl_launch(k_halo_layout, 1, 1024, 0, s, G, S.pre, S.stride, S.list_len, S.send_base, S.g, S.gbase,
                                      S.boff, S.halo_info, S.cbase);
    if (S.marks) S.marks->mark(s, "halo_layout");
    // the tile's records staged in shared memory (all but the forces) when
    // they fit; plain launches keep the per-image reads
    const int stage = staged_bytes(A) - kForceStageBytes;
    if (!plain && stage <= kStagedMaxBytes) {
        static bool attribute_set = false;   // once per process (one device per process)
        if (!attribute_set) {
            cudaFuncSetAttribute(k_halo_scatter_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kStagedMaxBytes);
            attribute_set = true;
        }
        pdl_launch(k_halo_scatter_staged, G.max_tiles, NT, static_cast<std::size_t>(stage), s, G, A,
                   owned_off, ghost_off, G.tiles, G.tile_start + G.P, S.mask, S.pre, S.stride,
                   S.cbase, S.ghost_owner, S.ghost_entry, S.bowner, S.boff, S.bslot, S.bfirst);
    } else {
        per_subdomain(G, plain, [&](const Grid& Gs, int grid) {
            pdl_launch(k_halo_scatter, grid, NT, 0, s, Gs, A, owned_off, ghost_off, G.tiles,
                       G.tile_start + G.P, S.mask, S.pre, S.stride, S.cbase, S.ghost_owner,
                       S.ghost_entry, S.bowner, S.boff, S.bslot, S.bfirst);
        });
    }
    if (S.marks) S.marks->mark(s, "halo_scatter");
}


// A staged pass holds at most this much of the record, so that three CTAs
// (their tiles in flight at once) fit an SM's shared memory.
constexpr int kStagedPassBytes = 56 * 1024;

// Consecutive array groups of at most kStagedPassBytes; false if one array
// alone is wider.
bool staged_passes(const Arrays& A, int* ends, int& passes) {
    const int narrays = 13 + A.f.count;
    passes = 0;
    int start = 0;
    while (start < narrays) {
        int end = start;
        while (end < narrays && staged_range_bytes(A, start, end + 1) <= kStagedPassBytes) ++end;
        if (end == start || passes == kStagedArrays) return false;
        ends[passes++] = end;
        start = end;
    }
    return true;
}

void launch_step_classify(const Grid& G, const Arrays& A, long long src_off, const Scratch& S,
                          cudaStream_t s, bool counters_zeroed) {
    if (!counters_zeroed) cudaMemsetAsync(S.imm_total, 0, sizeof(int) * G.P * (3 + kMaxNeighbors), s);
    if (S.pairs) cudaMemsetAsync(S.pairs, 0, sizeof(int) * G.P * G.P, s);
    const double* x = A.d[0] + src_off;
    const double* y = A.d[1] + src_off;
    const double* z = A.d[2] + src_off;
    // the two forms of each shape have one signature
    auto pick = [&](auto plain, auto combined) { return S.classify_combine ? combined : plain; };
    switch (S.classify_threads) {
    case 64:
        pdl_launch(pick(k_step_classify<64, 16, false>, k_step_classify<64, 16, true>), G.max_tiles, 64, 0, s,
            G, x, y, z, S.cnt, S.stride, S.imm_total, S.imm_list, S.imm_bnd, S.imm_img, S.dest16,
            S.mask, S.pairs);
        break;
    case 256:
        pdl_launch(pick(k_step_classify<256, 5, false>, k_step_classify<256, 5, true>), G.max_tiles, 256, 0, s,
            G, x, y, z, S.cnt, S.stride, S.imm_total, S.imm_list, S.imm_bnd, S.imm_img, S.dest16,
            S.mask, S.pairs);
        break;
    default:
        pdl_launch(pick(k_step_classify<128, 12, false>, k_step_classify<128, 12, true>), G.max_tiles, 128, 0, s,
            G, x, y, z, S.cnt, S.stride, S.imm_total, S.imm_list, S.imm_bnd, S.imm_img, S.dest16,
            S.mask, S.pairs);
    }
}

void launch_step_layout(const Grid& G, const Scratch& S, cudaStream_t s) {
    StepTables T{S.imm_total, S.imm_list, S.imm_bnd, S.imm_img, S.imm_base, S.emig_info,
                 S.mig_results, S.list_ret, S.list_len, S.send_base, S.g, S.gbase, S.boff,
                 S.halo_info, S.cbase, S.cbase_imm, S.imm_tile_start, S.imm_tiles};
    pdl_launch(k_step_scan_layout, kStepCounters, 1024, 0, s, G, S.cnt, S.pre, S.stride, T, S.ticket);
    pdl_launch(k_tile_bases, stream_grid(static_cast<long long>(G.max_tiles) * 32), NT, 0, s,
        G, S.pre, S.stride, S.cbase, S.tile_bases, S.imm_total, S.imm_base, S.imm_tile_start,
        S.imm_tiles);
}

int staged_move_modes(const Arrays& A) {
    int ends[kStagedArrays], passes = 0;
    const bool split = staged_passes(A, ends, passes);
    const bool one = staged_bytes(A) <= kStagedMaxBytes;
    int modes = 1;   // direct reads always apply
    if (one || split) modes |= 2;
    if (one && split && passes > 1) modes |= 4;   // passes as an alternative to one pass
    if (staged_bytes(A) - kForceStageBytes <= kStagedMaxBytes) modes |= 8;
    return modes;
}

void launch_step_move(const Grid& G, const Arrays& A, long long src_off, long long dst_off,
                      long long ghost_off, const Scratch& S, cudaStream_t s) {
    static bool attribute_set = false;   // once per process (one device per process)
    if (!attribute_set) {
        cudaFuncSetAttribute(k_step_move_staged<true, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedMaxBytes);
        cudaFuncSetAttribute(k_step_move_staged<true, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedMaxBytes);
        cudaFuncSetAttribute(k_step_move_staged<false, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedMaxBytes);
        attribute_set = true;
    }
    const int narrays = 13 + A.f.count;
    const int whole = staged_bytes(A);
    int ends[kStagedArrays], passes = 0;
    const bool split = staged_passes(A, ends, passes);
    auto staged = [&](bool full, int a0, int a1, int index_outputs) {
        const int bytes = staged_range_bytes(A, a0, a1);
        if (full)
            pdl_launch(k_step_move_staged<true, false>, G.max_tiles, NT, bytes, s,
                G, A, src_off, dst_off, ghost_off, S.pre, S.stride, S.cbase, S.dest16, S.mask,
                S.tile_bases, S.emig_src, S.emig_dst, S.ghost_owner, S.ghost_entry, S.bowner,
                S.boff, S.bslot, S.bfirst, a0, a1, index_outputs);
        else
            pdl_launch(k_step_move_staged<false, false>, G.max_tiles, NT, bytes, s,
                G, A, src_off, dst_off, ghost_off, S.pre, S.stride, S.cbase, S.dest16, S.mask,
                S.tile_bases, S.emig_src, S.emig_dst, S.ghost_owner, S.ghost_entry, S.bowner,
                S.boff, S.bslot, S.bfirst, a0, a1, index_outputs);
    };
    if (S.move_staged == 3 && whole - kForceStageBytes <= kStagedMaxBytes) {
        pdl_launch(k_step_move_staged<true, true>, G.max_tiles, NT, whole - kForceStageBytes, s,
            G, A, src_off, dst_off, ghost_off, S.pre, S.stride, S.cbase, S.dest16, S.mask,
            S.tile_bases, S.emig_src, S.emig_dst, S.ghost_owner, S.ghost_entry, S.bowner, S.boff,
            S.bslot, S.bfirst, 0, narrays, 1);
    } else if (S.move_staged == 1 && whole <= kStagedMaxBytes) {
        staged(true, 0, narrays, 1);
    } else if (S.move_staged != 0 && split) {
        if (passes == 1) {
            staged(true, 0, narrays, 1);
        } else {
            for (int p = 0, a0 = 0; p < passes; a0 = ends[p++])
                staged(false, a0, ends[p], p == 0 ? 1 : 0);
        }
    } else {
        pdl_launch(k_step_move, G.max_tiles, NT, 0, s, G, A, src_off, dst_off, ghost_off, S.pre, S.stride,
                                               S.cbase, S.dest16, S.mask, S.emig_src, S.emig_dst,
                                               S.ghost_owner, S.ghost_entry, S.bowner, S.boff,
                                               S.bslot, S.bfirst);
    }
}

void launch_step_emigrants(const Grid& G, const Arrays& A, long long src_off, long long dst_off,
                           const Scratch& S, const int* local_imm, const int* gap, cudaStream_t s) {
    const int chunk_grid = S.max_chunks < sm_count() * 4 ? S.max_chunks : sm_count() * 4;
    const size_t smem = sizeof(int) * NW * G.P;
    pdl_launch(k_emig_hist, chunk_grid > 0 ? chunk_grid : 1, NT, smem, s, G.P, S.emig_info, S.emig_dst,
                                                                  S.emig_hist);
    pdl_launch(k_emig_colscan, G.P, NT, 0, s, G.P, S.emig_info, S.emig_hist, local_imm, G.status);
    pdl_launch(k_emig_place, chunk_grid > 0 ? chunk_grid : 1, NT, smem, s,
        G, A, src_off, dst_off, S.emig_info, S.emig_src, S.emig_dst, S.emig_hist, S.imm_base, gap);
    if (S.marks) S.marks->mark(s, "emig_place");
}

void launch_step_scan(const Grid& G, const Scratch& S, cudaStream_t s) {
    pdl_launch(k_scan_counters, kStepCounters, 1024, 0, s, S.cnt, S.pre, S.stride, G.tile_start + G.P);
}

void launch_step_export(const Grid& G, const Scratch& S, int* out, cudaStream_t s) {
    pdl_launch(k_step_export, 1, 1024, 0, s, G, S.pre, S.stride, out);
}

void launch_step_bases(const Grid& G, const Scratch& S, const int* imm_in, cudaStream_t s) {
    pdl_launch(k_tile_bases, stream_grid(static_cast<long long>(G.max_tiles) * 32), NT, 0, s,
        G, S.pre, S.stride, S.cbase, S.tile_bases, imm_in, S.imm_base, S.imm_tile_start,
        S.imm_tiles);
}

void launch_step_finish(const Grid& G, const Grid& Gn, const Arrays& A, long long src_off,
                        long long dst_off, long long ghost_off, const Scratch& S, cudaStream_t s) {
    launch_step_emigrants(G, A, src_off, dst_off, S, S.imm_total, nullptr, s);
    launch_step_immigrant_halo(Gn, A, dst_off, ghost_off, S, s);
}

void launch_step_immigrant_halo(const Grid& Gn, const Arrays& A, long long dst_off,
                                long long ghost_off, const Scratch& S, cudaStream_t s) {
    const Grid& G = Gn;
    // immigrants: masks, list ranks and ghost images over their segments
    const int imm_grid = G.max_tiles < sm_count() * 4 ? G.max_tiles : sm_count() * 4;
    pdl_launch(k_halo_classify, imm_grid, NT, 0, s, Gn, S.imm_tiles, S.imm_tile_start + G.P,
                                            A.d[0] + dst_off, A.d[1] + dst_off, A.d[2] + dst_off,
                                            S.mask, S.cnt2, S.stride);
    pdl_launch(k_scan_counters, kHaloCounters, 1024, 0, s, S.cnt2, S.pre2, S.stride,
                                                   S.imm_tile_start + G.P);
    pdl_launch(k_halo_scatter, imm_grid, NT, 0, s, Gn, A, dst_off, ghost_off, S.imm_tiles,
                                           S.imm_tile_start + G.P, S.mask, S.pre2, S.stride,
                                           S.cbase_imm, S.ghost_owner, S.ghost_entry, S.bowner,
                                           S.boff, S.bslot, S.bfirst);
}

void launch_fused_step(const Grid& G, const Grid& Gn, const Arrays& A, long long src_off,
                       long long dst_off, long long ghost_off, const Scratch& S, cudaStream_t s,
                       bool counters_zeroed) {
    launch_step_classify(G, A, src_off, S, s, counters_zeroed);
    if (S.marks) S.marks->mark(s, "step_classify");
    launch_step_layout(G, S, s);
    if (S.marks) S.marks->mark(s, "step_layout");
    launch_step_move(G, A, src_off, dst_off, ghost_off, S, s);
    if (S.marks) S.marks->mark(s, "step_move");
    launch_step_finish(G, Gn, A, src_off, dst_off, ghost_off, S, s);
    if (S.marks) S.marks->mark(s, "immigrant_halo");
}

// Shared memory of one tile of the arrays a refresh copies (x, y, z; with
// velocities and the fields for a full refresh).
int refresh_stage_bytes(const Arrays& A, bool positions_only) {
    int bytes = (positions_only ? 3 : 6) * (TILE * 8 + 32);
    if (!positions_only)
        for (int f = 0; f < A.f.count; ++f) bytes += TILE * A.f.bytes[f] + 32;
    return bytes;
}

void launch_halo_refresh(const Grid& G, const Arrays& A, long long owned_off, long long ghost_off,
                         bool positions_only, const Scratch& S, cudaStream_t s, int ctas_per_sm) {
    const int stage = refresh_stage_bytes(A, positions_only);
    // the tile walk pays a fixed latency per tile, the ghost walk one sector
    // per copied array and ghost: the tiles win once a full refresh copies
    // nine arrays or more (measured: 11 arrays 1.19 against 1.50 ms, 7 arrays
    // 0.39 against 0.31 ms, positions 0.30 against 0.15 ms)
    const bool tiles = S.refresh_kind == 2 || (S.refresh_kind == 3 && !positions_only &&
                                                6 + A.f.count >= 9);
    if (tiles && stage <= kStagedMaxBytes) {
        static bool attribute_set = false;   // once per process (one device per process)
        static std::mutex lock;
        static std::vector<std::pair<int, int>> per_sm_of;   // stage bytes -> CTAs per SM
        int per_sm = 0;
        {
            std::lock_guard<std::mutex> hold(lock);
            if (!attribute_set) {
                cudaFuncSetAttribute(k_halo_refresh_staged,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedMaxBytes);
                attribute_set = true;
            }
            for (const auto& e : per_sm_of)
                if (e.first == stage) per_sm = e.second;
            if (!per_sm) {
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_halo_refresh_staged, NT,
                                                                  stage) != cudaSuccess ||
                    per_sm < 1)
                    per_sm = 1;
                per_sm_of.emplace_back(stage, per_sm);
            }
        }
        if (ctas_per_sm > 0 && per_sm > ctas_per_sm) per_sm = ctas_per_sm;
        int grid = sm_count() * per_sm;
        if (grid > G.max_tiles) grid = G.max_tiles > 0 ? G.max_tiles : 1;
        pdl_launch(k_tile_boundary_starts, stream_grid(static_cast<long long>(G.max_tiles) + 1), NT, 0, s,
                   G, S.halo_info, S.bowner, S.tile_b0);
        pdl_launch(k_halo_refresh_staged, grid, NT, static_cast<std::size_t>(stage), s, G, A, owned_off,
                   ghost_off, positions_only ? 1 : 0, S.bowner, S.boff, S.bslot, S.bfirst,
                   S.ghost_entry, S.tile_b0);
        return;
    }
    if (S.refresh_kind == 1) {
        int grid = resident_grid(reinterpret_cast<const void*>(k_halo_refresh_owners), G.ncap);
        if (ctas_per_sm > 0 && grid > sm_count() * ctas_per_sm) grid = sm_count() * ctas_per_sm;
        pdl_launch(k_halo_refresh_owners, grid, NT, 0, s, G, A, owned_off, ghost_off, positions_only ? 1 : 0,
                                                  S.halo_info, S.bowner, S.boff, S.bslot,
                                                  S.bfirst, S.ghost_entry);
        return;
    }
    int grid = resident_grid(reinterpret_cast<const void*>(k_halo_refresh), G.gcap);
    if (ctas_per_sm > 0 && grid > sm_count() * ctas_per_sm) grid = sm_count() * ctas_per_sm;
    pdl_launch(k_halo_refresh, grid, NT, 0, s, G, A, owned_off, ghost_off,
                                                      positions_only ? 1 : 0, S.halo_info,
                                                      S.ghost_owner, S.ghost_entry);
}

void launch_forward_fields(const Grid& G, const Arrays& A, long long owned_off,
                           long long ghost_off, const FieldOps& F, const Scratch& S,
                           cudaStream_t s) {
    pdl_launch(k_forward_fields, resident_grid(reinterpret_cast<const void*>(k_forward_fields), G.gcap), NT, 0, s, A, owned_off, ghost_off, F, S.halo_info,
                                                        S.ghost_owner, G.status);
}

void launch_reverse_sum3(const Grid& G, double* ox, double* oy, double* oz, const double* gx,
                         const double* gy, const double* gz, const Scratch& S, cudaStream_t s,
                         const PlainLaunch* plain) {
    if (plain && plain->boundary_start) {
        for (int r = 0; r < G.P; ++r) {
            const int b0 = plain->boundary_start[r], b1 = plain->boundary_start[r + 1];
            if (b1 <= b0) continue;
            pdl_launch(k_reverse_sum3, stream_grid(b1 - b0), NT, 0, s, S.halo_info, S.bowner, S.boff,
                                                               S.bslot, S.bfirst, ox, oy, oz, gx, gy, gz,
                                                               G.status, b0, b1);
        }
    } else {
        const int grid = S.reverse_per_sm > 0 ? sm_count() * S.reverse_per_sm : stream_grid(G.ncap);
        pdl_launch(k_reverse_sum3, grid, NT, 0, s, S.halo_info, S.bowner, S.boff, S.bslot, S.bfirst, ox, oy, oz, gx,
                                           gy, gz, G.status, 0, -1);
    }
    if (S.marks) S.marks->mark(s, "reverse_sum");
}

void launch_reverse_fields(const Grid& G, const Arrays& A, long long owned_off,
                           long long ghost_off, const FieldOps& F, const Scratch& S,
                           cudaStream_t s) {
    pdl_launch(k_reverse_fields, resident_grid(reinterpret_cast<const void*>(k_reverse_fields), G.ncap), NT, 0, s, A, owned_off, ghost_off, F, S.halo_info,
                                                        S.bowner, S.boff, S.bslot, G.status);
}

void launch_rebalance(const Grid& G, const double* work, RebalanceParams params,
                      long long* call_counter, double* result, cudaStream_t s) {
    pdl_launch(k_rebalance, 1, 32, 0, s, G, work, params, call_counter, result);
}

void launch_owner_rank(const Grid& G, const double* x, const double* y, const double* z,
                       long long n, int* out, cudaStream_t s) {
    if (n > 0) pdl_launch(k_owner_rank, resident_grid(reinterpret_cast<const void*>(k_owner_rank), n), NT, 0, s, G, x, y, z, n, out);
}

void launch_out_of_domain(const Grid& G, const double* x, const double* y, const double* z,
                          int* flags, cudaStream_t s) {
    cudaMemsetAsync(flags, 0, sizeof(int) * G.P, s);
    pdl_launch(k_out_of_domain, resident_grid(reinterpret_cast<const void*>(k_out_of_domain), G.ncap), NT, 0, s, G, x, y, z, flags);
}

void mark(const Scratch& S, cudaStream_t s, const char* what) {
    if (S.marks) S.marks->mark(s, what);
}

void launch_pair_counts(int P, const Scratch& S, const int* obase_old, long long ncap, int* pairs,
                        cudaStream_t s) {
    cudaMemsetAsync(pairs, 0, sizeof(int) * static_cast<std::size_t>(P) * P, s);
    if (ncap > 0) {
        const long long want = (ncap + NT - 1) / NT, cap = static_cast<long long>(sm_count()) * 4;
        pdl_launch(k_pair_counts, static_cast<int>(want < cap ? want : cap), NT, 0, s,
            P, S.emig_info, S.emig_src, S.emig_dst, obase_old, pairs);
    }
}

namespace {
// Descriptor staging of launch_copies, reused from call to call: pinned host
// and device buffers, and an event after the kernel that last read them
// (the next call waits for it before it overwrites them).
struct CopyStage {
    std::mutex lock;
    CopyPiece* host = nullptr;
    CopyPiece* device = nullptr;
    std::size_t capacity = 0;
    cudaEvent_t done = nullptr;
};
CopyStage g_copy_stage;
}  // namespace

cudaError_t launch_copies(const std::vector<CopyPiece>& copies, cudaStream_t s) {
    std::size_t n = 0;
    for (const CopyPiece& c : copies) n += static_cast<std::size_t>((c.bytes + kCopyPiece - 1) / kCopyPiece);
    if (!n) return cudaSuccess;
    CopyStage& st = g_copy_stage;
    std::lock_guard<std::mutex> hold(st.lock);
    cudaError_t e = cudaSuccess;
    if (!st.done && (e = cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(st.done)) != cudaSuccess) return e;
    if (n > st.capacity) {
        const std::size_t cap = n + n / 2 + 1024;
        cudaFreeHost(st.host);
        cudaFree(st.device);
        st.host = nullptr;
        st.device = nullptr;
        st.capacity = 0;
        if ((e = cudaMallocHost(reinterpret_cast<void**>(&st.host), sizeof(CopyPiece) * cap)) != cudaSuccess) return e;
        if ((e = cudaMalloc(reinterpret_cast<void**>(&st.device), sizeof(CopyPiece) * cap)) != cudaSuccess) return e;
        st.capacity = cap;
    }
    std::size_t k = 0;
    for (const CopyPiece& c : copies)
        for (long long at = 0; at < c.bytes; at += kCopyPiece)
            st.host[k++] = {c.src + at, c.dst + at, c.bytes - at < kCopyPiece ? c.bytes - at : kCopyPiece};
    e = cudaMemcpyAsync(st.device, st.host, sizeof(CopyPiece) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    const long long cap = static_cast<long long>(sm_count()) * 8;
    const long long count = static_cast<long long>(n);
    pdl_launch(k_copy_pieces, static_cast<int>(count < cap ? count : cap), NT, 0, s, st.device, count);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaEventRecord(st.done, s);
}

void launch_wrap_inplace(double* x, double* y, double* z, long long n, const double* lower,
                         const double* extent, const int* periodic, cudaStream_t s) {
    if (n <= 0) return;
    const long long blocks = (n + NT - 1) / NT;   // one particle per thread
    pdl_launch(k_wrap_inplace, static_cast<int>(blocks < 1 ? 1 : (blocks < (1 << 30) ? blocks : (1 << 30))), NT, 0, s,
        x, y, z, n, make_double3(lower[0], lower[1], lower[2]),
        make_double3(extent[0], extent[1], extent[2]),
        make_int3(periodic[0], periodic[1], periodic[2]));
}

}  // namespace dsx
