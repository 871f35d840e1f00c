// dsx_migrate_noalloc: a one-shot migrate of caller-owned device arrays that
// allocates no memory.  The reference has no counterpart: its migrate grows
// device buffers with cudaMalloc on demand (dsDecompX src/cuda/cuda_buffer.cpp).
//
// Who needs it: code that is not allowed to call cudaMalloc/cudaFree -- a
// solver whose framework owns all device memory through its own pool, code
// running in a latency-critical loop where an allocation's implicit device
// synchronization is unacceptable, or a plugin that must not change the
// process's memory footprint while it runs.  Such callers cannot create a
// dsx_grid (which allocates its storage once), so this entry point takes
// inputs and outputs from the caller and keeps its scratch (layout tables,
// per-tile counters, the emigrant list) in one file-scope device array of a
// fixed size.  The driver places that array on a device when it loads the
// library's device code there: at the first call on that device with lazy
// module loading (CUDA's default), or at library load with eager loading.
// From then on it is held until the process exits.
//
// Limits: at most kMaxRanks subdomains and kMaxParticles particles; core
// arrays only (no registered fields); the cuts are an input, so there is no
// automatic Dynamic rebalance.  All calls share the one scratch array and it
// keeps the previous call's contents: calls that overlap on the GPU (two
// streams, or two host threads) race and must be serialized by the caller.
#include "dsx.h"
#include "dsx_device.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

namespace {

constexpr int kMaxRanks = 64;
constexpr long long kMaxParticles = 262144;
constexpr int NT = 256;
constexpr int ITEMS = 4;
constexpr int TILE = NT * ITEMS;
constexpr int kMaxTiles = static_cast<int>(kMaxParticles / TILE) + kMaxRanks;

// Layout of the scratch array (byte offsets, each 256-aligned).
constexpr std::size_t align256(std::size_t v) { return (v + 255) / 256 * 256; }
namespace Layout {
constexpr std::size_t cuts = 0;                                            // 3*(kMaxRanks+1) doubles
constexpr std::size_t tables = align256(cuts + 3 * (kMaxRanks + 1) * 8);   // 8 int tables of kMaxRanks+1
constexpr std::size_t cnt = align256(tables + 8 * (kMaxRanks + 1) * 4);    // 2 x kMaxTiles+1 ints
constexpr std::size_t pre = align256(cnt + 2 * (kMaxTiles + 1) * 4);       // 2 x kMaxTiles+1 ints
constexpr std::size_t emig_src = align256(pre + 2 * (kMaxTiles + 1) * 4); // kMaxParticles ints
constexpr std::size_t emig_dst = align256(emig_src + kMaxParticles * 4);   // kMaxParticles ints
constexpr std::size_t results = align256(emig_dst + kMaxParticles * 4);    // kMaxRanks*6 long long
constexpr std::size_t info = align256(results + kMaxRanks * 6 * 8);        // 4 ints
constexpr std::size_t total = align256(info + 4 * 4);
}  // namespace Layout

// The scratch: about 2.2 MB per GPU, placed on a device when the library's
// device code is loaded there (the first call, with lazy loading) and held
// until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[Layout::total];

// tables: 0 n_in, 1 obase_in, 2 tile_start_in, 3 imm_total, 4 n_out,
//         5 obase_out, 6 imm_base, 7 retained
struct Scratch {
    double* cuts;
    int* t[8];
    int* cnt;
    int* pre;
    int* emig_src;
    int* emig_dst;
    long long* results;
    int* info;
};

Scratch carve(unsigned char* base) {
    Scratch s;
    s.cuts = reinterpret_cast<double*>(base + Layout::cuts);
    for (int k = 0; k < 8; ++k)
        s.t[k] = reinterpret_cast<int*>(base + Layout::tables) + k * (kMaxRanks + 1);
    s.cnt = reinterpret_cast<int*>(base + Layout::cnt);
    s.pre = reinterpret_cast<int*>(base + Layout::pre);
    s.emig_src = reinterpret_cast<int*>(base + Layout::emig_src);
    s.emig_dst = reinterpret_cast<int*>(base + Layout::emig_dst);
    s.results = reinterpret_cast<long long*>(base + Layout::results);
    s.info = reinterpret_cast<int*>(base + Layout::info);
    return s;
}

struct Box {
    int P;
    int dims[3];
    int periodic[3];
    double lower[3];
    double extent[3];
    int cut_offset[3];
};

struct Soa {
    const double* d[11];
    const int* type;
    const int* gid;
};

struct SoaOut {
    double* d[11];
    int* type;
    int* gid;
};

__device__ __forceinline__ int na_destination(const Box& B, const double* cuts, double px, double py,
                                              double pz, double& wx, double& wy, double& wz) {
    const double p[3] = {px, py, pz};
    double w[3];
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (B.periodic[a]) {
            w[a] = dsx::wrap_axis(p[a], B.lower[a], B.extent[a]);
            c[a] = dsx::axis_coordinate(cuts + B.cut_offset[a], B.dims[a],
                                        dsx::wrap_axis(w[a], B.lower[a], B.extent[a]));
        } else {
            w[a] = p[a];
            c[a] = dsx::axis_coordinate(cuts + B.cut_offset[a], B.dims[a], p[a]);
        }
    }
    wx = w[0];
    wy = w[1];
    wz = w[2];
    return (c[0] * B.dims[1] + c[1]) * B.dims[2] + c[2];
}

template <int THREADS>
__device__ __forceinline__ int na_scan(int v, int& total, int* ws) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < THREADS / 32 ? ws[lane] : 0;
        int winc = w;
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

__device__ __forceinline__ void na_copy(const Soa& in, const SoaOut& out, int src, int dst,
                                        double wx, double wy, double wz) {
    out.d[0][dst] = wx;
    out.d[1][dst] = wy;
    out.d[2][dst] = wz;
#pragma unroll
    for (int a = 3; a < 11; ++a) out.d[a][dst] = in.d[a][src];
    out.type[dst] = in.type[src];
    out.gid[dst] = in.gid[src];
}

// stays / emigrants per tile of the input layout; immigrants per destination
__global__ void __launch_bounds__(NT) k_na_classify(Box B, Soa in, Scratch S) {
    __shared__ int ws[33];
    const int g = blockIdx.x;
    const int* tile_start = S.t[2];
    if (g >= tile_start[B.P]) return;
    const int s = dsx::tile_owner(tile_start, B.P, g);
    const int begin = S.t[1][s] + (g - tile_start[s]) * TILE;
    const int end = min(begin + TILE, S.t[1][s] + S.t[0][s]);
    int stay = 0, emig = 0;
    for (int i = begin + threadIdx.x; i < end; i += NT) {
        double wx, wy, wz;
        const int d = na_destination(B, S.cuts, in.d[0][i], in.d[1][i], in.d[2][i], wx, wy, wz);
        if (d == s) ++stay;
        else {
            ++emig;
            atomicAdd(&S.t[3][d], 1);
        }
    }
    int stays, emigs;
    na_scan<NT>(stay, stays, ws);
    na_scan<NT>(emig, emigs, ws);
    if (threadIdx.x == 0) {
        S.cnt[g] = stays;
        S.cnt[(kMaxTiles + 1) + g] = emigs;
    }
}

// prefixes over tiles, the output layout and the per-subdomain results
__global__ void __launch_bounds__(1024) k_na_layout(Box B, Scratch S) {
    __shared__ int ws[33];
    const int ntiles = S.t[2][B.P];
    for (int k = 0; k < 2; ++k) {
        const int t = threadIdx.x;   // ntiles <= kMaxTiles < 1024
        const int v = t < ntiles ? S.cnt[k * (kMaxTiles + 1) + t] : 0;
        int total;
        const int e = na_scan<1024>(v, total, ws);
        if (t < ntiles) S.pre[k * (kMaxTiles + 1) + t] = e;
        if (t == 0) S.pre[k * (kMaxTiles + 1) + ntiles] = total;
    }
    __syncthreads();
    const int s = threadIdx.x;
    int retained = 0, next = 0, old = 0, received = 0;
    if (s < B.P) {
        retained = S.pre[S.t[2][s + 1]] - S.pre[S.t[2][s]];
        received = S.t[3][s];
        old = S.t[0][s];
        next = retained + received;
    }
    int total_next;
    const int ob = na_scan<1024>(next, total_next, ws);
    if (s < B.P) {
        S.t[4][s] = next;
        S.t[5][s] = ob;
        S.t[6][s] = ob + retained;
        S.t[7][s] = retained;
        long long* o = S.results + 6 * s;
        o[1] = old;
        o[2] = retained;
        o[3] = old - retained;
        o[4] = received;
        o[5] = next;
        o[0] = (o[3] != 0 || o[4] != 0) ? 1 : 0;
    }
    if (s == 0) {
        S.t[5][B.P] = total_next;
        S.info[0] = S.pre[(kMaxTiles + 1) + ntiles];   // emigrants
    }
}

// retained particles to their output slots (stable), emigrants listed in
// (source subdomain, source order)
__global__ void __launch_bounds__(NT) k_na_move(Box B, Soa in, SoaOut out, Scratch S) {
    __shared__ int s_stay[NT / 32], s_emig[NT / 32];
    const int g = blockIdx.x;
    const int* tile_start = S.t[2];
    if (g >= tile_start[B.P]) return;
    const int s = dsx::tile_owner(tile_start, B.P, g);
    const int begin = S.t[1][s] + (g - tile_start[s]) * TILE;
    const int end = min(begin + TILE, S.t[1][s] + S.t[0][s]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbegin = begin + warp * 32 * ITEMS;
    const unsigned lt = dsx::lanemask_lt();
    int dest[ITEMS];
    double wx[ITEMS], wy[ITEMS], wz[ITEMS];
    int nstay = 0, nemig = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = wbegin + j * 32 + lane;
        dest[j] = -1;
        if (i < end) dest[j] = na_destination(B, S.cuts, in.d[0][i], in.d[1][i], in.d[2][i], wx[j], wy[j], wz[j]);
        nstay += __popc(__ballot_sync(0xffffffffu, dest[j] == s));
        nemig += __popc(__ballot_sync(0xffffffffu, dest[j] >= 0 && dest[j] != s));
    }
    if (lane == 0) {
        s_stay[warp] = nstay;
        s_emig[warp] = nemig;
    }
    __syncthreads();
    int stay_base = S.t[5][s] + (S.pre[g] - S.pre[tile_start[s]]);
    int emig_base = S.pre[(kMaxTiles + 1) + g];
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
            na_copy(in, out, i, stay_base + __popc(bs & lt), wx[j], wy[j], wz[j]);
        } else if (dest[j] >= 0) {
            const int e = emig_base + __popc(be & lt);
            S.emig_src[e] = i;
            S.emig_dst[e] = dest[j];
        }
        stay_base += __popc(bs);
        emig_base += __popc(be);
    }
}

// one CTA per destination: its immigrants in emigrant-list order, i.e. by
// source subdomain, then source order (dsDecompX src/migration.cpp:511-518)
__global__ void __launch_bounds__(NT) k_na_place(Box B, Soa in, SoaOut out, Scratch S) {
    __shared__ int ws[33];
    const int d = blockIdx.x;
    const int E = S.info[0];
    int run = S.t[6][d];
    for (int base = 0; base < E; base += NT) {
        const int e = base + threadIdx.x;
        const int mine = e < E && S.emig_dst[e] == d ? 1 : 0;
        int total;
        const int rank = na_scan<NT>(mine, total, ws);
        if (mine) {
            const int src = S.emig_src[e];
            const double ox = in.d[0][src], oy = in.d[1][src], oz = in.d[2][src];
            const double wx = B.periodic[0] ? dsx::wrap_axis(ox, B.lower[0], B.extent[0]) : ox;
            const double wy = B.periodic[1] ? dsx::wrap_axis(oy, B.lower[1], B.extent[1]) : oy;
            const double wz = B.periodic[2] ? dsx::wrap_axis(oz, B.lower[2], B.extent[2]) : oz;
            na_copy(in, out, src, run + rank, wx, wy, wz);
        }
        run += total;
    }
}

std::mutex g_setup_mutex;
void* g_scratch_address[64] = {};

// Writes "dsDecompX: <message>" into the caller's buffer (if any); no heap.
int noalloc_fail(char* error, int capacity, int code, const char* message, long long value = -1) {
    if (error && capacity > 0) {
        if (value >= 0) std::snprintf(error, static_cast<std::size_t>(capacity), "dsDecompX: %s, got %lld", message, value);
        else std::snprintf(error, static_cast<std::size_t>(capacity), "dsDecompX: %s", message);
    }
    return code;
}

}  // namespace

extern "C" {

int dsx_migrate_noalloc(const dsx_grid_desc* desc, const double* cuts, const long long* counts_in,
                        const void* const* arrays_in, long long* counts_out,
                        void* const* arrays_out, long long* results, void* stream, char* error,
                        int error_capacity) {
    if (error && error_capacity > 0) error[0] = '\0';
    if (!desc || !counts_in || !arrays_in || !counts_out || !arrays_out)
        return noalloc_fail(error, error_capacity, DSX_E_INVALID, "null argument");
    const int P = desc->nranks;
    if (P < 1 || P > kMaxRanks)
        return noalloc_fail(error, error_capacity, DSX_E_LENGTH,
                            "dsx_migrate_noalloc handles 1 to 64 subdomains", P);
    const int dims[3] = {desc->dims[0], desc->dims[1], desc->dims[2]};
    // each factor is checked against P before the product is formed, so the
    // product cannot overflow (and the cut tables below cannot be overrun)
    for (int a = 0; a < 3; ++a)
        if (dims[a] < 1 || dims[a] > P)
            return noalloc_fail(error, error_capacity, DSX_E_INVALID,
                                "dsx_migrate_noalloc needs explicit dims whose product is nranks");
    if (static_cast<long long>(dims[0]) * dims[1] * dims[2] != P)
        return noalloc_fail(error, error_capacity, DSX_E_INVALID,
                            "dsx_migrate_noalloc needs explicit dims whose product is nranks");
    long long total = 0;
    for (int r = 0; r < P; ++r) {
        if (counts_in[r] < 0) return noalloc_fail(error, error_capacity, DSX_E_INVALID, "negative particle count");
        total += counts_in[r];
    }
    if (total > kMaxParticles)
        return noalloc_fail(error, error_capacity, DSX_E_LENGTH,
                            "dsx_migrate_noalloc handles at most 262144 particles", total);
    for (int a = 0; a < 13; ++a)
        if (total && (!arrays_in[a] || !arrays_out[a]))
            return noalloc_fail(error, error_capacity, DSX_E_INVALID,
                                "dsx_migrate_noalloc needs all 13 core arrays in and out");
    // Inputs and outputs must not overlap: the kernels read the inputs while
    // other CTAs write the outputs.
    const std::size_t elem[13] = {8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 4, 4};
    for (int a = 0; a < 13 && total; ++a)
        for (int b = 0; b < 13; ++b) {
            const auto in_lo = reinterpret_cast<std::uintptr_t>(arrays_in[a]);
            const auto out_lo = reinterpret_cast<std::uintptr_t>(arrays_out[b]);
            const std::uintptr_t in_hi = in_lo + elem[a] * static_cast<std::size_t>(total);
            const std::uintptr_t out_hi = out_lo + elem[b] * static_cast<std::size_t>(total);
            if (in_lo < out_hi && out_lo < in_hi)
                return noalloc_fail(error, error_capacity, DSX_E_INVALID,
                                    "dsx_migrate_noalloc: input and output arrays overlap");
        }
    Box B{};
    B.P = P;
    double host_cuts[3 * (kMaxRanks + 1)];
    int ncuts = 0;
    for (int a = 0; a < 3; ++a) {
        if (!(desc->upper[a] > desc->lower[a]))
            return noalloc_fail(error, error_capacity, DSX_E_INVALID, "global-domain extent must be positive");
        B.dims[a] = dims[a];
        B.periodic[a] = desc->periodic[a] ? 1 : 0;
        B.lower[a] = desc->lower[a];
        B.extent[a] = desc->upper[a] - desc->lower[a];
        B.cut_offset[a] = ncuts;
        for (int i = 0; i <= dims[a]; ++i, ++ncuts)
            host_cuts[ncuts] = cuts ? cuts[ncuts]
                                    : desc->lower[a] + B.extent[a] * static_cast<double>(i) /
                                                           static_cast<double>(dims[a]);
        // the rule of dsx_grid_set_cuts (Decomposition::set_axis_cuts,
        // dsDecompX src/decomp.cpp:146-163): span the domain, increase strictly
        const double* c = host_cuts + B.cut_offset[a];
        bool ok = c[0] == desc->lower[a] && c[dims[a]] == desc->upper[a];
        for (int i = 0; i < dims[a]; ++i) ok = ok && c[i] < c[i + 1];
        if (!ok)
            return noalloc_fail(error, error_capacity, DSX_E_INVALID,
                                "cuts must be strictly increasing and span the domain");
    }
    // Once per device, with that device current: the device address of the
    // scratch array (in host code its name is only a host-side stand-in).
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64)
        return noalloc_fail(error, error_capacity, DSX_E_RUNTIME, "no current CUDA device");
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_address[device]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
                return noalloc_fail(error, error_capacity, DSX_E_RUNTIME,
                                    "cudaGetSymbolAddress of the scratch array failed");
            g_scratch_address[device] = p;
        }
        base = static_cast<unsigned char*>(g_scratch_address[device]);
    }
    const Scratch S = carve(base);
    const auto s = static_cast<cudaStream_t>(stream);
    // input layout on the host: obase and tile_start are prefixes of the counts
    int tables[3 * (kMaxRanks + 1)] = {};
    int ob = 0, ts = 0;
    for (int r = 0; r < P; ++r) {
        tables[r] = static_cast<int>(counts_in[r]);
        tables[(kMaxRanks + 1) + r] = ob;
        tables[2 * (kMaxRanks + 1) + r] = ts;
        ob += static_cast<int>(counts_in[r]);
        ts += static_cast<int>((counts_in[r] + TILE - 1) / TILE);
    }
    tables[(kMaxRanks + 1) + P] = ob;
    tables[2 * (kMaxRanks + 1) + P] = ts;
    cudaError_t st = cudaMemcpyAsync(S.cuts, host_cuts, ncuts * sizeof(double), cudaMemcpyHostToDevice, s);
    if (st == cudaSuccess) st = cudaMemcpyAsync(S.t[0], tables, sizeof(tables), cudaMemcpyHostToDevice, s);
    // the immigrant counters must start at zero (the array keeps the last call's values)
    if (st == cudaSuccess) st = cudaMemsetAsync(S.t[3], 0, (kMaxRanks + 1) * sizeof(int), s);
    if (st != cudaSuccess) return noalloc_fail(error, error_capacity, DSX_E_RUNTIME, cudaGetErrorString(st));
    Soa in{};
    SoaOut out{};
    for (int a = 0; a < 11; ++a) {
        in.d[a] = static_cast<const double*>(arrays_in[a]);
        out.d[a] = static_cast<double*>(arrays_out[a]);
    }
    in.type = static_cast<const int*>(arrays_in[11]);
    in.gid = static_cast<const int*>(arrays_in[12]);
    out.type = static_cast<int*>(arrays_out[11]);
    out.gid = static_cast<int*>(arrays_out[12]);
    const int grid = ts > 0 ? ts : 1;
    k_na_classify<<<grid, NT, 0, s>>>(B, in, S);
    k_na_layout<<<1, 1024, 0, s>>>(B, S);
    k_na_move<<<grid, NT, 0, s>>>(B, in, out, S);
    k_na_place<<<P, NT, 0, s>>>(B, in, out, S);
    st = cudaGetLastError();
    if (st != cudaSuccess) return noalloc_fail(error, error_capacity, DSX_E_RUNTIME, cudaGetErrorString(st));
    int n_out[kMaxRanks];
    st = cudaMemcpyAsync(n_out, S.t[4], P * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (st == cudaSuccess && results)
        st = cudaMemcpyAsync(results, S.results, 6 * P * sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (st == cudaSuccess) st = cudaStreamSynchronize(s);
    if (st != cudaSuccess) return noalloc_fail(error, error_capacity, DSX_E_RUNTIME, cudaGetErrorString(st));
    for (int r = 0; r < P; ++r) counts_out[r] = n_out[r];
    return DSX_OK;
}

}  // extern "C"
