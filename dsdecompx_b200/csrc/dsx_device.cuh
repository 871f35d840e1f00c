// Device-side data model of the B200 particle-bookkeeping engine.
//
// A virtual Cartesian grid of P subdomains lives in one GPU's HBM:
//
//   particle arrays  one allocation per array (11 doubles: x y z vx vy vz fx fy
//                    fz mass charge; 2 int32: type global_id; F registered
//                    fields of `bytes` bytes per particle), each laid out as
//                    [ owned A | owned B | ghosts ]
//                    with |owned A| = |owned B| = ncap (the total owned count,
//                    which migration conserves) and |ghosts| = gcap.
//   owned region     subdomain s owns [obase[s], obase[s] + n[s]) of the current
//                    owned half (A or B, swapped by every migrate), packed in
//                    subdomain order.
//   ghost region     receiver q's ghosts are [gbase[q], gbase[q] + g[q]),
//                    neighbor block by neighbor block in q's neighbor order.
//   tiles            work is cut into tiles of `tile` consecutive owned
//                    particles that never straddle two subdomains; tile_start
//                    (P+1 entries) is the exclusive prefix of ceil(n[s]/tile).
//
// All counts live on the device so that a whole step can be captured in a
// CUDA graph; the host reads them back only when an API call must return them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dsx {

// particles per tile of the tile kernels (256 threads x 2 groups of 32)
constexpr int kTile = 512;
constexpr int kMaxNeighbors = 26;
constexpr int kMaxFields = 16;
constexpr int kMaxRanks = 1024;
// per-tile halo counters: 26 neighbor lists, boundary owners, images
constexpr int kHaloCounters = 28;
constexpr int kBoundaryCounter = 26;
constexpr int kImageCounter = 27;

// status bits (device word, read by the host after a step)
constexpr unsigned kStatusGhostOverflow = 1u;
constexpr unsigned kStatusCutsInvalid = 2u;
constexpr unsigned kStatusMigrationMismatch = 4u;
constexpr unsigned kStatusCopyTimeout = 8u;   // a bulk copy did not complete

struct FieldSet {
    int count = 0;
    int bytes[kMaxFields] = {};          // per particle
    unsigned char* base[kMaxFields] = {}; // start of the [A|B|ghost] allocation
};

struct Arrays {
    double* d[11] = {};
    int* type = nullptr;
    int* gid = nullptr;
    FieldSet f;
};

// Static description of the grid and pointers to the device tables.
struct Grid {
    int P = 1;
    int dims[3] = {1, 1, 1};
    int periodic[3] = {1, 1, 1};
    double lower[3] = {0, 0, 0};
    double upper[3] = {1, 1, 1};
    double extent[3] = {1, 1, 1};   // upper - lower, computed once on the host
    double width = 0.0;             // halo width
    long long ncap = 0;             // owned half length (= total owned count)
    long long gcap = 0;             // ghost capacity
    int tile = 1024;
    int max_tiles = 1;              // ceil(ncap / tile) + P
    // window of tiles one launch covers: [tile_first, tile_end), tile_end < 0
    // meaning "to the layout's last tile" (plain mode launches per subdomain)
    int tile_first = 0;
    int tile_end = -1;
    int cut_offset[3] = {0, 0, 0};  // start of each axis in `cuts`

    // topology (static)
    const int* nn = nullptr;             // [P] neighbor count
    const int* nbr = nullptr;            // [P*26] neighbor rank or -1
    const int* recv_entry = nullptr;     // [P*26] entry index at the receiver
    const int* sender_of = nullptr;      // [P*26] receiver (q,m) -> sender r*26+n or -1
    const double* shift = nullptr;       // [P*26*3]
    const signed char* dir = nullptr;    // [P*26*3]
    const unsigned* lut = nullptr;       // [P*64] halo flags -> neighbor mask
    const int* coord = nullptr;          // [P] grid coordinates, 10 bits each (x<<20|y<<10|z)

    // geometry (changes with Dynamic boundaries)
    double* cuts = nullptr;

    // layout of the current owned half
    int* n = nullptr;            // [P]
    int* obase = nullptr;        // [P+1]
    int* tile_start = nullptr;   // [P+1]
    // per tile of the current layout: {subdomain, first particle, end, first
    // tile of that subdomain}, so a CTA finds its work with one 16-byte load
    const int4* tiles = nullptr;
    // next layout (written by migrate)
    int* n_next = nullptr;
    int* obase_next = nullptr;
    int* tile_start_next = nullptr;
    int4* tiles_next = nullptr;

    unsigned* status = nullptr;
};

// ---------------------------------------------------------------- helpers

// Periodic wrap exactly as the reference Host path rounds it:
// v -= lower; v -= floor(v / extent) * extent; v += lower
// (dsDecompX src/migration.cpp:83-87, 106-113).  No FMA contraction.
//
// Fast path: for 0 <= t < extent the correctly rounded quotient t / extent is
// at most 1 - 2^-53, so floor() of it is a zero q carrying t's sign; then
// q * extent is that zero and t - q * extent is t itself, except that a zero t
// (of either sign) gives +0.  So the fast path is (t == 0 ? +0 : t) + lower:
// the FP64 division, multiply and subtract are skipped without changing a bit
// of the result.  Every other input (outside the box, NaN, inf) divides.
//
// With lower == 0 the fast path needs no arithmetic at all: t is v itself
// and (t == 0 ? +0 : t) + 0 is v, or +0 for a zero of either sign.
__device__ __forceinline__ double wrap_axis(double v, double lower, double extent) {
    if (lower == 0.0 && v >= 0.0 && v < extent) return v == 0.0 ? 0.0 : v;
    const double t = __dsub_rn(v, lower);
    if (t >= 0.0 && t < extent) return __dadd_rn(t == 0.0 ? 0.0 : t, lower);
    const double q = floor(__ddiv_rn(t, extent));
    return __dadd_rn(__dsub_rn(t, __dmul_rn(q, extent)), lower);
}

// std::upper_bound(cuts, cuts + count, v) - cuts - 1, clamped to [0, dims-1]
// (dsDecompX src/migration.cpp:89-93).
__device__ __forceinline__ int axis_coordinate(const double* cuts, int dims, double v) {
    int lo = 0, hi = dims + 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v < cuts[mid]) hi = mid;
        else lo = mid + 1;
    }
    int c = lo - 1;
    c = c > dims - 1 ? dims - 1 : c;
    return c < 0 ? 0 : c;
}

// Subdomain that owns tile g: largest s with tile_start[s] <= g.
__device__ __forceinline__ int tile_owner(const int* tile_start, int P, int g) {
    int lo = 0, hi = P;   // invariant: tile_start[lo] <= g < tile_start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tile_start[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Programmatic dependent launch (sm_90+): every kernel of the library is
// launched with programmatic stream serialisation (pdl_launch in
// dsx_kernels.cu), so it may become resident while the kernel before it on
// the stream drains its last wave.  griddepcontrol.wait, the first thing
// every kernel does, holds it until that kernel has completed and its memory
// is visible; only then does it let the next kernel launch.  Since each
// kernel waits for its predecessor before anything else, a kernel's
// completion still implies the completion of everything enqueued before it.
// Launched without the attribute, both instructions do nothing.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Read-only (non-coherent) load: the copy kernels read one region and write
// another, so source loads may be reordered past the stores.
template <class T>
__device__ __forceinline__ T ro(const T* p) { return __ldg(p); }

// Copies one particle's registered fields (bytes per particle as laid out in
// `f`) from global index `src` to global index `dst`.
__device__ __forceinline__ void copy_fields(const FieldSet& f, long long src, long long dst) {
    for (int k = 0; k < f.count; ++k) {
        const int b = f.bytes[k];
        unsigned char* base = f.base[k];
        if ((b & 7) == 0) {
            const unsigned long long* s = reinterpret_cast<const unsigned long long*>(base + src * b);
            unsigned long long* d = reinterpret_cast<unsigned long long*>(base + dst * b);
            for (int w = 0; w < (b >> 3); ++w) d[w] = ro(s + w);
        } else {
            const unsigned* s = reinterpret_cast<const unsigned*>(base + src * b);
            unsigned* d = reinterpret_cast<unsigned*>(base + dst * b);
            for (int w = 0; w < (b >> 2); ++w) d[w] = ro(s + w);
        }
    }
}

}  // namespace dsx
