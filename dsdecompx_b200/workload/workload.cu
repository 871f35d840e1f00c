// Synthetic-workload kernels for the benchmark harness (not part of the
// bookkeeping path): the per-step drift of the owned particles and the ghost
// forces that stand in for a user's force computation, and a compute-bound
// stand-in for interior force work (split-phase timings).  The first two draw
// N(0,1) deviates from a counter-based generator (splitmix64 of seed, step,
// particle id and axis, then Box-Muller), so a step's inputs do not depend on
// the order the particles sit in and the kernels can be captured in a CUDA
// graph.
#include "dsx.h"

#include <cuda_runtime.h>
#include <cstdint>

namespace {

// step number of the synthetic inputs; advanced on the device so that a
// captured step draws fresh deviates at every replay
__device__ unsigned long long g_step = 0;

__device__ __forceinline__ std::uint64_t splitmix64(std::uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Three standard normal deviates for counter `id` at `step`: two Box-Muller
// pairs in FP32 arithmetic (synthetic inputs only; the values are then used as
// FP64 displacements and forces).
__device__ __forceinline__ void normals3(std::uint64_t seed, std::uint64_t step, std::uint64_t id,
                                         double& a, double& b, double& c) {
    const std::uint64_t k1 = splitmix64(seed ^ splitmix64(step * 0x100000001B3ull + id));
    const std::uint64_t k2 = splitmix64(k1);
    const float u1 = (static_cast<float>(k1 >> 40) + 1.0f) * (1.0f / 16777216.0f);
    const float u2 = static_cast<float>((k1 >> 16) & 0xFFFFFFull) * (1.0f / 16777216.0f);
    const float u3 = (static_cast<float>(k2 >> 40) + 1.0f) * (1.0f / 16777216.0f);
    const float u4 = static_cast<float>((k2 >> 16) & 0xFFFFFFull) * (1.0f / 16777216.0f);
    const float r1 = sqrtf(-2.0f * __logf(u1)), r2 = sqrtf(-2.0f * __logf(u3));
    float s1, c1, s2, c2;
    __sincosf(6.2831853f * u2, &s1, &c1);
    __sincosf(6.2831853f * u4, &s2, &c2);
    a = r1 * c1;
    b = r1 * s1;
    c = r2 * c2;
}

__global__ void k_drift(double* x, double* y, double* z, const int* gid, long long n,
                        std::uint64_t seed, std::uint64_t step, double sigma) {
    step += g_step;
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += gridDim.x * 256ll) {
        double a, b, c;
        normals3(seed, step, static_cast<std::uint32_t>(gid[i]), a, b, c);
        x[i] += sigma * a;
        y[i] += sigma * b;
        z[i] += sigma * c;
    }
}

__global__ void k_ghost_forces(double* fx, double* fy, double* fz, const int* totals,
                               std::uint64_t seed, std::uint64_t step) {
    step += g_step;
    const long long n = totals[0];
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += gridDim.x * 256ll) {
        double a, b, c;
        normals3(seed, step, static_cast<std::uint64_t>(i), a, b, c);
        fx[i] = a;
        fy[i] = b;
        fz[i] = c;
    }
}

__global__ void k_advance() { ++g_step; }
__global__ void k_set_step(unsigned long long v) { g_step = v; }

// Drift of the owned particles and ghost forces in one launch (the step
// callback's work): a grid-stride pass over the owned particles (two per
// thread and pass, their loads issued together), then one over the ghosts;
// the CTA that finishes last moves the step counter on, after every CTA has
// read it.
__device__ unsigned int g_done = 0;

__global__ void __launch_bounds__(256, 5) k_step_work(double* x, double* y, double* z, const int* gid, long long n,
                            double* fx, double* fy, double* fz, const int* totals,
                            std::uint64_t seed, double sigma) {
    const std::uint64_t step = g_step;
    const long long stride = gridDim.x * 256ll;
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += 2 * stride) {
        const long long k = i + stride;
        const bool two = k < n;
        const int id0 = gid[i], id1 = two ? gid[k] : 0;
        double x0 = x[i], y0 = y[i], z0 = z[i], x1 = 0.0, y1 = 0.0, z1 = 0.0;
        if (two) {
            x1 = x[k];
            y1 = y[k];
            z1 = z[k];
        }
        double a, b, c;
        normals3(seed, step, static_cast<std::uint32_t>(id0), a, b, c);
        x[i] = x0 + sigma * a;
        y[i] = y0 + sigma * b;
        z[i] = z0 + sigma * c;
        if (two) {
            normals3(seed, step, static_cast<std::uint32_t>(id1), a, b, c);
            x[k] = x1 + sigma * a;
            y[k] = y1 + sigma * b;
            z[k] = z1 + sigma * c;
        }
    }
    const long long g = totals[0];
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < g; i += stride) {
        double a, b, c;
        normals3(seed, step, static_cast<std::uint64_t>(i), a, b, c);
        fx[i] = a;
        fy[i] = b;
        fz[i] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&g_done, 1u) == gridDim.x - 1) {
            g_done = 0;
            ++g_step;
        }
    }
}

// Stand-in for interior (owned-owned) force work between begin and end of a
// split halo exchange: per owned particle 24 B of positions in, `rounds` x 4
// independent FP64 multiply-add chains, 8 B out.  Bandwidth-light: it needs
// the SMs, not HBM.
__global__ void k_interior(const double* x, const double* y, const double* z, long long n,
                           int rounds, double* out) {
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += gridDim.x * 256ll) {
        double a = x[i], b = y[i], c = z[i], d = a + b;
        const double k1 = 0.999999, k2 = 1.0e-7;
        for (int r = 0; r < rounds; ++r) {
            a = fma(a, k1, k2);
            b = fma(b, k1, k2);
            c = fma(c, k1, k2);
            d = fma(d, k1, k2);
        }
        out[i] = a + b + c + d;
    }
}

int grid_for(long long n, int per_sm = 8) {
    int sms = 148, device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const long long want = (n + 255) / 256;
    const long long cap = static_cast<long long>(sms) * per_sm;
    return static_cast<int>(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

extern "C" {

// owned x, y, z += sigma * N(0,1), keyed by global_id
int dsxw_drift(const dsx_grid_view* v, unsigned long long seed, long long step, double sigma,
               void* stream) {
    const long long o = v->owned_offset;
    k_drift<<<grid_for(v->particles), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double*>(v->base[0]) + o, static_cast<double*>(v->base[1]) + o,
        static_cast<double*>(v->base[2]) + o, static_cast<const int*>(v->base[12]) + o,
        v->particles, seed, static_cast<std::uint64_t>(step), sigma);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// drift of plain device arrays (the single-rank drop-in workload)
int dsxw_drift_arrays(double* x, double* y, double* z, const int* gid, long long n,
                      unsigned long long seed, long long step, double sigma, void* stream) {
    k_drift<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        x, y, z, gid, n, seed, static_cast<std::uint64_t>(step), sigma);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// ghost forces of the current halo = N(0,1), keyed by ghost slot
int dsxw_ghost_forces(const dsx_grid_view* v, unsigned long long seed, long long step,
                      void* stream) {
    const long long g = v->ghost_offset;
    k_ghost_forces<<<grid_for(v->ghost_capacity), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double*>(v->base[6]) + g, static_cast<double*>(v->base[7]) + g,
        static_cast<double*>(v->base[8]) + g, v->halo_totals, seed, static_cast<std::uint64_t>(step));
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// dsxw_drift + dsxw_ghost_forces + dsxw_advance in one launch: the same
// values as the three calls with the same seed (step 0 offsets)
int dsxw_step_work(const dsx_grid_view* v, unsigned long long seed, double sigma, void* stream) {
    const long long o = v->owned_offset, g = v->ghost_offset;
    const long long span = v->particles > v->ghost_capacity ? v->particles : v->ghost_capacity;
    k_step_work<<<grid_for(span, 5), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double*>(v->base[0]) + o, static_cast<double*>(v->base[1]) + o,
        static_cast<double*>(v->base[2]) + o, static_cast<const int*>(v->base[12]) + o,
        v->particles, static_cast<double*>(v->base[6]) + g, static_cast<double*>(v->base[7]) + g,
        static_cast<double*>(v->base[8]) + g, v->halo_totals, seed, sigma);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// interior stand-in over the owned particles of a view; out holds v->particles
int dsxw_interior(const dsx_grid_view* v, int rounds, double* out, void* stream) {
    const long long o = v->owned_offset;
    k_interior<<<grid_for(v->particles), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double*>(v->base[0]) + o, static_cast<const double*>(v->base[1]) + o,
        static_cast<const double*>(v->base[2]) + o, v->particles, rounds, out);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// moves the device step counter on (call once per step, after the draws)
int dsxw_advance(void* stream) {
    k_advance<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>();
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// sets the device step counter (to replay the same draws on a second grid)
int dsxw_set_step(unsigned long long value, void* stream) {
    k_set_step<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(value);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // extern "C"
