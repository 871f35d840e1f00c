// The virtual grid's C++ face (include/dsx_grid.hpp) driven like the
// reference's own sanity programs (examples/sanity_check/mpi/regression.cpp):
// migration conserves the particles and their ids, every ghost adds exactly
// its own contribution to its owner in reverse_halo (the sum of what the
// reverse adds equals the number of ghosts), the batched step (captured in a
// CUDA graph, callback a std::function) keeps both, split-phase misuse and
// bad cut planes raise the reference's exception types.
//
// usage: grid_sanity    (exits 0 and prints "grid_sanity: ok" when every
//                        check passed)
#include <dsx_grid.hpp>

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <stdexcept>
#include <vector>

namespace {
int failures = 0;
void expect(bool ok, const char* what) {
    if (!ok) {
        std::fprintf(stderr, "FAILED: %s\n", what);
        ++failures;
    }
}
void check(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

// splitmix64 -> uniform doubles, so that the program needs nothing else
struct Rng {
    std::uint64_t s;
    double uniform() {
        std::uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    }
};

constexpr int kP = 8;
constexpr long long kN = 40000;
constexpr double kL = 20.0;

std::vector<int> sorted_ids(dsx::VirtualGrid& grid) {
    std::vector<int> ids(static_cast<std::size_t>(kN));
    std::vector<void*> arrays(14, nullptr);
    arrays[12] = ids.data();   // global_id
    grid.download(arrays);
    std::sort(ids.begin(), ids.end());
    return ids;
}

// Sum of fx over every owned particle.
double owned_fx(dsx::VirtualGrid& grid) {
    std::vector<double> fx(static_cast<std::size_t>(kN));
    std::vector<void*> arrays(14, nullptr);
    arrays[6] = fx.data();
    grid.download(arrays);
    return std::accumulate(fx.begin(), fx.end(), 0.0);
}

long long total_ghosts(dsx::VirtualGrid& grid) {
    const auto c = grid.counts();
    return std::accumulate(c.second.begin(), c.second.end(), 0ll);
}
}  // namespace

int main() {
    try {
        dsx_grid_desc desc{};
        desc.nranks = kP;
        desc.dims[0] = desc.dims[1] = desc.dims[2] = 2;
        desc.policy = DSX_MANUAL;
        for (int a = 0; a < 3; ++a) {
            desc.lower[a] = 0.0;
            desc.upper[a] = kL;
            desc.periodic[a] = 1;
        }
        desc.halo_width = 1.5;
        desc.edges_and_corners = 1;
        desc.dyn_interval = 1.0;
        desc.dyn_threshold = 1.10;
        desc.dyn_relaxation = 0.5;
        desc.dyn_min_fraction = 0.10;
        dsx::VirtualGrid grid(desc, {{"tag", DSX_INT64, 1}}, kN);
        expect(grid.size() == kP, "size");
        expect(grid.dims() == std::array<int, 3>{2, 2, 2}, "dims");

        // every particle starts on rank 0, positions anywhere in the box
        Rng rng{42};
        std::vector<double> x(kN), y(kN), z(kN), zero(kN, 0.0);
        std::vector<int> id(kN);
        std::vector<long long> tag(kN);
        for (long long i = 0; i < kN; ++i) {
            x[i] = kL * rng.uniform();
            y[i] = kL * rng.uniform();
            z[i] = kL * rng.uniform();
            id[i] = static_cast<int>(i);
            tag[i] = 1000 + i;
        }
        std::vector<const void*> arrays(14, nullptr);
        arrays[0] = x.data();
        arrays[1] = y.data();
        arrays[2] = z.data();
        arrays[6] = zero.data();
        arrays[12] = id.data();
        arrays[13] = tag.data();
        std::vector<long long> counts(kP, 0);
        counts[0] = kN;
        grid.upload(counts, arrays);

        const auto mig = grid.migrate();
        long long sent = 0, received = 0;
        for (const auto& r : mig) {
            sent += r[3];
            received += r[4];
        }
        expect(sent == received && sent > kN / 2, "migration sends and receives every mover");
        std::vector<int> want(static_cast<std::size_t>(kN));
        std::iota(want.begin(), want.end(), 0);
        expect(sorted_ids(grid) == want, "ids conserved by migrate");
        for (int v : grid.out_of_domain()) expect(v == 0, "every particle owned where it lies");

        // per call: each ghost gets f = 1, the reverse adds exactly #ghosts
        grid.exchange_halo(true);
        const long long ghosts = total_ghosts(grid);
        expect(ghosts > 0, "ghosts built");
        const dsx_grid_view v = grid.view();
        std::vector<double> ones(static_cast<std::size_t>(v.ghost_capacity), 1.0);
        check(cudaMemcpy(static_cast<double*>(v.base[6]) + v.ghost_offset, ones.data(),
                         sizeof(double) * ghosts, cudaMemcpyHostToDevice));
        const double before = owned_fx(grid);
        grid.reverse_halo();
        expect(owned_fx(grid) - before == static_cast<double>(ghosts), "sum of reverse == #ghosts");

        // the batched step, captured: the callback fills every ghost slot
        cudaStream_t stream;
        check(cudaStreamCreate(&stream));
        double* pinned = nullptr;
        const std::size_t most = 1u << 21;
        check(cudaMallocHost(reinterpret_cast<void**>(&pinned), sizeof(double) * most));
        std::fill(pinned, pinned + most, 1.0);
        grid.set_step_callback([&](void* s, const dsx_grid_view& view) {
            const std::size_t n = static_cast<std::size_t>(view.ghost_capacity);
            if (n > most) throw std::length_error("ghost region larger than the test buffer");
            check(cudaMemcpyAsync(static_cast<double*>(view.base[6]) + view.ghost_offset, pinned,
                                  sizeof(double) * n, cudaMemcpyHostToDevice,
                                  static_cast<cudaStream_t>(s)));
        });
        for (int step = 0; step < 3; ++step) {
            const double f0 = owned_fx(grid);
            expect(grid.step(true, stream) == 0, "step status");
            check(cudaStreamSynchronize(stream));
            expect(owned_fx(grid) - f0 == static_cast<double>(total_ghosts(grid)),
                   "step: sum of reverse == #ghosts");
            expect(sorted_ids(grid) == want, "step: ids conserved");
        }
        // the same steps queued back to back, completed by one wait
        for (int step = 0; step < 3; ++step) grid.step_async(stream);
        expect(grid.step_wait() == 0, "queued steps' status");
        expect(sorted_ids(grid) == want, "queued steps: ids conserved");

        // split phase and its misuse (std::logic_error), bad cuts (invalid_argument)
        grid.begin_halo_exchange(true);
        bool threw = false;
        try {
            grid.migrate();
        } catch (const std::logic_error&) {
            threw = true;
        }
        expect(threw, "migrate during a split exchange throws logic_error");
        const auto h = grid.end_halo_exchange();
        expect(h[0][0] >= 0, "end_halo_exchange counts");
        threw = false;
        try {
            grid.end_halo_exchange();
        } catch (const std::logic_error&) {
            threw = true;
        }
        expect(threw, "end without begin throws logic_error");
        threw = false;
        try {
            grid.set_cuts({std::vector<double>{0.0, 12.0, 12.0}, {0.0, 10.0, kL}, {0.0, 10.0, kL}});
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        expect(threw, "cuts that do not span the box throw invalid_argument");
        grid.set_cuts({std::vector<double>{0.0, 7.0, kL}, {0.0, 12.0, kL}, {0.0, 9.5, kL}});
        expect(grid.cuts()[0][1] == 7.0 && grid.cuts()[2][1] == 9.5, "cuts set");
        grid.migrate();
        expect(sorted_ids(grid) == want, "ids conserved after new cuts");
        grid.rescale_domain({0.0, 0.0, 0.0}, {2 * kL, 2 * kL, 2 * kL});
        // Decomposition::rescale_domain's arithmetic: lower + fraction * extent
        volatile double cut = 7.0, old_extent = kL, new_extent = 2 * kL;
        const double fraction = (cut - 0.0) / old_extent;
        expect(grid.cuts()[0][1] == 0.0 + fraction * new_extent, "rescale keeps the cut fractions");

        cudaFreeHost(pinned);
        cudaStreamDestroy(stream);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "FAILED with exception: %s\n", e.what());
        return 1;
    }
    if (failures) return 1;
    std::printf("grid_sanity: ok\n");
    return 0;
}
