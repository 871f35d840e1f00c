// The C++ drop-in (include/dsdecompx.hpp) driven like the reference's own
// sanity programs (examples/sanity_check/cuda/*.cu, mpi/regression.cpp),
// adapted to what one rank does: no ghosts, migrate wraps positions in place,
// split-phase misuse and bad arguments raise the reference's exception types.
//
// usage: dropin_sanity <positions.bin>
//   writes the x, y, z arrays before and after migrate (6 x 4096 doubles) for
//   the Python side to compare with the oracle; exits 0 when every check passed.
#include <dsdecompx.hpp>

#include <cuda_runtime_api.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
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
template <class E, class F>
bool throws(F&& f) {
    try {
        f();
    } catch (const E&) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}
double pseudo(unsigned long long seed, unsigned long long i) {
    unsigned long long z = seed * 0x9E3779B97F4A7C15ull + i * 0xBF58476D1CE4E5B9ull + 0x94D049BB133111EBull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return static_cast<double>(z >> 11) / static_cast<double>(1ull << 53);
}
}  // namespace

int main(int argc, char** argv) {
    int provided = 0;
    MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
    {
        using namespace dsdecompx;
        expect(halo_exchange_options_size() == sizeof(HaloExchangeOptions), "ABI probe");
        Config config;
        config.domain.upper = {10.0, 10.0, 10.0};
        config.halo.width = 1.5;
        expect(throws<std::invalid_argument>([&] { Decomp d(MPI_COMM_NULL, config); }), "null communicator");
        Config bad = config;
        bad.dynamic.relaxation = 0.0;
        expect(throws<std::invalid_argument>([&] { Decomp d(MPI_COMM_WORLD, bad); }), "bad dynamic config");
        bad = config;
        bad.process_grid.dimensions = {2, 1, 1};
        expect(throws<std::invalid_argument>([&] { Decomp d(MPI_COMM_WORLD, bad); }), "grid larger than ranks");
        bad = config;
        bad.domain.upper = {0.0, 1.0, 1.0};
        expect(throws<std::invalid_argument>([&] { Decomp d(MPI_COMM_WORLD, bad); }), "empty box");

        Decomp decomp(MPI_COMM_WORLD, config);
        decomp.set_performance_counters_enabled(true, true);
        const auto& topo = decomp.topology();
        expect(topo.size() == 1 && topo.rank() == 0, "one rank");
        expect(topo.neighbors().empty(), "one rank has no neighbors");
        expect(topo.local_domain().upper[0] == 10.0 && topo.local_domain().lower[2] == 0.0, "local domain");
        expect(decomp.owner_rank({25.0, -3.0, 5.0}) == 0, "owner of any position");

        constexpr std::size_t owned = 4096;
        auto particles = ParticleInfo::allocate(MemorySpace::CudaDevice, owned);
        std::vector<double> x(owned), y(owned), z(owned), ones(owned, 1.0);
        std::vector<int> ids(owned);
        for (std::size_t i = 0; i < owned; ++i) {
            x[i] = -15.0 + 40.0 * pseudo(1, i);
            y[i] = -15.0 + 40.0 * pseudo(2, i);
            z[i] = 10.0 * pseudo(3, i);
            ids[i] = static_cast<int>(i);
        }
        if (owned > 10) { x[3] = 10.0; y[5] = -0.0; z[7] = 20.0; x[9] = -1e-17; }
        if (argc > 1) {   // inputs first, outputs after the migrate below
            FILE* f = std::fopen(argv[1], "wb");
            if (f) {
                std::fwrite(x.data(), 8, owned, f);
                std::fwrite(y.data(), 8, owned, f);
                std::fwrite(z.data(), 8, owned, f);
                std::fclose(f);
            }
        }
        check(cudaMemcpy(particles.x_data(), x.data(), owned * 8, cudaMemcpyHostToDevice));
        check(cudaMemcpy(particles.y_data(), y.data(), owned * 8, cudaMemcpyHostToDevice));
        check(cudaMemcpy(particles.z_data(), z.data(), owned * 8, cudaMemcpyHostToDevice));
        check(cudaMemcpy(particles.mass_data(), ones.data(), owned * 8, cudaMemcpyHostToDevice));
        check(cudaMemcpy(particles.global_id_data(), ids.data(), owned * 4, cudaMemcpyHostToDevice));
        std::vector<double> feature(2 * owned * 3, 0.5);
        double* dfeat = nullptr;
        check(cudaMalloc(reinterpret_cast<void**>(&dfeat), feature.size() * 8));
        particles.add_field<double>("feature", dfeat, 2 * owned, 3);
        expect(throws<std::invalid_argument>([&] { particles.add_field<double>("feature", dfeat, 2 * owned, 3); }),
               "duplicate field");
        expect(throws<std::invalid_argument>([&] { particles.add_field<double>("small", dfeat, 3, 1); }),
               "undersized field");

        cudaStream_t stream{};
        check(cudaStreamCreate(&stream));
        expect(throws<std::invalid_argument>([&] { decomp.migrate(particles, nullptr); }),
               "migrate without a stream");
        const MigrationResult moved = decomp.migrate(particles, stream);
        check(cudaStreamSynchronize(stream));
        expect(moved.new_owned_count == owned && moved.retained_count == owned && moved.sent_count == 0 &&
                   !moved.ownership_changed, "one rank keeps every particle");
        expect(particles.owned_count() == owned && particles.ghost_count() == 0, "counts after migrate");
        check(cudaMemcpy(x.data(), particles.x_data(), owned * 8, cudaMemcpyDeviceToHost));
        check(cudaMemcpy(y.data(), particles.y_data(), owned * 8, cudaMemcpyDeviceToHost));
        check(cudaMemcpy(z.data(), particles.z_data(), owned * 8, cudaMemcpyDeviceToHost));
        bool inside = true;
        for (std::size_t i = 0; i < owned; ++i)
            inside = inside && x[i] >= 0.0 && x[i] <= 10.0 && y[i] >= 0.0 && y[i] <= 10.0 && z[i] >= 0.0 && z[i] <= 10.0;
        expect(inside, "wrapped into the box");
        if (argc > 1) {
            FILE* f = std::fopen(argv[1], "ab");
            if (f) {
                std::fwrite(x.data(), 8, owned, f);
                std::fwrite(y.data(), 8, owned, f);
                std::fwrite(z.data(), 8, owned, f);
                std::fclose(f);
            }
        }

        // halo on one rank: no ghosts (src/halo.cpp:325-350)
        const HaloResult built = decomp.exchange_halo(particles, HaloExchangeOptions{true, stream});
        expect(built.ghost_count == 0 && built.layout_changed && !built.plan_reused, "rebuild on one rank");
        const HaloResult again = decomp.exchange_halo(particles, HaloExchangeOptions{false, stream});
        expect(again.ghost_count == 0 && !again.layout_changed, "refresh on one rank");
        expect(!decomp.can_refresh_halo(particles), "one rank never refreshes a plan");

        // split-phase misuse is reported, not hung on (cuda/halo_reuse.cu:128-168)
        decomp.begin_halo_exchange(particles, HaloExchangeOptions{false, stream});
        expect(throws<std::logic_error>([&] {
                   decomp.begin_halo_exchange(particles, HaloExchangeOptions{false, stream});
               }), "second begin");
        expect(throws<std::logic_error>([&] { decomp.migrate(particles, stream); }), "migrate inside split phase");
        const HaloResult split = decomp.end_halo_exchange(particles);
        expect(split.ghost_count == 0, "split exchange");
        expect(throws<std::logic_error>([&] { decomp.end_halo_exchange(particles); }), "end without begin");

        // reverse and field exchanges: argument checks (cuda/forward_exchange.cu:173-179)
        expect(throws<std::invalid_argument>([&] { decomp.reverse_halo(particles, nullptr); }),
               "reverse_halo without a stream");
        decomp.reverse_halo(particles, stream);
        expect(throws<std::invalid_argument>([&] { decomp.forward_exchange(particles, {"no_such_field"}, stream); }),
               "unknown forward field");
        expect(throws<std::invalid_argument>([&] { decomp.forward_exchange(particles, {"feature"}, nullptr); }),
               "forward without a stream");
        decomp.forward_exchange(particles, {"feature"}, stream);
        expect(throws<std::invalid_argument>([&] {
                   decomp.reverse_exchange(particles, {{"feature", ReduceOp::Sum}, {"feature", ReduceOp::Max}}, stream);
               }), "duplicate reverse field");
        decomp.reverse_exchange(particles, {{"feature", ReduceOp::Sum}}, stream);

        // perf counters (mpi/regression.cpp:103-108, one rank)
        const PerfStats stats = decomp.get_stats();
        expect(stats.halo_calls == 3 && stats.migration_calls == 1, "perf counters");
        decomp.reset_stats();
        expect(decomp.get_stats().halo_calls == 0, "reset perf counters");

        // rebalance on one rank: attempted, no geometry change, then migrate
        RebalanceOptions options;
        options.force = true;
        options.local_work = 100.0;
        const RebalanceResult balance = decomp.rebalance(particles, options, stream);
        expect(balance.attempted && !balance.geometry_changed && balance.imbalance_before == 1.0 &&
                   balance.migration.new_owned_count == owned, "rebalance on one rank");
        // a negative (or NaN) work falls back to the owned count; an infinite
        // one is rejected (src/runtime.cpp:1025-1027, 350-354)
        options.local_work = std::numeric_limits<double>::infinity();
        expect(throws<std::invalid_argument>([&] { decomp.rebalance(particles, options, stream); }),
               "non-finite work");
        options.local_work = std::nan("");
        expect(decomp.rebalance(particles, options, stream).attempted, "NaN work means the owned count");

        // storage growth keeps the owned particles
        auto small = ParticleInfo::allocate(MemorySpace::CudaDevice, 16);
        std::vector<int> sixteen(16);
        for (int i = 0; i < 16; ++i) sixteen[static_cast<std::size_t>(i)] = 100 + i;
        check(cudaMemcpy(small.global_id_data(), sixteen.data(), 64, cudaMemcpyHostToDevice));
        small.resize_owned(1000);
        expect(small.capacity() >= 1000 && small.owned_count() == 1000, "growth");
        std::vector<int> back(16);
        check(cudaMemcpy(back.data(), small.global_id_data(), 64, cudaMemcpyDeviceToHost));
        expect(back == sixteen, "growth preserves the owned particles");

        // borrowed storage cannot grow
        auto borrowed = ParticleInfo::external(MemorySpace::CudaDevice, 8, 8);
        expect(throws<std::logic_error>([&] { borrowed.resize_owned(16); }), "borrowed storage");
        expect(throws<std::invalid_argument>([&] { ParticleInfo::external(MemorySpace::CudaDevice, 4, 8); }),
               "external view smaller than its counts");

        // managed memory works the same way and is readable from the host
        auto managed = ParticleInfo::allocate(MemorySpace::CudaManaged, 4);
        for (int i = 0; i < 4; ++i) {
            managed.x_data()[i] = 10.0 + i;
            managed.y_data()[i] = -1.0;
            managed.z_data()[i] = 5.0;
            managed.global_id_data()[i] = i;
        }
        decomp.migrate(managed, stream);
        check(cudaStreamSynchronize(stream));
        expect(managed.x_data()[0] == 0.0 && managed.x_data()[1] == 1.0 && managed.y_data()[2] == 9.0,
               "managed memory migrate");

        // host memory is not this build's path
        ParticleInfo host(4);
        expect(throws<std::invalid_argument>([&] { decomp.migrate(host, stream); }), "host memory");

        check(cudaStreamDestroy(stream));
        cudaFree(dfeat);
    }
    MPI_Finalize();
    if (failures) {
        std::fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    std::printf("dropin_sanity: ok\n");
    return 0;
}
