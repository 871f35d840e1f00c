// Drives the UNMODIFIED reference Host path (dsDecompX ExecutionMode::Host)
// with P virtual ranks, one thread per rank, over the in-process MPI stand-in
// in mpi_shim/.  TEST INFRASTRUCTURE ONLY: the pytest suite uses it to pin the
// C restatement (dsx_oracle.c) and to generate golden fixtures, and bench.py's
// reference arm times it as the reference's own CPU implementation.
//
// Every rank owns one dsdecompx::Decomp and one host dsdecompx::ParticleInfo;
// each ref_* operation runs the same public call on all ranks at once (the
// calls are collective in the reference, e.g. include/dsdecompx.hpp:200-237).
#include "dsdecompx.hpp"
#include "mpi.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace {

using dsdecompx::FieldType;

struct FieldSpec {
    std::string name;
    FieldType type = FieldType::Float64;
    std::size_t components = 1;
    std::size_t record_bytes() const {
        return components * dsdecompx::field_type_size(type);
    }
};

struct RankState {
    std::unique_ptr<dsdecompx::Decomp> decomp;
    dsdecompx::ParticleInfo particles;
    std::vector<std::vector<unsigned char>> field_storage;
    dsdecompx::MigrationResult migration{};
    dsdecompx::HaloResult halo{};
    dsdecompx::RebalanceResult rebalance{};
    std::string error;
    double seconds = 0.0;
};

struct Session {
    int size = 1;
    dsdecompx::Config config;
    std::vector<FieldSpec> fields;
    std::size_t field_capacity = 0;
    shim_world* world = nullptr;
    std::vector<RankState> ranks;
    std::vector<std::thread> threads;
    std::mutex mutex;
    std::condition_variable command_cv, done_cv;
    std::uint64_t generation = 0;
    int done = 0;
    bool quit = false;
    std::function<void(int, RankState&)> command;
    std::string error;
};

void worker(Session* s, int rank) {
    shim_bind_rank(s->world, rank);
    std::uint64_t seen = 0;
    for (;;) {
        std::function<void(int, RankState&)> command;
        {
            std::unique_lock<std::mutex> lock(s->mutex);
            s->command_cv.wait(lock, [&] { return s->quit || s->generation != seen; });
            if (s->quit) break;
            seen = s->generation;
            command = s->command;
        }
        RankState& state = s->ranks[static_cast<std::size_t>(rank)];
        state.error.clear();
        try {
            command(rank, state);
        } catch (const std::exception& e) {
            state.error = e.what();
        } catch (...) {
            state.error = "unknown exception";
        }
        {
            std::lock_guard<std::mutex> lock(s->mutex);
            ++s->done;
        }
        s->done_cv.notify_all();
    }
    shim_unbind_rank();
}

// Runs `command` on every rank and waits for all of them; returns 0 or -1
// with the first rank's error message kept in the session.
int run_all(Session* s, std::function<void(int, RankState&)> command) {
    {
        std::lock_guard<std::mutex> lock(s->mutex);
        s->command = std::move(command);
        s->done = 0;
        ++s->generation;
    }
    s->command_cv.notify_all();
    {
        std::unique_lock<std::mutex> lock(s->mutex);
        s->done_cv.wait(lock, [&] { return s->done == s->size; });
    }
    for (int r = 0; r < s->size; ++r) {
        const auto& e = s->ranks[static_cast<std::size_t>(r)].error;
        if (!e.empty()) {
            s->error = "rank " + std::to_string(r) + ": " + e;
            return -1;
        }
    }
    return 0;
}

template <class T>
void add_typed(dsdecompx::ParticleInfo& p, const FieldSpec& f, void* data,
               std::size_t capacity) {
    p.add_field<T>(f.name, static_cast<T*>(data), capacity, f.components);
}

void register_fields(Session* s, RankState& state) {
    for (std::size_t f = 0; f < s->fields.size(); ++f) {
        const FieldSpec& spec = s->fields[f];
        void* data = state.field_storage[f].data();
        switch (spec.type) {
        case FieldType::Int32: add_typed<std::int32_t>(state.particles, spec, data, s->field_capacity); break;
        case FieldType::Int64: add_typed<std::int64_t>(state.particles, spec, data, s->field_capacity); break;
        case FieldType::UInt32: add_typed<std::uint32_t>(state.particles, spec, data, s->field_capacity); break;
        case FieldType::UInt64: add_typed<std::uint64_t>(state.particles, spec, data, s->field_capacity); break;
        case FieldType::Float32: add_typed<float>(state.particles, spec, data, s->field_capacity); break;
        case FieldType::Float64: add_typed<double>(state.particles, spec, data, s->field_capacity); break;
        }
    }
}

// Array ids shared with the C restatement and the CUDA C-ABI:
// 0 x, 1 y, 2 z, 3 vx, 4 vy, 5 vz, 6 fx, 7 fy, 8 fz, 9 mass, 10 charge,
// 11 type, 12 global_id, 13 + f = registered field f.
unsigned char* array_base(Session* s, RankState& state, int array,
                          std::size_t* element) {
    auto& p = state.particles;
    if (array >= 0 && array <= 10) {
        *element = sizeof(double);
        double* base[11] = {p.x.data(), p.y.data(), p.z.data(), p.vx.data(),
                            p.vy.data(), p.vz.data(), p.fx.data(), p.fy.data(),
                            p.fz.data(), p.mass.data(), p.charge.data()};
        return reinterpret_cast<unsigned char*>(base[array]);
    }
    if (array == 11) { *element = sizeof(int); return reinterpret_cast<unsigned char*>(p.type.data()); }
    if (array == 12) { *element = sizeof(int); return reinterpret_cast<unsigned char*>(p.global_id.data()); }
    const int f = array - 13;
    if (f < 0 || f >= static_cast<int>(s->fields.size())) return nullptr;
    *element = s->fields[static_cast<std::size_t>(f)].record_bytes();
    return state.field_storage[static_cast<std::size_t>(f)].data();
}

std::vector<std::string> split_names(const char* joined) {
    std::vector<std::string> names;
    if (!joined) return names;
    std::stringstream stream(joined);
    std::string item;
    while (std::getline(stream, item, '\n')) names.push_back(item);
    return names;
}

}  // namespace

extern "C" {

const char* ref_last_error(void* handle) {
    return handle ? static_cast<Session*>(handle)->error.c_str() : "null session";
}

// policy: 0 Manual, 1 Balanced, 2 TopologyAware, 3 Dynamic.
// dynamic: {interval, imbalance_threshold, relaxation, minimum_cell_fraction}.
void* ref_create(int nranks, const int* dims, int policy, const double* lower,
                 const double* upper, const int* periodic, double halo_width,
                 int edges_and_corners, const double* dynamic, int nfields,
                 const char* names, const int* types,
                 const long long* components, long long field_capacity,
                 char* error, int error_length) {
    auto* s = new Session();
    s->size = nranks;
    dsdecompx::Config& c = s->config;
    c.execution = dsdecompx::ExecutionMode::Host;
    c.advanced.read_environment = false;
    for (int a = 0; a < 3; ++a) {
        c.domain.lower[a] = lower[a];
        c.domain.upper[a] = upper[a];
        c.domain.periodic[a] = periodic[a] != 0;
        c.process_grid.dimensions[a] = dims[a];
    }
    c.grid_policy = static_cast<dsdecompx::GridPolicy>(policy);
    c.halo.width = halo_width;
    c.halo.include_edges_and_corners = edges_and_corners != 0;
    if (dynamic) {
        c.dynamic.interval = static_cast<std::size_t>(dynamic[0]);
        c.dynamic.imbalance_threshold = dynamic[1];
        c.dynamic.relaxation = dynamic[2];
        c.dynamic.minimum_cell_fraction = dynamic[3];
    }
    const auto field_names = split_names(names);
    for (int f = 0; f < nfields; ++f) {
        FieldSpec spec;
        spec.name = field_names.at(static_cast<std::size_t>(f));
        spec.type = static_cast<FieldType>(types[f]);
        spec.components = static_cast<std::size_t>(components[f]);
        s->fields.push_back(spec);
    }
    s->field_capacity = static_cast<std::size_t>(field_capacity);
    s->world = shim_world_create(nranks);
    s->ranks.resize(static_cast<std::size_t>(nranks));
    for (auto& state : s->ranks) {
        state.field_storage.resize(s->fields.size());
        for (std::size_t f = 0; f < s->fields.size(); ++f)
            state.field_storage[f].assign(s->field_capacity * s->fields[f].record_bytes(), 0);
    }
    for (int r = 0; r < nranks; ++r) s->threads.emplace_back(worker, s, r);
    const int status = run_all(s, [s](int, RankState& state) {
        state.decomp = std::make_unique<dsdecompx::Decomp>(MPI_COMM_WORLD, s->config);
        state.particles = dsdecompx::ParticleInfo(0);
        register_fields(s, state);
    });
    if (status != 0) {
        if (error && error_length > 0) {
            std::strncpy(error, s->error.c_str(), static_cast<std::size_t>(error_length - 1));
            error[error_length - 1] = '\0';
        }
        run_all(s, [](int, RankState& state) { state.decomp.reset(); });
        {
            std::lock_guard<std::mutex> lock(s->mutex);
            s->quit = true;
        }
        s->command_cv.notify_all();
        for (auto& t : s->threads) t.join();
        shim_world_destroy(s->world);
        delete s;
        return nullptr;
    }
    return s;
}

int ref_destroy(void* handle) {
    auto* s = static_cast<Session*>(handle);
    if (!s) return 0;
    run_all(s, [](int, RankState& state) {
        state.particles = dsdecompx::ParticleInfo();
        state.decomp.reset();
    });
    {
        std::lock_guard<std::mutex> lock(s->mutex);
        s->quit = true;
    }
    s->command_cv.notify_all();
    for (auto& t : s->threads) t.join();
    shim_world_destroy(s->world);
    delete s;
    return 0;
}

int ref_size(void* handle) { return static_cast<Session*>(handle)->size; }

// dims[3], coords[3], local domain {lower xyz, upper xyz}
int ref_topology(void* handle, int rank, int* dims, int* coords, double* local) {
    auto* s = static_cast<Session*>(handle);
    const auto& t = s->ranks[static_cast<std::size_t>(rank)].decomp->topology();
    for (int a = 0; a < 3; ++a) {
        dims[a] = t.dimensions()[a];
        coords[a] = t.coordinates()[a];
        local[a] = t.local_domain().lower[a];
        local[3 + a] = t.local_domain().upper[a];
    }
    return 0;
}

// Per neighbor (in the reference's order): {rank, dx, dy, dz, slot} and shift.
int ref_neighbors(void* handle, int rank, int* count, int* info, double* shifts) {
    auto* s = static_cast<Session*>(handle);
    const auto& n = s->ranks[static_cast<std::size_t>(rank)].decomp->topology().neighbors();
    *count = static_cast<int>(n.size());
    for (std::size_t i = 0; i < n.size(); ++i) {
        info[5 * i + 0] = n[i].rank;
        info[5 * i + 1] = n[i].direction[0];
        info[5 * i + 2] = n[i].direction[1];
        info[5 * i + 3] = n[i].direction[2];
        info[5 * i + 4] = n[i].direction_slot;
        for (int a = 0; a < 3; ++a) shifts[3 * i + a] = n[i].periodic_shift[a];
    }
    return 0;
}

// Cuts of rank 0 (all ranks hold the same cuts), axis by axis.
int ref_cuts(void* handle, double* out) {
    auto* s = static_cast<Session*>(handle);
    const auto& cuts = s->ranks[0].decomp->topology().axis_cuts();
    std::size_t k = 0;
    for (int a = 0; a < 3; ++a)
        for (double c : cuts[static_cast<std::size_t>(a)]) out[k++] = c;
    return 0;
}

// Replaces rank's particles with n owned particles (no ghosts). `core` holds
// 11 double arrays (x..charge); missing arrays (null) become zeros.
int ref_set_owned(void* handle, int rank, long long n, const double* const* core,
                  const int* type, const int* global_id,
                  const void* const* fields) {
    auto* s = static_cast<Session*>(handle);
    RankState& state = s->ranks[static_cast<std::size_t>(rank)];
    if (static_cast<std::size_t>(n) > s->field_capacity && !s->fields.empty()) {
        s->error = "owned count exceeds the field capacity";
        return -1;
    }
    state.particles = dsdecompx::ParticleInfo(static_cast<std::size_t>(n));
    auto& p = state.particles;
    std::vector<double>* arrays[11] = {&p.x, &p.y, &p.z, &p.vx, &p.vy, &p.vz,
                                       &p.fx, &p.fy, &p.fz, &p.mass, &p.charge};
    for (int a = 0; a < 11; ++a) {
        if (core && core[a]) std::memcpy(arrays[a]->data(), core[a], sizeof(double) * static_cast<std::size_t>(n));
        else std::fill(arrays[a]->begin(), arrays[a]->end(), 0.0);
    }
    if (type) std::memcpy(p.type.data(), type, sizeof(int) * static_cast<std::size_t>(n));
    if (global_id) std::memcpy(p.global_id.data(), global_id, sizeof(int) * static_cast<std::size_t>(n));
    for (std::size_t f = 0; f < s->fields.size(); ++f) {
        auto& storage = state.field_storage[f];
        std::fill(storage.begin(), storage.end(), 0);
        if (fields && fields[f])
            std::memcpy(storage.data(), fields[f], s->fields[f].record_bytes() * static_cast<std::size_t>(n));
    }
    register_fields(s, state);
    return 0;
}

int ref_counts(void* handle, int rank, long long* owned, long long* ghosts) {
    auto* s = static_cast<Session*>(handle);
    const auto& p = s->ranks[static_cast<std::size_t>(rank)].particles;
    *owned = static_cast<long long>(p.owned_count());
    *ghosts = static_cast<long long>(p.ghost_count());
    return 0;
}

int ref_read(void* handle, int rank, int array, long long start, long long count, void* out) {
    auto* s = static_cast<Session*>(handle);
    std::size_t element = 0;
    unsigned char* base = array_base(s, s->ranks[static_cast<std::size_t>(rank)], array, &element);
    if (!base && count) { s->error = "bad array id"; return -1; }
    if (count) std::memcpy(out, base + element * static_cast<std::size_t>(start), element * static_cast<std::size_t>(count));
    return 0;
}

int ref_write(void* handle, int rank, int array, long long start, long long count, const void* in) {
    auto* s = static_cast<Session*>(handle);
    std::size_t element = 0;
    unsigned char* base = array_base(s, s->ranks[static_cast<std::size_t>(rank)], array, &element);
    if (!base && count) { s->error = "bad array id"; return -1; }
    if (count) std::memcpy(base + element * static_cast<std::size_t>(start), in, element * static_cast<std::size_t>(count));
    return 0;
}

// results per rank: {ownership_changed, previous, retained, sent, received, new_owned}
int ref_migrate(void* handle, long long* results) {
    auto* s = static_cast<Session*>(handle);
    const int status = run_all(s, [](int, RankState& state) {
        state.migration = state.decomp->migrate(state.particles);
    });
    if (status == 0 && results) {
        for (int r = 0; r < s->size; ++r) {
            const auto& m = s->ranks[static_cast<std::size_t>(r)].migration;
            long long* o = results + 6 * r;
            o[0] = m.ownership_changed; o[1] = static_cast<long long>(m.previous_owned_count);
            o[2] = static_cast<long long>(m.retained_count); o[3] = static_cast<long long>(m.sent_count);
            o[4] = static_cast<long long>(m.received_count); o[5] = static_cast<long long>(m.new_owned_count);
        }
    }
    return status;
}

// results per rank: {ghost_count, layout_changed, storage_reallocated, plan_reused}
int ref_exchange_halo(void* handle, int rebuild, long long* results) {
    auto* s = static_cast<Session*>(handle);
    const int status = run_all(s, [rebuild](int, RankState& state) {
        dsdecompx::HaloExchangeOptions options;
        options.rebuild = rebuild != 0;
        state.halo = state.decomp->exchange_halo(state.particles, options);
    });
    if (status == 0 && results) {
        for (int r = 0; r < s->size; ++r) {
            const auto& h = s->ranks[static_cast<std::size_t>(r)].halo;
            long long* o = results + 4 * r;
            o[0] = static_cast<long long>(h.ghost_count); o[1] = h.layout_changed;
            o[2] = h.storage_reallocated; o[3] = h.plan_reused;
        }
    }
    return status;
}

int ref_reverse_halo(void* handle) {
    auto* s = static_cast<Session*>(handle);
    return run_all(s, [](int, RankState& state) { state.decomp->reverse_halo(state.particles); });
}

// ops: 0 Sum, 1 Min, 2 Max, 3 Replace
int ref_reverse_exchange(void* handle, int nfields, const char* names, const int* ops) {
    auto* s = static_cast<Session*>(handle);
    const auto list = split_names(names);
    std::vector<dsdecompx::ReverseExchangeField> fields;
    for (int f = 0; f < nfields; ++f)
        fields.push_back({list.at(static_cast<std::size_t>(f)), static_cast<dsdecompx::ReduceOp>(ops[f])});
    return run_all(s, [fields](int, RankState& state) {
        state.decomp->reverse_exchange(state.particles, fields);
    });
}

// local_work: per-rank work metric or null (owned counts); results per rank:
// {attempted, geometry_changed, new_owned}; imbalance per rank.
int ref_rebalance(void* handle, const double* local_work, int force,
                  long long* results, double* imbalance) {
    auto* s = static_cast<Session*>(handle);
    const int status = run_all(s, [local_work, force](int rank, RankState& state) {
        dsdecompx::RebalanceOptions options;
        options.local_work = local_work ? local_work[rank] : -1.0;
        options.force = force != 0;
        state.rebalance = state.decomp->rebalance(state.particles, options);
    });
    if (status == 0) {
        for (int r = 0; r < s->size; ++r) {
            const auto& b = s->ranks[static_cast<std::size_t>(r)].rebalance;
            if (results) {
                results[3 * r + 0] = b.attempted;
                results[3 * r + 1] = b.geometry_changed;
                results[3 * r + 2] = static_cast<long long>(b.migration.new_owned_count);
            }
            if (imbalance) imbalance[r] = b.imbalance_before;
        }
    }
    return status;
}

int ref_set_halo_width(void* handle, double width) {
    auto* s = static_cast<Session*>(handle);
    return run_all(s, [width](int, RankState& state) { state.decomp->set_halo_width(width); });
}

int ref_invalidate_halo(void* handle) {
    auto* s = static_cast<Session*>(handle);
    return run_all(s, [](int, RankState& state) { state.decomp->invalidate_halo(); });
}

// Decomp::rescale_domain (invalidate == 0) or Decomp::update_domain on every rank.
int ref_rescale_domain(void* handle, const double* lower, const double* upper, int invalidate) {
    auto* s = static_cast<Session*>(handle);
    dsdecompx::GlobalDomain d = s->config.domain;   // periodicity as created
    for (int a = 0; a < 3; ++a) {
        d.lower[a] = lower[a];
        d.upper[a] = upper[a];
    }
    s->config.domain = d;
    return run_all(s, [d, invalidate](int, RankState& state) {
        if (invalidate) state.decomp->update_domain(d);
        else state.decomp->rescale_domain(d);
    });
}

int ref_owner_rank(void* handle, long long n, const double* positions, int* out) {
    auto* s = static_cast<Session*>(handle);
    const auto& d = *s->ranks[0].decomp;
    // owner_rank reads the Cartesian communicator: act as rank 0 meanwhile.
    shim_bind_rank(s->world, 0);
    for (long long i = 0; i < n; ++i)
        out[i] = d.owner_rank({positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]});
    shim_unbind_rank();
    return 0;
}

// Times one operation per call on all ranks, communication_test style: every
// rank waits at a barrier, runs the call and reports its wall time; the
// session's time is the slowest rank's.  op: 0 migrate, 1 exchange_halo
// (rebuild), 2 exchange_halo (refresh), 3 reverse_halo.
int ref_timed(void* handle, int op, double* seconds) {
    auto* s = static_cast<Session*>(handle);
    const int status = run_all(s, [op](int, RankState& state) {
        MPI_Barrier(MPI_COMM_WORLD);
        const auto start = std::chrono::steady_clock::now();
        dsdecompx::HaloExchangeOptions options;
        switch (op) {
        case 0: state.migration = state.decomp->migrate(state.particles); break;
        case 1: options.rebuild = true; state.halo = state.decomp->exchange_halo(state.particles, options); break;
        case 2: state.halo = state.decomp->exchange_halo(state.particles, options); break;
        case 3: state.decomp->reverse_halo(state.particles); break;
        default: throw std::invalid_argument("bad timed op");
        }
        state.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    });
    double slowest = 0.0;
    for (const auto& state : s->ranks) slowest = std::max(slowest, state.seconds);
    *seconds = slowest;
    return status;
}

}  // extern "C"
