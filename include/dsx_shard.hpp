// C++ face of the native sharded grid (dsx_shard_* of dsx_shard.h): RAII
// ownership, std::vector in and out, the drop-in's exception types (see
// dsx_grid.hpp), and the transport as three std::function objects.
//
//   dsx::Transport tr;
//   tr.sum_i64 = [&](long long* v, long long n) { MPI_Allreduce(MPI_IN_PLACE, v, n, ...); };
//   tr.sum_f64 = [&](double* v, long long n) { ... };
//   tr.messages = [&](const std::vector<dsx::Message>& out, const std::vector<dsx::Message>& in,
//                     void* stream) { ... };
//   dsx::ShardedGrid grid(desc, fields, capacity, rank, size, tr);
#pragma once

#include "dsx_grid.hpp"
#include "dsx_shard.h"

#include <array>
#include <functional>
#include <memory>
#include <vector>

namespace dsx {

// One point-to-point message: a device buffer and the peer shard.
struct Message {
    int peer;
    void* data;
    long long bytes;
};

// Throwing from a transport function makes the collective call fail with
// std::runtime_error on this shard (the other shards learn of it through
// their own transport).
struct Transport {
    std::function<void(long long* values, long long n)> sum_i64;
    std::function<void(double* values, long long n)> sum_f64;
    std::function<void(const std::vector<Message>& send, const std::vector<Message>& recv,
                       void* stream)> messages;
};

class ShardedGrid {
public:
    ShardedGrid(const dsx_grid_desc& desc, const std::vector<FieldSpec>& fields, long long capacity,
                int shard, int nshards, Transport transport, const std::vector<int>& owners = {},
                long long ghost_capacity = 0)
        : transport_(std::make_unique<Transport>(std::move(transport))) {
        std::vector<dsx_field_desc> f;
        for (const FieldSpec& s : fields) f.push_back({s.name.c_str(), s.type, s.components});
        const dsx_transport tr{transport_.get(), &sum_i64, &sum_f64, &messages};
        check(dsx_shard_create(&desc, f.empty() ? nullptr : f.data(), static_cast<int>(f.size()),
                               capacity, ghost_capacity, shard, nshards,
                               owners.empty() ? nullptr : owners.data(), &tr, &handle_));
        nranks_ = desc.nranks;
    }
    ~ShardedGrid() {
        if (handle_) dsx_shard_destroy(handle_);
    }
    ShardedGrid(const ShardedGrid&) = delete;
    ShardedGrid& operator=(const ShardedGrid&) = delete;

    dsx_shard* handle() const noexcept { return handle_; }

    std::vector<int> owners() const {
        std::vector<int> o(static_cast<std::size_t>(nranks_));
        check(dsx_shard_owners(handle_, o.data()));
        return o;
    }
    // The owners a shard created without them would get (host only).
    static std::vector<int> plan_owners(const std::array<int, 3>& dims, int nshards) {
        std::vector<int> o(static_cast<std::size_t>(dims[0]) * static_cast<std::size_t>(dims[1]) *
                           static_cast<std::size_t>(dims[2]));
        check(dsx_shard_plan_owners(dims.data(), nshards, o.data()));
        return o;
    }
    void upload(const std::vector<long long>& counts, const std::vector<const void*>& arrays,
                void* stream = nullptr) {
        check(dsx_shard_upload(handle_, counts.data(), arrays.data(), stream));
    }
    std::vector<long long> download(const std::vector<void*>& arrays, void* stream = nullptr) {
        std::vector<long long> counts(static_cast<std::size_t>(nranks_));
        check(dsx_shard_download(handle_, counts.data(), arrays.data(), stream));
        return counts;
    }
    std::pair<std::vector<long long>, std::vector<long long>> counts(void* stream = nullptr) {
        std::vector<long long> o(static_cast<std::size_t>(nranks_)), g(o.size());
        check(dsx_shard_counts(handle_, o.data(), g.data(), stream));
        return {o, g};
    }
    // Per subdomain {changed, previous, retained, sent, received, new_owned}
    // (this shard's subdomains filled).
    std::vector<std::array<long long, 6>> migrate(void* stream = nullptr) {
        std::vector<std::array<long long, 6>> r(static_cast<std::size_t>(nranks_));
        check(dsx_shard_migrate(handle_, stream, r.front().data()));
        return r;
    }
    std::vector<std::array<long long, 4>> exchange_halo(bool rebuild = false,
                                                        bool positions_only = false,
                                                        void* stream = nullptr) {
        std::vector<std::array<long long, 4>> r(static_cast<std::size_t>(nranks_));
        check(dsx_shard_exchange_halo(handle_, rebuild ? 1 : 0, positions_only ? 1 : 0, stream,
                                      r.front().data()));
        return r;
    }
    void reverse_halo(void* stream = nullptr) { check(dsx_shard_reverse_halo(handle_, stream)); }
    // One fused step (dsx_shard_step): migrate -> halo build ->
    // callback(stream, view of this shard's particles and receivers' ghosts)
    // -> reverse_halo; returns the device status bits (0: ok).
    unsigned step(const std::function<void(void* stream, const dsx_grid_view& view)>& callback,
                  void* stream = nullptr) {
        unsigned status = 0;
        check(dsx_shard_step(handle_, callback ? &step_trampoline : nullptr,
                             const_cast<void*>(static_cast<const void*>(&callback)), stream, &status));
        return status;
    }
    void forward_exchange(const std::vector<int>& ids, void* stream = nullptr) {
        check(dsx_shard_forward_exchange(handle_, static_cast<int>(ids.size()), ids.data(), stream));
    }
    void reverse_exchange(const std::vector<int>& ids, const std::vector<int>& ops,
                          void* stream = nullptr) {
        if (ids.size() != ops.size()) throw std::invalid_argument("dsDecompX: one op per field");
        check(dsx_shard_reverse_exchange(handle_, static_cast<int>(ids.size()), ids.data(),
                                         ops.data(), stream));
    }
    std::vector<std::array<long long, 3>> rebalance(const std::vector<double>& work = {},
                                                    bool force = false, void* stream = nullptr) {
        std::vector<std::array<long long, 3>> r(static_cast<std::size_t>(nranks_));
        double imbalance = 0.0;
        check(dsx_shard_rebalance(handle_, work.empty() ? nullptr : work.data(), force ? 1 : 0,
                                  stream, r.front().data(), &imbalance));
        return r;
    }
    dsx_grid_view owned_view() const {
        dsx_grid_view v{};
        check(dsx_shard_owned_view(handle_, &v));
        return v;
    }
    dsx_grid_view ghost_view() const {
        dsx_grid_view v{};
        check(dsx_shard_ghost_view(handle_, &v));
        return v;
    }

private:
    static void step_trampoline(void* user, void* stream, const dsx_grid_view* view) {
        (*static_cast<const std::function<void(void*, const dsx_grid_view&)>*>(user))(stream, *view);
    }
    static int sum_i64(void* u, long long* v, long long n) {
        return call([&] { static_cast<Transport*>(u)->sum_i64(v, n); });
    }
    static int sum_f64(void* u, double* v, long long n) {
        return call([&] { static_cast<Transport*>(u)->sum_f64(v, n); });
    }
    static int messages(void* u, int ns, const int* to, const void* const* sb, const long long* sn,
                        int nr, const int* from, void* const* rb, const long long* rn, void* stream) {
        return call([&] {
            std::vector<Message> out, in;
            for (int k = 0; k < ns; ++k) out.push_back({to[k], const_cast<void*>(sb[k]), sn[k]});
            for (int k = 0; k < nr; ++k) in.push_back({from[k], rb[k], rn[k]});
            static_cast<Transport*>(u)->messages(out, in, stream);
        });
    }
    template <class F>
    static int call(F&& f) {
        try {
            f();
            return DSX_OK;
        } catch (...) {   // never through the library's C frames
            return DSX_E_RUNTIME;
        }
    }

    dsx_shard* handle_ = nullptr;
    int nranks_ = 0;
    std::unique_ptr<Transport> transport_;
};

}  // namespace dsx
