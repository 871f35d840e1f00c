// C++ face of the virtual grid (the dsx_grid_* calls of dsx.h): P subdomains
// of one box on one GPU, each the counterpart of one rank of a dsDecompX job,
// every collective call of the reference made once for all of them.
//
// Header-only over the C ABI: RAII ownership, std::vector in and out, and
// the drop-in's error convention (include/dsdecompx.hpp) -- exceptions whose
// message starts with "dsDecompX:": std::invalid_argument, std::logic_error,
// std::runtime_error, std::length_error, std::overflow_error.  Streams are
// cudaStream_t values passed as void*; null means the legacy default stream.
#pragma once

#include "dsx.h"

#include <array>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace dsx {

inline void check(int status) {
    if (status == DSX_OK) return;
    const std::string msg = dsx_last_error();
    switch (status) {
    case DSX_E_INVALID: throw std::invalid_argument(msg);
    case DSX_E_LOGIC: throw std::logic_error(msg);
    case DSX_E_LENGTH: throw std::length_error(msg);
    case DSX_E_OVERFLOW: throw std::overflow_error(msg);
    default: throw std::runtime_error(msg);
    }
}

struct FieldSpec {
    std::string name;
    int type = DSX_FLOAT64;   // DSX_INT32 .. DSX_FLOAT64
    int components = 1;
};

// Called inside a batched step with the step's stream and the grid's device
// view (counts in the view's device arrays); see dsx_grid_step.
using StepCallback = std::function<void(void* stream, const dsx_grid_view& view)>;

class VirtualGrid {
public:
    // particles: owned particles in total (migration conserves the count);
    // ghost_capacity: 0 estimates it (it grows on overflow).
    VirtualGrid(const dsx_grid_desc& desc, const std::vector<FieldSpec>& fields,
                long long particles, long long ghost_capacity = 0) {
        std::vector<dsx_field_desc> f;
        for (const FieldSpec& s : fields) f.push_back({s.name.c_str(), s.type, s.components});
        check(dsx_grid_create(&desc, f.empty() ? nullptr : f.data(), static_cast<int>(f.size()),
                              particles, ghost_capacity, &handle_));
        nranks_ = desc.nranks;
        nfields_ = static_cast<int>(fields.size());
    }
    ~VirtualGrid() {
        if (handle_) dsx_grid_destroy(handle_);
    }
    VirtualGrid(VirtualGrid&& o) noexcept { swap(o); }
    VirtualGrid& operator=(VirtualGrid&& o) noexcept {
        swap(o);
        return *this;
    }
    VirtualGrid(const VirtualGrid&) = delete;
    VirtualGrid& operator=(const VirtualGrid&) = delete;

    dsx_grid* handle() const noexcept { return handle_; }
    int size() const noexcept { return nranks_; }

    std::array<int, 3> dims() const {
        std::array<int, 3> d{};
        int coords[3];
        double local[6];
        check(dsx_grid_topology(handle_, 0, d.data(), coords, local));
        return d;
    }

    // ---- particles ----------------------------------------------------
    // counts[P] and host arrays (13 core arrays in dsx.h's id order, then
    // the fields), each concatenated in rank order; null core arrays are 0.
    void upload(const std::vector<long long>& counts, const std::vector<const void*>& arrays,
                void* stream = nullptr) {
        check(dsx_grid_upload(handle_, counts.data(), arrays.data(), stream));
    }
    std::vector<long long> download(const std::vector<void*>& arrays, void* stream = nullptr) {
        std::vector<long long> counts(static_cast<std::size_t>(nranks_));
        check(dsx_grid_download(handle_, counts.data(), arrays.data(), stream));
        return counts;
    }
    std::pair<std::vector<long long>, std::vector<long long>> counts(void* stream = nullptr) {
        std::vector<long long> owned(static_cast<std::size_t>(nranks_)), ghosts(owned.size());
        check(dsx_grid_counts(handle_, owned.data(), ghosts.data(), stream));
        return {owned, ghosts};
    }
    template <class T>
    std::vector<T> read(int rank, int array, long long start, long long count,
                        void* stream = nullptr) {
        std::vector<T> out(static_cast<std::size_t>(count));
        check(dsx_grid_read(handle_, rank, array, start, count, out.data(), stream));
        return out;
    }
    template <class T>
    void write(int rank, int array, long long start, const std::vector<T>& values,
               void* stream = nullptr) {
        check(dsx_grid_write(handle_, rank, array, start, static_cast<long long>(values.size()),
                             values.data(), stream));
    }
    dsx_grid_view view() const {
        dsx_grid_view v{};
        check(dsx_grid_view_get(handle_, &v));
        return v;
    }

    // ---- the reference's collective calls ------------------------------
    // Per rank {ownership_changed, previous, retained, sent, received, new_owned}.
    std::vector<std::array<long long, 6>> migrate(void* stream = nullptr) {
        std::vector<std::array<long long, 6>> r(static_cast<std::size_t>(nranks_));
        check(dsx_grid_migrate(handle_, stream, r.front().data()));
        return r;
    }
    // Per rank {ghost_count, layout_changed, storage_reallocated, plan_reused}.
    std::vector<std::array<long long, 4>> exchange_halo(bool rebuild = false,
                                                        bool positions_only = false,
                                                        void* stream = nullptr) {
        std::vector<std::array<long long, 4>> r(static_cast<std::size_t>(nranks_));
        check(dsx_grid_exchange_halo(handle_, rebuild ? 1 : 0, positions_only ? 1 : 0, stream,
                                     r.front().data()));
        return r;
    }
    void begin_halo_exchange(bool rebuild = false, bool positions_only = false,
                             void* stream = nullptr) {
        check(dsx_grid_begin_halo_exchange(handle_, rebuild ? 1 : 0, positions_only ? 1 : 0,
                                           stream));
    }
    std::vector<std::array<long long, 4>> end_halo_exchange(void* stream = nullptr) {
        std::vector<std::array<long long, 4>> r(static_cast<std::size_t>(nranks_));
        check(dsx_grid_end_halo_exchange(handle_, stream, r.front().data()));
        return r;
    }
    void reverse_halo(void* stream = nullptr) { check(dsx_grid_reverse_halo(handle_, stream)); }
    // field ids: indices into the create-time list; ops: DSX_SUM .. DSX_REPLACE
    void reverse_exchange(const std::vector<int>& ids, const std::vector<int>& ops,
                          void* stream = nullptr) {
        if (ids.size() != ops.size()) throw std::invalid_argument("dsDecompX: one op per field");
        check(dsx_grid_reverse_exchange(handle_, static_cast<int>(ids.size()), ids.data(),
                                        ops.data(), stream));
    }
    void forward_exchange(const std::vector<int>& ids, void* stream = nullptr) {
        check(dsx_grid_forward_exchange(handle_, static_cast<int>(ids.size()), ids.data(), stream));
    }
    void set_halo_width(double width) { check(dsx_grid_set_halo_width(handle_, width)); }
    void invalidate_halo() { check(dsx_grid_invalidate_halo(handle_)); }

    // ---- geometry -------------------------------------------------------
    std::array<std::vector<double>, 3> cuts(void* stream = nullptr) {
        const std::array<int, 3> d = dims();
        std::vector<double> flat(static_cast<std::size_t>(d[0] + d[1] + d[2] + 3));
        check(dsx_grid_cuts(handle_, flat.data(), stream));
        std::array<std::vector<double>, 3> out;
        for (int a = 0, k = 0; a < 3; k += d[a] + 1, ++a)
            out[a].assign(flat.begin() + k, flat.begin() + k + d[a] + 1);
        return out;
    }
    void set_cuts(const std::array<std::vector<double>, 3>& cuts, void* stream = nullptr) {
        const std::array<int, 3> d = dims();
        std::vector<double> flat;
        for (int a = 0; a < 3; ++a) {
            if (cuts[a].size() != static_cast<std::size_t>(d[a] + 1))
                throw std::invalid_argument("dsDecompX: dynamic cut count does not match process grid");
            flat.insert(flat.end(), cuts[a].begin(), cuts[a].end());
        }
        check(dsx_grid_set_cuts(handle_, flat.data(), stream));
    }
    // Decomp::rescale_domain (update = false) or update_domain (update = true).
    void rescale_domain(const std::array<double, 3>& lower, const std::array<double, 3>& upper,
                        bool update = false, void* stream = nullptr) {
        check(dsx_grid_rescale_domain(handle_, lower.data(), upper.data(), update ? 1 : 0, stream));
    }
    // Decomp::rebalance: work per rank (empty: owned counts).
    std::vector<std::array<long long, 3>> rebalance(const std::vector<double>& work = {},
                                                    bool force = false,
                                                    void* stream = nullptr) {
        std::vector<std::array<long long, 3>> r(static_cast<std::size_t>(nranks_));
        double imbalance = 0.0;
        check(dsx_grid_rebalance(handle_, work.empty() ? nullptr : work.data(), force ? 1 : 0,
                                 stream, r.front().data(), &imbalance));
        return r;
    }
    std::vector<int> out_of_domain(void* stream = nullptr) {
        std::vector<int> flags(static_cast<std::size_t>(nranks_));
        int any = 0;
        check(dsx_grid_out_of_domain(handle_, flags.data(), &any, stream));
        return flags;
    }

    // ---- the batched step -------------------------------------------------
    // The callback is kept until replaced; replacing it makes the next
    // captured step capture anew.
    void set_step_callback(StepCallback callback) {
        callback_ = std::make_unique<StepCallback>(std::move(callback));
    }
    // One step (migrate -> halo build -> callback -> reverse_halo); returns
    // the device status bits (0: ok).
    unsigned step(bool capture, void* stream) {
        unsigned status = 0;
        check(dsx_grid_step(handle_, callback_ ? &trampoline : nullptr, callback_.get(),
                            capture ? 1 : 0, stream, &status));
        return status;
    }
    // The same step queued behind the previous one (dsx_grid_step_async; a
    // created stream); step_wait completes the queue and returns the OR of
    // the queued steps' status bits.
    void step_async(void* stream) {
        check(dsx_grid_step_async(handle_, callback_ ? &trampoline : nullptr, callback_.get(),
                                  stream));
    }
    unsigned step_wait() {
        unsigned status = 0;
        check(dsx_grid_step_wait(handle_, &status));
        return status;
    }
    // Refresh walk (dsx_grid_set_refresh_kind): 0 ghosts, 1 owners, 2 tiles, 3 auto
    void set_refresh_kind(int kind) { check(dsx_grid_set_refresh_kind(handle_, kind)); }
    // classify_threads 64/128/256, move_kind as dsx_tune_report.move_staged,
    // reverse_ctas_per_sm 0..32, classify_combine as dsx_tune_report's
    void set_tuning(int classify_threads, int move_kind, int reverse_ctas_per_sm,
                    bool classify_combine = false) {
        check(dsx_grid_set_tuning(handle_, classify_threads, move_kind, reverse_ctas_per_sm,
                                  classify_combine ? 1 : 0));
    }
    dsx_tune_report autotune(void* stream = nullptr) {
        dsx_tune_report r{};
        check(dsx_grid_autotune(handle_, stream, &r));
        return r;
    }

private:
    static void trampoline(void* user, void* stream, const dsx_grid_view* view) {
        (*static_cast<StepCallback*>(user))(stream, *view);
    }
    void swap(VirtualGrid& o) noexcept {
        std::swap(handle_, o.handle_);
        std::swap(nranks_, o.nranks_);
        std::swap(nfields_, o.nfields_);
        std::swap(callback_, o.callback_);
    }

    dsx_grid* handle_ = nullptr;
    int nranks_ = 0;
    int nfields_ = 0;
    std::unique_ptr<StepCallback> callback_;
};

}  // namespace dsx
