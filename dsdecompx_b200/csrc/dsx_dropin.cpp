// The dsDecompX drop-in (include/dsdecompx.hpp) for ExecutionMode::Cuda on a
// single-rank periodic box, over the C ABI of dsx.h.
//
// Behaviour follows the reference's public contract call by call
// (dsDecompX src/runtime.cpp:757-1071, src/halo.cpp:296-872, src/migration.cpp):
// the same validation and exception types, the same counts and flags.  One rank
// owns the whole box, so the reference creates no ghosts (src/halo.cpp:325-350)
// and its Host path has nothing to reverse; migrate keeps every particle in its
// slot and wraps its position (dsx_rank_migrate, on the GPU).
#include "dsdecompx.hpp"
#include "dsx.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_set>

namespace dsdecompx {

namespace detail {
struct TopologyAccess {
    static int& rank(Topology& t) { return t.rank_; }
    static int& size(Topology& t) { return t.size_; }
    static Vec3i& dimensions(Topology& t) { return t.dimensions_; }
    static Vec3i& coordinates(Topology& t) { return t.coordinates_; }
    static LocalDomain& local_domain(Topology& t) { return t.local_domain_; }
    static std::vector<Neighbor>& neighbors(Topology& t) { return t.neighbors_; }
    static std::array<std::vector<double>, 3>& axis_cuts(Topology& t) { return t.axis_cuts_; }
};
}  // namespace detail

namespace {

[[noreturn]] void invalid(const std::string& what) { throw std::invalid_argument("dsDecompX: " + what); }

void cuda_require(cudaError_t status, const char* what) {
    if (status != cudaSuccess)
        throw std::runtime_error(std::string("dsDecompX: ") + what + ": " + cudaGetErrorString(status));
}

bool device_space(MemorySpace s) { return s == MemorySpace::CudaDevice || s == MemorySpace::CudaManaged; }

ParticleView allocate_device(MemorySpace space, std::size_t capacity) {
    ParticleView v;
    v.memory_space = space;
    v.count = capacity;
    if (capacity == 0) return v;
    auto one = [&](auto** p, std::size_t bytes) {
        cudaError_t st = space == MemorySpace::CudaManaged
                             ? cudaMallocManaged(reinterpret_cast<void**>(p), bytes)
                             : cudaMalloc(reinterpret_cast<void**>(p), bytes);
        cuda_require(st, space == MemorySpace::CudaManaged ? "cudaMallocManaged failed" : "cudaMalloc failed");
    };
    double** d[11] = {&v.x, &v.y, &v.z, &v.vx, &v.vy, &v.vz, &v.fx, &v.fy, &v.fz, &v.mass, &v.charge};
    try {
        for (auto* p : d) one(p, capacity * sizeof(double));
        one(&v.type, capacity * sizeof(int));
        one(&v.global_id, capacity * sizeof(int));
    } catch (...) {
        for (auto* p : d) if (*p) cudaFree(*p);
        if (v.type) cudaFree(v.type);
        if (v.global_id) cudaFree(v.global_id);
        throw;
    }
    return v;
}

void free_device(ParticleView& v) noexcept {
    double* d[11] = {v.x, v.y, v.z, v.vx, v.vy, v.vz, v.fx, v.fy, v.fz, v.mass, v.charge};
    for (double* p : d) if (p) cudaFree(p);
    if (v.type) cudaFree(v.type);
    if (v.global_id) cudaFree(v.global_id);
    v = {};
}

void copy_device(const ParticleView& from, ParticleView& to, std::size_t count) {
    if (!count) return;
    const double* s[11] = {from.x, from.y, from.z, from.vx, from.vy, from.vz, from.fx, from.fy,
                           from.fz, from.mass, from.charge};
    double* t[11] = {to.x, to.y, to.z, to.vx, to.vy, to.vz, to.fx, to.fy, to.fz, to.mass, to.charge};
    for (int a = 0; a < 11; ++a)
        cuda_require(cudaMemcpy(t[a], s[a], count * sizeof(double), cudaMemcpyDefault),
                     "cudaMemcpy while growing ParticleInfo failed");
    cuda_require(cudaMemcpy(to.type, from.type, count * sizeof(int), cudaMemcpyDefault),
                 "cudaMemcpy while growing ParticleInfo failed");
    cuda_require(cudaMemcpy(to.global_id, from.global_id, count * sizeof(int), cudaMemcpyDefault),
                 "cudaMemcpy while growing ParticleInfo failed");
}

double balanced_score(const GridShape& g, const DomainShape& d) {
    const double lx = d.lengths[0] / g.px, ly = d.lengths[1] / g.py, lz = d.lengths[2] / g.pz;
    const double surface = 2.0 * (1.0 / lx + 1.0 / ly + 1.0 / lz);
    return surface * (1.0 + 0.05 * std::log(std::max({lx, ly, lz}) / std::min({lx, ly, lz})));
}

double topology_score(const GridShape& g, const DomainShape& d, const TopologyInfo& t) {
    if (!t.available || t.rank_to_node.size() != static_cast<std::size_t>(g.px * g.py * g.pz))
        return balanced_score(g, d);
    const double local[3] = {d.lengths[0] / g.px, d.lengths[1] / g.py, d.lengths[2] / g.pz};
    const double face[3] = {local[1] * local[2], local[0] * local[2], local[0] * local[1]};
    const int dims[3] = {g.px, g.py, g.pz};
    double cost = 0.0;
    for (int x = 0; x < g.px; ++x)
        for (int y = 0; y < g.py; ++y)
            for (int z = 0; z < g.pz; ++z) {
                const int source = (x * g.py + y) * g.pz + z;
                for (int a = 0; a < 3; ++a) {
                    int c[3] = {x, y, z};
                    if (++c[a] == dims[a]) {
                        if (!d.periodic[a] || dims[a] == 1) continue;
                        c[a] = 0;
                    }
                    const int peer = (c[0] * g.py + c[1]) * g.pz + c[2];
                    if (peer == source) continue;
                    const bool same = t.rank_to_node[static_cast<std::size_t>(source)] ==
                                      t.rank_to_node[static_cast<std::size_t>(peer)];
                    cost += face[a] * (same ? t.intra_node_weight : t.inter_node_weight);
                }
            }
    return cost / (local[0] * local[1] * local[2] * g.px * g.py * g.pz) + 0.01 * balanced_score(g, d);
}

std::uint64_t field_schema_hash(const ConstParticleView& v) {
    std::uint64_t hash = 1469598103934665603ull;
    auto mix = [&](std::uint64_t value) {
        hash ^= value;
        hash *= 1099511628211ull;
    };
    mix(v.field_count);
    for (std::size_t f = 0; f < v.field_count; ++f) {
        for (const unsigned char c : v.fields[f].name) mix(c);
        mix(0xffu);
        mix(static_cast<std::uint8_t>(v.fields[f].type));
        mix(v.fields[f].components);
    }
    return hash;
}

}  // namespace

// ------------------------------------------------------------- free functions

const char* backend_selection_name(BackendSelection s) noexcept {
    switch (s) {
    case BackendSelection::Auto: return "auto";
    case BackendSelection::Mpi: return "mpi";
    case BackendSelection::Nccl: return "nccl";
    case BackendSelection::Nvshmem: return "nvshmem";
    }
    return "unknown";
}

BackendSelection parse_backend_selection(std::string_view value) {
    std::string v(value);
    std::transform(v.begin(), v.end(), v.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
    if (v == "auto") return BackendSelection::Auto;
    if (v == "mpi") return BackendSelection::Mpi;
    if (v == "nccl") return BackendSelection::Nccl;
    if (v == "nvshmem") return BackendSelection::Nvshmem;
    invalid("BACKEND must be auto, mpi, nccl, or nvshmem");
}

// Only the transport-free path exists: a single rank needs no backend.
bool backend_compiled(BackendSelection s) noexcept {
    return s == BackendSelection::Auto || s == BackendSelection::Mpi;
}

GridShape choose_process_grid(int nranks, const DomainShape& domain, const TopologyInfo& topology,
                              GridPolicy policy, GridShape manual) {
    if (nranks <= 0) invalid("nranks must be positive");
    for (double l : domain.lengths)
        if (!(l > 0.0)) invalid("domain lengths must be positive");
    if (policy == GridPolicy::Manual) {
        if (manual.px <= 0 || manual.py <= 0 || manual.pz <= 0 || manual.px * manual.py * manual.pz != nranks)
            invalid("manual process grid does not match nranks");
        return manual;
    }
    const bool use_topology = policy == GridPolicy::TopologyAware && topology.available &&
                              topology.rank_to_node.size() == static_cast<std::size_t>(nranks);
    double best_score = std::numeric_limits<double>::infinity();
    GridShape best{nranks, 1, 1};
    for (int px = 1; px <= nranks; ++px) {
        if (nranks % px) continue;
        const int rest = nranks / px;
        for (int py = 1; py <= rest; ++py) {
            if (rest % py) continue;
            const GridShape cand{px, py, rest / py};
            const double score = use_topology ? topology_score(cand, domain, topology) : balanced_score(cand, domain);
            if (std::make_tuple(score, px, py, cand.pz) < std::make_tuple(best_score, best.px, best.py, best.pz)) {
                best_score = score;
                best = cand;
            }
        }
    }
    return best;
}

std::size_t halo_exchange_options_size() noexcept { return sizeof(HaloExchangeOptions); }

// ---------------------------------------------------------------- ParticleInfo

ParticleInfo::~ParticleInfo() { release_device_memory(); }

ParticleInfo::ParticleInfo(ParticleInfo&& other) noexcept { *this = std::move(other); }

ParticleInfo& ParticleInfo::operator=(ParticleInfo&& o) noexcept {
    if (this == &o) return *this;
    release_device_memory();
    x = std::move(o.x); y = std::move(o.y); z = std::move(o.z);
    vx = std::move(o.vx); vy = std::move(o.vy); vz = std::move(o.vz);
    fx = std::move(o.fx); fy = std::move(o.fy); fz = std::move(o.fz);
    mass = std::move(o.mass); charge = std::move(o.charge);
    type = std::move(o.type); global_id = std::move(o.global_id);
    num_particles = o.num_particles;
    external_ = o.external_;
    owns_device_memory_ = o.owns_device_memory_;
    owned_count_ = o.owned_count_;
    ghost_count_ = o.ghost_count_;
    fields_ = std::move(o.fields_);
    storage_ = o.storage_;
    provider_ = o.provider_;
    storage_.fields = fields_.empty() ? nullptr : fields_.data();
    storage_.field_count = fields_.size();
    o.num_particles = 0;
    o.external_ = o.owns_device_memory_ = false;
    o.owned_count_ = o.ghost_count_ = 0;
    o.fields_.clear();
    o.storage_ = {};
    o.provider_ = nullptr;
    return *this;
}

void ParticleInfo::release_device_memory() noexcept {
    if (!owns_device_memory_) return;
    free_device(storage_);
    owns_device_memory_ = false;
}

ParticleInfo ParticleInfo::allocate(MemorySpace space, std::size_t owned) {
    if (space == MemorySpace::Host) return ParticleInfo(owned);
    ParticleInfo p;
    p.external_ = true;
    p.owns_device_memory_ = true;
    p.owned_count_ = owned;
    p.storage_ = allocate_device(space, owned);
    return p;
}

ParticleInfo ParticleInfo::external(MemorySpace space, std::size_t capacity, std::size_t owned,
                                    std::size_t ghosts) {
    ParticleView v;
    v.memory_space = space;
    v.count = capacity;
    return ParticleInfo(owned, ghosts, v);
}

ParticleInfo::ParticleInfo(std::size_t owned, std::size_t ghosts, ParticleView storage)
    : external_(true), owned_count_(owned), ghost_count_(ghosts), storage_(storage) {
    if (storage_.count < owned + ghosts) invalid("external particle view is smaller than its particle counts");
    if (storage.fields && storage.field_count) {
        fields_.assign(storage.fields, storage.fields + storage.field_count);
        storage_.fields = fields_.data();
        storage_.field_count = fields_.size();
    }
}

ParticleInfo::ParticleInfo(std::size_t owned, std::size_t ghosts, Provider& provider)
    : ParticleInfo(owned, ghosts, provider.particle_info_view(owned + ghosts)) {
    provider_ = &provider;
}

ParticleInfo& ParticleInfo::positions(double* a, double* b, double* c) noexcept {
    storage_.x = a; storage_.y = b; storage_.z = c;
    return *this;
}
ParticleInfo& ParticleInfo::velocities(double* a, double* b, double* c) noexcept {
    storage_.vx = a; storage_.vy = b; storage_.vz = c;
    return *this;
}
ParticleInfo& ParticleInfo::forces(double* a, double* b, double* c) noexcept {
    storage_.fx = a; storage_.fy = b; storage_.fz = c;
    return *this;
}
ParticleInfo& ParticleInfo::properties(double* m, double* q, int* t, int* id) noexcept {
    storage_.mass = m; storage_.charge = q; storage_.type = t; storage_.global_id = id;
    return *this;
}

std::size_t ParticleInfo::capacity() const noexcept { return external_ ? storage_.count : x.size(); }
MemorySpace ParticleInfo::memory_space() const noexcept {
    return external_ ? storage_.memory_space : MemorySpace::Host;
}

double* ParticleInfo::x_data() noexcept { return external_ ? storage_.x : x.data(); }
double* ParticleInfo::y_data() noexcept { return external_ ? storage_.y : y.data(); }
double* ParticleInfo::z_data() noexcept { return external_ ? storage_.z : z.data(); }
double* ParticleInfo::vx_data() noexcept { return external_ ? storage_.vx : vx.data(); }
double* ParticleInfo::vy_data() noexcept { return external_ ? storage_.vy : vy.data(); }
double* ParticleInfo::vz_data() noexcept { return external_ ? storage_.vz : vz.data(); }
double* ParticleInfo::fx_data() noexcept { return external_ ? storage_.fx : fx.data(); }
double* ParticleInfo::fy_data() noexcept { return external_ ? storage_.fy : fy.data(); }
double* ParticleInfo::fz_data() noexcept { return external_ ? storage_.fz : fz.data(); }
double* ParticleInfo::mass_data() noexcept { return external_ ? storage_.mass : mass.data(); }
double* ParticleInfo::charge_data() noexcept { return external_ ? storage_.charge : charge.data(); }
int* ParticleInfo::type_data() noexcept { return external_ ? storage_.type : type.data(); }
int* ParticleInfo::global_id_data() noexcept { return external_ ? storage_.global_id : global_id.data(); }

void ParticleInfo::commit_counts(std::size_t owned, std::size_t ghosts) noexcept {
    owned_count_ = owned;
    ghost_count_ = ghosts;
}

void ParticleInfo::reset_counts(std::size_t owned, std::size_t ghosts) {
    const std::size_t total = owned + ghosts;
    if (read_view(total).count < total) invalid("particle storage is smaller than the supplied counts");
    commit_counts(owned, ghosts);
}

void ParticleInfo::resize(std::size_t count) {
    x.resize(count); y.resize(count); z.resize(count);
    vx.resize(count); vy.resize(count); vz.resize(count);
    fx.resize(count); fy.resize(count); fz.resize(count);
    mass.resize(count); charge.resize(count);
    type.resize(count); global_id.resize(count);
    num_particles = count;
}

ParticleView ParticleInfo::host_view(std::size_t count) {
    ParticleView v;
    v.memory_space = MemorySpace::Host;
    v.count = count;
    v.x = x.data(); v.y = y.data(); v.z = z.data();
    v.vx = vx.data(); v.vy = vy.data(); v.vz = vz.data();
    v.fx = fx.data(); v.fy = fy.data(); v.fz = fz.data();
    v.mass = mass.data(); v.charge = charge.data();
    v.type = type.data(); v.global_id = global_id.data();
    v.fields = fields_.empty() ? nullptr : fields_.data();
    v.field_count = fields_.size();
    return v;
}

ConstParticleView ParticleInfo::read_view(std::size_t count) const {
    if (external_) {
        if (storage_.count < count) invalid("external particle memory has insufficient capacity");
        return as_const_view(storage_);
    }
    return as_const_view(const_cast<ParticleInfo*>(this)->host_view(count));
}

void ParticleInfo::resize_owned(std::size_t count) {
    if (external_) {
        if (!owns_device_memory_) throw std::logic_error("dsDecompX: resize_owned cannot resize borrowed particle memory");
        resize_storage(count, std::min(count, owned_count_));
        commit_counts(count, 0);
        return;
    }
    for (const auto& f : fields_)
        if (f.capacity < count)
            throw std::length_error("dsDecompX: custom particle field '" + f.name + "' has insufficient capacity");
    resize(count);
    commit_counts(count, 0);
}

ParticleInfo& ParticleInfo::add_field_view(ParticleFieldView field) {
    if (field.name.empty() || !field.data || field.components == 0 || field.capacity < size())
        invalid("invalid or undersized custom particle field");
    for (const auto& f : fields_)
        if (f.name == field.name) invalid("duplicate custom particle field '" + field.name + "'");
    fields_.push_back(std::move(field));
    storage_.fields = fields_.data();
    storage_.field_count = fields_.size();
    return *this;
}

StorageResizeResult ParticleInfo::resize_storage(std::size_t required, std::size_t preserve) {
    for (const auto& f : fields_)
        if (f.capacity < required)
            throw std::length_error("dsDecompX: custom particle field '" + f.name + "' has insufficient capacity");
    if (!external_) {
        const double* old = x.data();
        resize(required);
        return {host_view(required), old != x.data()};
    }
    if (required <= storage_.count) return {storage_, false};
    if (owns_device_memory_) {
        const std::size_t grown = std::max(required, std::max<std::size_t>(64, storage_.count + storage_.count / 2));
        ParticleView next = allocate_device(storage_.memory_space, grown);
        try {
            copy_device(storage_, next, std::min(preserve, storage_.count));
        } catch (...) {
            free_device(next);
            throw;
        }
        free_device(storage_);
        storage_ = next;
        storage_.fields = fields_.empty() ? nullptr : fields_.data();
        storage_.field_count = fields_.size();
        return {storage_, true};
    }
    if (!provider_) throw std::length_error("dsDecompX: fixed external particle storage is too small");
    StorageResizeResult r = provider_->resize_particle_info(required, preserve);
    storage_ = r.view;
    storage_.fields = fields_.empty() ? nullptr : fields_.data();
    storage_.field_count = fields_.size();
    r.view = storage_;
    return r;
}

void ParticleInfo::reset_view(ParticleView storage) {
    if (storage.count < size()) invalid("replacement particle view is smaller than current particles");
    release_device_memory();
    external_ = true;
    owns_device_memory_ = false;
    provider_ = nullptr;
    storage_ = storage;
    fields_.clear();
    if (storage.fields && storage.field_count) {
        fields_.assign(storage.fields, storage.fields + storage.field_count);
        storage_.fields = fields_.data();
        storage_.field_count = fields_.size();
    }
}

// ----------------------------------------------------------------------- Decomp

struct Decomp::Impl {
    Config config;
    Topology topology;
    double halo_width = 0.0;
    std::size_t migration_calls = 0;
    bool rebalance_in_progress = false;
    bool perf_enabled = false;
    PerfStats stats;
    struct Pending {
        bool active = false;
        HaloExchangeOptions options;
        std::size_t owned = 0;
    } pending;

    void refresh_geometry() {
        auto& cuts = detail::TopologyAccess::axis_cuts(topology);
        auto& local = detail::TopologyAccess::local_domain(topology);
        for (int a = 0; a < 3; ++a) {
            local.lower[a] = cuts[static_cast<std::size_t>(a)][0];
            local.upper[a] = cuts[static_cast<std::size_t>(a)][1];
        }
        // one rank: every direction moves along an axis of extent 1, which the
        // reference skips (src/topology.cpp:118-127)
        detail::TopologyAccess::neighbors(topology).clear();
    }
};

Decomp::Decomp(MPI_Comm communicator, Config config) : impl_(std::make_unique<Impl>()) {
    if (communicator == MPI_COMM_NULL) invalid("MPI communicator is null");
    int size = 1;
    MPI_Comm_size(communicator, &size);
    if (size != 1)
        invalid("this drop-in handles one rank per process (a Decomp per GPU with its own box); "
                "several subdomains on one GPU are the virtual grid of dsx.h");
    if (config.execution != ExecutionMode::Cuda)
        invalid("this build implements ExecutionMode::Cuda (device or managed particle memory)");
    if (!(config.dynamic.imbalance_threshold >= 1.0) ||
        !(config.dynamic.relaxation > 0.0 && config.dynamic.relaxation <= 1.0) ||
        !(config.dynamic.minimum_cell_fraction > 0.0 && config.dynamic.minimum_cell_fraction <= 1.0))
        invalid("invalid dynamic load-balance configuration");
    if (config.grid_policy == GridPolicy::TopologyAware && !config.topology_info.available) {
        config.topology_info.available = true;
        config.topology_info.local_rank = 0;
        config.topology_info.local_size = 1;
        config.topology_info.node_count = 1;
        config.topology_info.rank_to_node = {0};
    }
    // CUDA device selection (src/runtime.cpp:149-231, one rank)
    {
        int count = 0;
        int error = cudaGetDeviceCount(&count) != cudaSuccess || count <= 0 ? 1 : 0;
        const int requested = config.advanced.cuda_device;
        if (!error && requested == kCudaDeviceByLocalRank) error = cudaSetDevice(0) != cudaSuccess;
        else if (!error && requested >= 0) error = requested >= count || cudaSetDevice(requested) != cudaSuccess;
        if (error)
            throw std::runtime_error("dsDecompX: could not select a CUDA device (no visible device, "
                                     "Config::advanced.cuda_device out of range, or cudaSetDevice failed)");
    }
    for (int a = 0; a < 3; ++a)
        if (!(config.domain.upper[a] > config.domain.lower[a])) invalid("global-domain extent must be positive");
    if (config.halo.width < 0.0) invalid("halo width cannot be negative");
    if (config.process_grid.allow_rank_reorder)
        invalid("dsDecompX CUDA execution currently requires allow_rank_reorder=false");
    Vec3i dims = config.process_grid.dimensions;
    if (config.grid_policy != GridPolicy::Manual) {
        DomainShape shape;
        for (int a = 0; a < 3; ++a) shape.lengths[a] = config.domain.upper[a] - config.domain.lower[a];
        shape.periodic = config.domain.periodic;
        dims = choose_process_grid(1, shape, config.topology_info, config.grid_policy).as_array();
    }
    for (int d : dims)
        if (d < 0) invalid("process-grid dimensions cannot be negative");
    for (int& d : dims) if (d == 0) d = 1;
    if (dims[0] * dims[1] * dims[2] != 1) invalid("process-grid dimensions do not match communicator size");
    Impl& m = *impl_;
    m.config = config;
    m.halo_width = config.halo.width;
    detail::TopologyAccess::rank(m.topology) = 0;
    detail::TopologyAccess::size(m.topology) = 1;
    detail::TopologyAccess::dimensions(m.topology) = {1, 1, 1};
    detail::TopologyAccess::coordinates(m.topology) = {0, 0, 0};
    auto& cuts = detail::TopologyAccess::axis_cuts(m.topology);
    for (int a = 0; a < 3; ++a) {
        const double extent = config.domain.upper[a] - config.domain.lower[a];
        cuts[static_cast<std::size_t>(a)] = {config.domain.lower[a] + extent * 0.0 / 1.0,
                                             config.domain.lower[a] + extent * 1.0 / 1.0};
    }
    m.refresh_geometry();
}

Decomp::~Decomp() = default;
Decomp::Decomp(Decomp&&) noexcept = default;
Decomp& Decomp::operator=(Decomp&&) noexcept = default;

const Topology& Decomp::topology() const noexcept { return impl_->topology; }
BackendKind Decomp::backend_kind() const noexcept { return BackendKind::Mpi; }
bool Decomp::mpi_takes_device_pointers() const noexcept { return false; }
int Decomp::owner_rank(const Vec3d&) const { return 0; }
bool Decomp::any_rank_true(bool local_flag) const { return local_flag; }
bool Decomp::has_out_of_domain_particles(const ParticleInfo&) const { return false; }

void Decomp::rescale_domain(const GlobalDomain& domain) {
    Impl& m = *impl_;
    if (domain.periodic != m.config.domain.periodic)
        invalid("changing periodicity after topology creation requires reconstructing Decomp");
    auto& cuts = detail::TopologyAccess::axis_cuts(m.topology);
    const GlobalDomain previous = m.config.domain;
    for (int a = 0; a < 3; ++a) {
        const double old_extent = previous.upper[a] - previous.lower[a];
        const double new_extent = domain.upper[a] - domain.lower[a];
        for (double& cut : cuts[static_cast<std::size_t>(a)]) {
            const double fraction = (cut - previous.lower[a]) / old_extent;
            cut = domain.lower[a] + fraction * new_extent;
        }
    }
    m.config.domain = domain;
    m.refresh_geometry();
}

void Decomp::update_domain(const GlobalDomain& domain) { rescale_domain(domain); }

void Decomp::set_halo_width(double width) {
    if (width < 0.0) invalid("halo width cannot be negative");
    impl_->config.halo.width = width;
    impl_->halo_width = width;
}

double Decomp::halo_width() const noexcept { return impl_->halo_width; }
void Decomp::invalidate_halo() noexcept {}

bool Decomp::can_refresh_halo(const ParticleInfo&) const { return false; }

void Decomp::begin_halo_exchange(ParticleInfo& particles, HaloExchangeOptions options) {
    Impl& m = *impl_;
    if (m.pending.active) throw std::logic_error("dsDecompX: a split-phase halo exchange is already in flight");
    const std::size_t owned = particles.owned_count();
    const ConstParticleView input = particles.read_view(owned);
    if (!device_space(input.memory_space))
        invalid("this build exchanges halos of CUDA particle memory (CudaDevice or CudaManaged)");
    (void)field_schema_hash(input);   // the collective schema check of one rank always agrees
    m.pending.active = true;
    m.pending.options = options;
    m.pending.owned = owned;
}

HaloResult Decomp::end_halo_exchange(ParticleInfo& particles) {
    Impl& m = *impl_;
    if (!m.pending.active)
        throw std::logic_error("dsDecompX: end_halo_exchange without a matching begin_halo_exchange");
    m.pending.active = false;
    const std::size_t owned = m.pending.owned;
    // one rank owns the whole periodic box: no ghosts (src/halo.cpp:325-350)
    const StorageResizeResult out = particles.resize_storage(owned, owned);
    if (out.view.count < owned) invalid("particle storage returned insufficient output capacity");
    const bool changed = m.pending.options.rebuild || particles.ghost_count() != 0;
    particles.commit_counts(owned, 0);
    if (m.perf_enabled) ++m.stats.halo_calls;
    return {0, changed, out.reallocated, false};
}

HaloResult Decomp::exchange_halo(ParticleInfo& particles, HaloExchangeOptions options) {
    begin_halo_exchange(particles, options);
    return end_halo_exchange(particles);
}

MigrationResult Decomp::migrate(ParticleInfo& particles, ExecutionStream stream) {
    Impl& m = *impl_;
    if (m.pending.active) throw std::logic_error("dsDecompX: migration cannot overlap an active halo operation");
    ++m.migration_calls;   // one rank: the Dynamic rebalance never moves a cut
    const std::size_t owned = particles.owned_count();
    const ConstParticleView in = particles.read_view(owned);
    if (!device_space(in.memory_space))
        invalid("this build migrates CUDA particle memory (CudaDevice or CudaManaged)");
    if (!stream) invalid("CUDA migration requires an explicit communication stream");
    if (owned && (!in.x || !in.y || !in.z || !in.vx || !in.vy || !in.vz || !in.fx || !in.fy || !in.fz ||
                  !in.mass || !in.charge || !in.type || !in.global_id))
        invalid("incomplete CUDA migration view");
    if (in.field_count > 16) invalid("at most 16 custom fields are supported on CUDA particle memory");
    std::unordered_set<std::string> names;
    for (std::size_t f = 0; f < in.field_count; ++f) {
        const auto& field = in.fields[f];
        if (field.name.empty() || !field.data || field.components == 0 || field.capacity < owned)
            invalid("invalid or undersized custom particle field");
        if (!names.insert(field.name).second) invalid("duplicate custom particle field '" + field.name + "'");
    }
    dsx_domain domain{};
    for (int a = 0; a < 3; ++a) {
        domain.lower[a] = m.config.domain.lower[a];
        domain.upper[a] = m.config.domain.upper[a];
        domain.periodic[a] = m.config.domain.periodic[a] ? 1 : 0;
    }
    dsx_migration_result r{};
    const int status = dsx_rank_migrate(const_cast<double*>(in.x), const_cast<double*>(in.y),
                                        const_cast<double*>(in.z), static_cast<long long>(owned), &domain,
                                        stream, &r);
    if (status != DSX_OK) {
        const std::string message = dsx_last_error();
        if (status == DSX_E_INVALID) throw std::invalid_argument(message);
        throw std::runtime_error(message);
    }
    MigrationResult result;
    result.ownership_changed = r.ownership_changed != 0;
    result.previous_owned_count = static_cast<std::size_t>(r.previous_owned_count);
    result.retained_count = static_cast<std::size_t>(r.retained_count);
    result.sent_count = static_cast<std::size_t>(r.sent_count);
    result.received_count = static_cast<std::size_t>(r.received_count);
    result.new_owned_count = static_cast<std::size_t>(r.new_owned_count);
    const StorageResizeResult out = particles.resize_storage(result.new_owned_count, 0);
    if (out.view.count < result.new_owned_count) invalid("particle storage returned insufficient output capacity");
    particles.commit_counts(result.new_owned_count, 0);
    if (m.perf_enabled) ++m.stats.migration_calls;
    return result;
}

RebalanceResult Decomp::rebalance(ParticleInfo& particles, RebalanceOptions options, ExecutionStream stream) {
    const double work = options.local_work >= 0.0 ? options.local_work : static_cast<double>(particles.owned_count());
    if (!std::isfinite(work) || work < 0.0) invalid("rebalance local_work must be finite and non-negative");
    RebalanceResult result;
    result.attempted = true;   // one rank: nothing to balance (src/runtime.cpp:378)
    impl_->rebalance_in_progress = true;
    try {
        result.migration = migrate(particles, stream);
    } catch (...) {
        impl_->rebalance_in_progress = false;
        throw;
    }
    impl_->rebalance_in_progress = false;
    return result;
}

void Decomp::reverse_halo(ParticleInfo& particles, ExecutionStream stream) {
    if (impl_->pending.active) throw std::logic_error("dsDecompX: reverse halo cannot overlap an active operation");
    const StorageResizeResult view = particles.resize_storage(particles.size(), particles.size());
    if (!device_space(view.view.memory_space))
        invalid("this build reverses halos of CUDA particle memory (CudaDevice or CudaManaged)");
    if (!stream) invalid("device reverse halo requires an explicit stream");
    if (view.view.count < particles.size() || !view.view.fx || !view.view.fy || !view.view.fz)
        invalid("invalid device reverse-halo view");
    // no ghosts on one rank: nothing returns to the owners (the Host path's semantics)
}

namespace {
const ParticleFieldView* find_field(const ParticleView& v, const std::string& name) {
    for (std::size_t f = 0; f < v.field_count; ++f)
        if (v.fields[f].name == name) return &v.fields[f];
    return nullptr;
}
}  // namespace

void Decomp::reverse_exchange(ParticleInfo& particles, const std::vector<ReverseExchangeField>& fields,
                              ExecutionStream stream) {
    if (impl_->pending.active) throw std::logic_error("dsDecompX: reverse exchange cannot overlap an active operation");
    const StorageResizeResult view = particles.resize_storage(particles.size(), particles.size());
    if (!device_space(view.view.memory_space))
        invalid("this build reverse-exchanges CUDA particle memory (CudaDevice or CudaManaged)");
    if (!stream) invalid("device reverse exchange requires an explicit stream");
    if (view.view.count < particles.size()) invalid("reverse exchange particle view is too small");
    if (fields.size() > 16) invalid("at most 16 fields can be reverse-exchanged on CUDA particle memory");
    std::unordered_set<std::string> seen;
    for (const auto& spec : fields) {
        if (!seen.insert(spec.name).second) invalid("duplicate reverse exchange field '" + spec.name + "'");
        const ParticleFieldView* f = find_field(view.view, spec.name);
        if (!f || !f->data || f->components == 0 || f->capacity < particles.size())
            invalid("missing or undersized reverse exchange field '" + spec.name + "'");
    }
}

void Decomp::forward_exchange(ParticleInfo& particles, const std::vector<std::string>& fields,
                              ExecutionStream stream) {
    if (impl_->pending.active) throw std::logic_error("dsDecompX: forward exchange cannot overlap an active operation");
    const StorageResizeResult view = particles.resize_storage(particles.size(), particles.size());
    if (!device_space(view.view.memory_space)) invalid("forward field exchange needs CUDA particle memory");
    if (!stream) invalid("device forward exchange requires an explicit stream");
    if (view.view.count < particles.size()) invalid("forward exchange particle view is too small");
    if (fields.size() > 16) invalid("at most 16 fields can be forward-exchanged on CUDA particle memory");
    std::unordered_set<std::string> seen;
    for (const auto& name : fields) {
        if (!seen.insert(name).second) invalid("duplicate forward exchange field '" + name + "'");
        const ParticleFieldView* f = find_field(view.view, name);
        if (!f || !f->data || f->components == 0 || f->capacity < particles.size())
            invalid("missing or undersized forward exchange field '" + name + "'");
        if (f->record_bytes() % 4 != 0)
            invalid("forward exchange field '" + name + "' must be a multiple of 4 bytes per particle");
    }
}

void Decomp::set_performance_counters_enabled(bool enabled, bool) noexcept { impl_->perf_enabled = enabled; }
PerfStats Decomp::get_stats() const { return impl_->stats; }
PerfStats Decomp::get_global_stats() const {
    PerfStats global = impl_->stats;
    global.neighbor_bytes.clear();
    return global;
}
void Decomp::reset_stats() noexcept { impl_->stats = {}; }

}  // namespace dsdecompx
