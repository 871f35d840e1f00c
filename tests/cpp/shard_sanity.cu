// The native sharded grid (include/dsx_shard.h): R shards as threads of one
// process on one GPU, their transport a host barrier plus device-to-device
// copies (no kernel ever waits on another shard), checked against one grid
// of all P subdomains: results and owned arrays after every migrate, ghost
// arrays after every halo build and refresh, owned forces after every
// reverse_halo, field values after a reverse and a forward field exchange,
// and every owned and ghost array after fused steps (dsx_shard_step) against
// the one grid's batched step; Manual cuts over 4 shards and Dynamic cuts
// over 2.
//
// usage: shard_sanity   (exits 0 and prints "shard_sanity: ok" when every
//                        check passed)
#include <dsx_shard.hpp>

#include <cuda_runtime_api.h>

#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <map>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

namespace {

int failures = 0;

void must(int status, const char* what) {
    if (status != DSX_OK) {
        std::fprintf(stderr, "FAILED %s: %s\n", what, dsx_last_error());
        std::_Exit(1);   // the other shards may be waiting in the transport
    }
}

void cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "FAILED %s: %s\n", what, cudaGetErrorString(e));
        std::_Exit(1);
    }
}

void expect(bool ok, const char* what, int t) {
    if (!ok) {
        std::fprintf(stderr, "FAILED: %s (subdomain %d)\n", what, t);
        ++failures;
    }
}

class Barrier {
public:
    explicit Barrier(int n) : n_(n) {}
    void wait() {
        std::unique_lock<std::mutex> lock(m_);
        const long gen = gen_;
        if (++count_ == n_) {
            count_ = 0;
            ++gen_;
            cv_.notify_all();
        } else {
            cv_.wait(lock, [&] { return gen_ != gen; });
        }
    }

private:
    std::mutex m_;
    std::condition_variable cv_;
    int n_, count_ = 0;
    long gen_ = 0;
};

struct Hub {
    explicit Hub(int r) : R(r), bar(r), li(r), ld(r), posted(r) {}
    int R;
    Barrier bar;
    std::vector<std::vector<long long>> li;
    std::vector<std::vector<double>> ld;
    std::vector<std::map<int, std::pair<const void*, long long>>> posted;
};

struct Ctx {
    Hub* hub;
    int me;
};

template <class T>
int allreduce(Ctx* c, std::vector<std::vector<T>>& slot, T* v, long long n) {
    Hub* h = c->hub;
    slot[c->me].assign(v, v + n);
    h->bar.wait();
    for (long long k = 0; k < n; ++k) {
        T s = 0;
        for (int r = 0; r < h->R; ++r) s += slot[r][k];   // every shard adds in shard order
        v[k] = s;
    }
    h->bar.wait();
    return DSX_OK;
}

int allreduce_i64(void* u, long long* v, long long n) {
    Ctx* c = static_cast<Ctx*>(u);
    return allreduce(c, c->hub->li, v, n);
}

int allreduce_f64(void* u, double* v, long long n) {
    Ctx* c = static_cast<Ctx*>(u);
    return allreduce(c, c->hub->ld, v, n);
}

int exchange(void* u, int nsend, const int* to, const void* const* send, const long long* send_bytes,
             int nrecv, const int* from, void* const* recv, const long long* recv_bytes, void* stream) {
    Ctx* c = static_cast<Ctx*>(u);
    Hub* h = c->hub;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cuda(cudaStreamSynchronize(s), "send buffers");
    h->posted[c->me].clear();
    for (int k = 0; k < nsend; ++k) h->posted[c->me][to[k]] = {send[k], send_bytes[k]};
    h->bar.wait();
    int status = DSX_OK;
    for (int k = 0; k < nrecv; ++k) {
        const auto& box = h->posted[from[k]];
        const auto it = box.find(c->me);
        if (it == box.end() || it->second.second != recv_bytes[k]) {
            status = DSX_E_RUNTIME;
            continue;
        }
        cuda(cudaMemcpyAsync(recv[k], it->second.first, recv_bytes[k], cudaMemcpyDeviceToDevice, s), "receive");
    }
    cuda(cudaStreamSynchronize(s), "receive");
    h->bar.wait();   // the senders' buffers are free again
    return status;
}

// The step callback of the fused-step checks: every ghost of the view
// (halo_totals[0] of them from the ghost offset) gets a force computed from
// its own id and position, so that equal ghosts get equal forces whatever
// slot they sit in.
__global__ void k_forces_from_ghosts(const double* x, const double* y, const int* id, const int* n,
                                     double* fx, double* fy, double* fz) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n[0]; i += gridDim.x * blockDim.x) {
        const double a = static_cast<double>(id[i] % 1009) * 0.001;
        fx[i] = x[i] * 0.5 + a;
        fy[i] = y[i] * 0.25 - a;
        fz[i] = a * a + 1.0;
    }
}

void forces_callback(void*, void* stream, const dsx_grid_view* v) {
    const long long g = v->ghost_offset;
    k_forces_from_ghosts<<<148, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double*>(v->base[0]) + g, static_cast<const double*>(v->base[1]) + g,
        static_cast<const int*>(v->base[12]) + g, v->halo_totals,
        static_cast<double*>(v->base[6]) + g, static_cast<double*>(v->base[7]) + g,
        static_cast<double*>(v->base[8]) + g);
}

// every shard runs `call` on its own thread
void on_shards(int R, const std::function<void(int)>& call) {
    std::vector<std::thread> th;
    for (int r = 0; r < R; ++r) th.emplace_back(call, r);
    for (auto& t : th) t.join();
}

std::uint64_t mix(std::uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double unit(std::uint64_t k) { return static_cast<double>(mix(k) >> 11) * (1.0 / 9007199254740992.0); }

// 13 core arrays + "tag" (int64), "vec" (float32 x 3), "u" (uint32), "wide" (float64 x 7)
constexpr int kArrays = 17;
const int kBytes[kArrays] = {8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 4, 4, 8, 12, 4, 56};

struct Case {
    const char* name;
    dsx_grid_desc desc;
    int R;
    long long N;
};

// the host arrays of subdomain t of the one grid: owned then ghosts
std::vector<std::vector<unsigned char>> read_ref(dsx_grid* g, int t, long long start, long long n) {
    std::vector<std::vector<unsigned char>> out(kArrays);
    for (int a = 0; a < kArrays; ++a) {
        out[a].resize(static_cast<std::size_t>(n * kBytes[a]));
        if (n) must(dsx_grid_read(g, t, a, start, n, out[a].data(), nullptr), "read");
    }
    return out;
}

// subdomain t of a shard: owned records (from the owned view) or assembled
// ghosts (from the ghost view)
std::vector<std::vector<unsigned char>> read_shard(dsx_shard* sh, int P, int t, bool ghosts) {
    std::vector<long long> o(P), g(P);
    must(dsx_shard_counts(sh, o.data(), g.data(), nullptr), "counts");
    dsx_grid_view v{};
    must(ghosts ? dsx_shard_ghost_view(sh, &v) : dsx_shard_owned_view(sh, &v), "view");
    const std::vector<long long>& c = ghosts ? g : o;
    long long base = 0;
    for (int u = 0; u < t; ++u) base += c[u];
    const long long off = ghosts ? 0 : v.owned_offset;
    std::vector<std::vector<unsigned char>> out(kArrays);
    for (int a = 0; a < kArrays; ++a) {
        out[a].resize(static_cast<std::size_t>(c[t] * kBytes[a]));
        if (c[t])
            cuda(cudaMemcpy(out[a].data(), static_cast<unsigned char*>(v.base[a]) + (off + base) * kBytes[a],
                            out[a].size(), cudaMemcpyDeviceToHost), "read shard");
    }
    return out;
}

void write_shard(dsx_shard* sh, int P, int t, bool ghosts, int a, const void* data) {
    std::vector<long long> o(P), g(P);
    must(dsx_shard_counts(sh, o.data(), g.data(), nullptr), "counts");
    dsx_grid_view v{};
    must(ghosts ? dsx_shard_ghost_view(sh, &v) : dsx_shard_owned_view(sh, &v), "view");
    const std::vector<long long>& c = ghosts ? g : o;
    long long base = 0;
    for (int u = 0; u < t; ++u) base += c[u];
    const long long off = ghosts ? 0 : v.owned_offset;
    if (c[t])
        cuda(cudaMemcpy(static_cast<unsigned char*>(v.base[a]) + (off + base) * kBytes[a], data,
                        static_cast<std::size_t>(c[t] * kBytes[a]), cudaMemcpyHostToDevice), "write shard");
}

// ghosts of subdomain t after a fused step: the shard grid's own ghost block
std::vector<std::vector<unsigned char>> read_step_ghosts(dsx_shard* sh, int P, int t) {
    std::vector<long long> o(P), g(P);
    must(dsx_shard_counts(sh, o.data(), g.data(), nullptr), "counts");
    dsx_grid_view v{};
    must(dsx_shard_owned_view(sh, &v), "view");
    std::vector<int> gb(P + 1);
    cuda(cudaMemcpy(gb.data(), v.gbase, sizeof(int) * (P + 1), cudaMemcpyDeviceToHost), "gbase");
    std::vector<std::vector<unsigned char>> out(kArrays);
    for (int a = 0; a < kArrays; ++a) {
        out[a].resize(static_cast<std::size_t>(g[t] * kBytes[a]));
        if (g[t])
            cuda(cudaMemcpy(out[a].data(),
                            static_cast<unsigned char*>(v.base[a]) + (v.ghost_offset + gb[t]) * kBytes[a],
                            out[a].size(), cudaMemcpyDeviceToHost), "read ghosts");
    }
    return out;
}

void run(const Case& cs) {
    const int P = cs.desc.nranks, R = cs.R;
    const dsx_field_desc fields[4] = {{"tag", DSX_INT64, 1}, {"vec", DSX_FLOAT32, 3},
                                      {"u", DSX_UINT32, 1}, {"wide", DSX_FLOAT64, 7}};
    dsx_grid* ref = nullptr;
    must(dsx_grid_create(&cs.desc, fields, 4, cs.N, 0, &ref), "create grid");
    // every particle starts in subdomain 0 of a Manual grid with the same
    // process grid, whose migrate places them (so that the grids under test
    // start with the same cuts and no migrate behind them)
    dsx_grid_desc place = cs.desc;
    {
        int count = 0, info[26 * 5];
        double shifts[26 * 3];
        must(dsx_plan_topology(&cs.desc, 0, place.dims, &count, info, shifts), "plan");
        place.policy = DSX_MANUAL;
    }
    dsx_grid* placer = nullptr;
    must(dsx_grid_create(&place, fields, 4, cs.N, 0, &placer), "create placer");
    {
        std::vector<std::vector<unsigned char>> host(kArrays);
        for (int a = 0; a < kArrays; ++a) host[a].resize(static_cast<std::size_t>(cs.N * kBytes[a]));
        for (long long i = 0; i < cs.N; ++i) {
            for (int a = 0; a < 3; ++a) {
                const double v = cs.desc.lower[a] + (cs.desc.upper[a] - cs.desc.lower[a]) * unit(3 * i + a);
                std::memcpy(&host[a][i * 8], &v, 8);
            }
            for (int a = 3; a < 11; ++a) {
                const double v = unit(1000003 * a + i) - 0.5;
                std::memcpy(&host[a][i * 8], &v, 8);
            }
            const int ty = static_cast<int>(i % 5), id = static_cast<int>(i);
            const long long tag = 7 * i + 1;
            const float vec[3] = {static_cast<float>(i), 0.5f * static_cast<float>(i), -1.0f};
            std::memcpy(&host[11][i * 4], &ty, 4);
            std::memcpy(&host[12][i * 4], &id, 4);
            std::memcpy(&host[13][i * 8], &tag, 8);
            std::memcpy(&host[14][i * 12], vec, 12);
            const unsigned u = static_cast<unsigned>(i) * 2654435761u;
            std::memcpy(&host[15][i * 4], &u, 4);
            for (int k = 0; k < 7; ++k) {
                const double wv = std::sin(0.01 * static_cast<double>(i) + k);
                std::memcpy(&host[16][i * 56 + 8 * k], &wv, 8);
            }
        }
        std::vector<long long> counts(P, 0);
        counts[0] = cs.N;
        std::vector<const void*> ptrs(kArrays);
        for (int a = 0; a < kArrays; ++a) ptrs[a] = host[a].data();
        must(dsx_grid_upload(placer, counts.data(), ptrs.data(), nullptr), "upload");
        must(dsx_grid_migrate(placer, nullptr, nullptr), "placing migrate");
        std::vector<long long> o(P), g(P);
        must(dsx_grid_counts(placer, o.data(), g.data(), nullptr), "counts");
        std::vector<std::vector<unsigned char>> all(kArrays);
        for (int t = 0; t < P; ++t) {
            const auto part = read_ref(placer, t, 0, o[t]);
            for (int a = 0; a < kArrays; ++a) all[a].insert(all[a].end(), part[a].begin(), part[a].end());
        }
        for (int a = 0; a < kArrays; ++a) ptrs[a] = all[a].data();
        must(dsx_grid_upload(ref, o.data(), ptrs.data(), nullptr), "upload");
    }
    dsx_grid_destroy(placer);
    Hub hub(R);
    std::vector<Ctx> ctx(R);
    std::vector<dsx_shard*> shards(R, nullptr);
    std::vector<cudaStream_t> streams(R);
    for (int r = 0; r < R; ++r) {
        ctx[r] = {&hub, r};
        dsx_transport tr{&ctx[r], allreduce_i64, allreduce_f64, exchange};
        must(dsx_shard_create(&cs.desc, fields, 4, cs.N, 0, r, R, nullptr, &tr, &shards[r]), "create shard");
        cuda(cudaStreamCreate(&streams[r]), "stream");
    }
    std::vector<int> owners(P);
    must(dsx_shard_owners(shards[0], owners.data()), "owners");
    {
        // a shard created without owners takes the host-side plan
        std::vector<int> planned(P);
        must(dsx_shard_plan_owners(place.dims, R, planned.data()), "plan owners");
        for (int t = 0; t < P; ++t) expect(planned[t] == owners[t], "planned owners", t);
    }
    // each shard uploads its subdomains' particles as the one grid holds them
    {
        std::vector<long long> o(P), g(P);
        must(dsx_grid_counts(ref, o.data(), g.data(), nullptr), "counts");
        for (int r = 0; r < R; ++r) {
            std::vector<long long> counts(P, 0);
            std::vector<std::vector<unsigned char>> host(kArrays);
            for (int t = 0; t < P; ++t) {
                if (owners[t] != r) continue;
                counts[t] = o[t];
                const auto part = read_ref(ref, t, 0, o[t]);
                for (int a = 0; a < kArrays; ++a) host[a].insert(host[a].end(), part[a].begin(), part[a].end());
            }
            std::vector<const void*> ptrs(kArrays);
            for (int a = 0; a < kArrays; ++a) ptrs[a] = host[a].empty() ? nullptr : host[a].data();
            must(dsx_shard_upload(shards[r], counts.data(), ptrs.data(), nullptr), "shard upload");
        }
    }
    auto displace = [&](int step, double sigma) {
        std::vector<long long> o(P), g(P);
        must(dsx_grid_counts(ref, o.data(), g.data(), nullptr), "counts");
        for (int t = 0; t < P; ++t) {
            const auto part = read_ref(ref, t, 0, o[t]);
            for (int a = 0; a < 3; ++a) {
                std::vector<double> x(o[t]);
                std::memcpy(x.data(), part[a].data(), x.size() * 8);
                for (long long i = 0; i < o[t]; ++i) {
                    int id;
                    std::memcpy(&id, &part[12][i * 4], 4);
                    x[i] += sigma * (unit(1000 * step + 3 * static_cast<std::uint64_t>(id) + a) - 0.5);
                }
                if (o[t]) must(dsx_grid_write(ref, t, a, 0, o[t], x.data(), nullptr), "write");
                write_shard(shards[owners[t]], P, t, false, a, x.data());
            }
        }
    };
    auto compare = [&](const char* what, bool ghosts) {
        std::vector<long long> o(P), g(P);
        must(dsx_grid_counts(ref, o.data(), g.data(), nullptr), "counts");
        for (int t = 0; t < P; ++t) {
            dsx_shard* sh = shards[owners[t]];
            std::vector<long long> so(P), sg(P);
            must(dsx_shard_counts(sh, so.data(), sg.data(), nullptr), "counts");
            expect(so[t] == o[t], what, t);
            if (ghosts) expect(sg[t] == g[t], what, t);
            const auto want = read_ref(ref, t, ghosts ? o[t] : 0, ghosts ? g[t] : o[t]);
            const auto got = read_shard(sh, P, t, ghosts);
            for (int a = 0; a < kArrays; ++a) expect(want[a] == got[a], what, t);
        }
    };
    for (int step = 0; step < 3; ++step) {
        displace(step, 1.2);
        std::vector<long long> mr(6 * P);
        must(dsx_grid_migrate(ref, nullptr, mr.data()), "migrate");
        std::vector<std::vector<long long>> ms(R, std::vector<long long>(6 * P));
        on_shards(R, [&](int r) { must(dsx_shard_migrate(shards[r], streams[r], ms[r].data()), "shard migrate"); });
        for (int t = 0; t < P; ++t)
            for (int k = 0; k < 6; ++k) expect(ms[owners[t]][6 * t + k] == mr[6 * t + k], "migrate results", t);
        compare("owned after migrate", false);

        std::vector<long long> hr(4 * P);
        must(dsx_grid_exchange_halo(ref, 1, 0, nullptr, hr.data()), "halo");
        std::vector<std::vector<long long>> hs(R, std::vector<long long>(4 * P));
        on_shards(R, [&](int r) { must(dsx_shard_exchange_halo(shards[r], 1, 0, streams[r], hs[r].data()), "shard halo"); });
        for (int t = 0; t < P; ++t)
            for (int k = 0; k < 2; ++k) expect(hs[owners[t]][4 * t + k] == hr[4 * t + k], "halo results", t);
        compare("ghosts after the build", true);

        // ghost forces and field values keyed by (ghost id, receiver)
        {
            std::vector<long long> o(P), g(P);
            must(dsx_grid_counts(ref, o.data(), g.data(), nullptr), "counts");
            for (int t = 0; t < P; ++t) {
                const auto gh = read_ref(ref, t, o[t], g[t]);
                std::vector<double> f(g[t]);
                std::vector<long long> tag(g[t]);
                for (int a = 6; a < 9; ++a) {
                    for (long long i = 0; i < g[t]; ++i) {
                        int id;
                        std::memcpy(&id, &gh[12][i * 4], 4);
                        f[i] = std::sin(0.37 * id + t + a);
                        tag[i] = 1000LL * id + t;
                    }
                    if (g[t]) must(dsx_grid_write(ref, t, a, o[t], g[t], f.data(), nullptr), "write");
                    write_shard(shards[owners[t]], P, t, true, a, f.data());
                }
                if (g[t]) must(dsx_grid_write(ref, t, 13, o[t], g[t], tag.data(), nullptr), "write");
                write_shard(shards[owners[t]], P, t, true, 13, tag.data());
                std::vector<unsigned> u(g[t]);
                std::vector<double> wide(7 * g[t]);
                for (long long i = 0; i < g[t]; ++i) {
                    int id;
                    std::memcpy(&id, &gh[12][i * 4], 4);
                    u[i] = static_cast<unsigned>(31 * id + t);
                    for (int k = 0; k < 7; ++k) wide[7 * i + k] = std::sin(0.1 * id + t + k);
                }
                if (g[t]) must(dsx_grid_write(ref, t, 15, o[t], g[t], u.data(), nullptr), "write");
                write_shard(shards[owners[t]], P, t, true, 15, u.data());
                if (g[t]) must(dsx_grid_write(ref, t, 16, o[t], g[t], wide.data(), nullptr), "write");
                write_shard(shards[owners[t]], P, t, true, 16, wide.data());
            }
        }
        must(dsx_grid_reverse_halo(ref, nullptr), "reverse");
        on_shards(R, [&](int r) { must(dsx_shard_reverse_halo(shards[r], streams[r]), "shard reverse"); });
        const int ids[3] = {0, 2, 3}, ops[3] = {step % 4, (step + 1) % 4, (step + 2) % 4};
        must(dsx_grid_reverse_exchange(ref, 3, ids, ops, nullptr), "reverse fields");
        on_shards(R, [&](int r) {
            must(dsx_shard_reverse_exchange(shards[r], 3, ids, ops, streams[r]), "shard reverse fields");
        });
        compare("owned after the reverse sums", false);
        const int all[4] = {3, 2, 1, 0};
        must(dsx_grid_forward_exchange(ref, 4, all, nullptr), "forward fields");
        on_shards(R, [&](int r) { must(dsx_shard_forward_exchange(shards[r], 4, all, streams[r]), "shard forward"); });
        compare("ghosts after the forward exchange", true);

        displace(step + 100, 0.05);
        must(dsx_grid_exchange_halo(ref, 0, 0, nullptr, nullptr), "refresh");
        on_shards(R, [&](int r) { must(dsx_shard_exchange_halo(shards[r], 0, 0, streams[r], nullptr), "shard refresh"); });
        compare("ghosts after the refresh", true);
    }
    // a positions-only refresh (the ghosts' positions follow, the rest stays
    // as both grids left it), then Decomp::rebalance with work per subdomain
    displace(500, 0.05);
    must(dsx_grid_exchange_halo(ref, 0, 1, nullptr, nullptr), "positions refresh");
    on_shards(R, [&](int r) { must(dsx_shard_exchange_halo(shards[r], 0, 1, streams[r], nullptr), "shard positions"); });
    compare("ghosts after the positions refresh", true);
    {
        std::vector<double> work(P);
        for (int t = 0; t < P; ++t) work[t] = 100.0 + 37.0 * ((t * 7) % P);
        std::vector<long long> fr(3 * P);
        std::vector<double> imb(P);
        must(dsx_grid_rebalance(ref, work.data(), 1, nullptr, fr.data(), imb.data()), "rebalance");
        std::vector<std::vector<long long>> fs(R, std::vector<long long>(3 * P));
        std::vector<double> is(R);
        on_shards(R, [&](int r) {
            must(dsx_shard_rebalance(shards[r], work.data(), 1, streams[r], fs[r].data(), &is[r]), "shard rebalance");
        });
        for (int t = 0; t < P; ++t)
            for (int k = 0; k < 3; ++k) expect(fs[owners[t]][3 * t + k] == fr[3 * t + k], "rebalance results", t);
        for (int r = 0; r < R; ++r) expect(is[r] == imb[0], "rebalance imbalance", r);
        compare("owned after the rebalance", false);
        must(dsx_grid_exchange_halo(ref, 1, 0, nullptr, nullptr), "halo");
        on_shards(R, [&](int r) { must(dsx_shard_exchange_halo(shards[r], 1, 0, streams[r], nullptr), "shard halo"); });
        compare("ghosts after the rebalance", true);
    }
    // the fused step (dsx_shard_step) against the one grid's batched step:
    // owned arrays (forces summed back included) and every ghost array
    for (int step = 0; step < 3; ++step) {
        displace(step + 200, 1.2);
        unsigned st = 0;
        must(dsx_grid_step(ref, forces_callback, nullptr, 0, nullptr, &st), "grid step");
        expect(st == 0, "grid step status", 0);
        std::vector<unsigned> ss(R, 0);
        on_shards(R, [&](int r) {
            must(dsx_shard_step(shards[r], forces_callback, nullptr, streams[r], &ss[r]), "shard step");
        });
        for (int r = 0; r < R; ++r) expect(ss[r] == 0, "shard step status", r);
        compare("owned after the fused step", false);
        std::vector<long long> o(P), g(P);
        must(dsx_grid_counts(ref, o.data(), g.data(), nullptr), "counts");
        for (int t = 0; t < P; ++t) {
            dsx_shard* sh = shards[owners[t]];
            std::vector<long long> so(P), sg(P);
            must(dsx_shard_counts(sh, so.data(), sg.data(), nullptr), "counts");
            expect(sg[t] == g[t], "ghost count after the fused step", t);
            const auto want = read_ref(ref, t, o[t], g[t]);
            const auto got = read_step_ghosts(sh, P, t);
            for (int a = 0; a < kArrays; ++a) expect(want[a] == got[a], "ghosts after the fused step", t);
        }
    }
    // the per-call calls go on from the fused step (a rebuild first)
    displace(300, 0.4);
    {
        std::vector<long long> mr(6 * P);
        must(dsx_grid_migrate(ref, nullptr, mr.data()), "migrate");
        on_shards(R, [&](int r) { must(dsx_shard_migrate(shards[r], streams[r], nullptr), "shard migrate"); });
        compare("owned after a migrate that follows the fused step", false);
        must(dsx_grid_exchange_halo(ref, 1, 0, nullptr, nullptr), "halo");
        on_shards(R, [&](int r) { must(dsx_shard_exchange_halo(shards[r], 1, 0, streams[r], nullptr), "shard halo"); });
        compare("ghosts after a rebuild that follows the fused step", true);
    }
    for (int r = 0; r < R; ++r) {
        dsx_shard_destroy(shards[r]);
        cudaStreamDestroy(streams[r]);
    }
    dsx_grid_destroy(ref);
    std::printf("%s: %s\n", cs.name, failures ? "FAILED" : "ok");
}

dsx_grid_desc desc(int P, int d0, int d1, int d2, int policy, double L);

// Shard 1 can hold 10 particles; migration would give it about half of
// them: both shards' migrate calls fail at the same collective, before any
// particle moves (neither waits in an exchange), and the C++ face
// (dsx_shard.hpp) raises std::length_error on both.
void shortfall() {
    const dsx_grid_desc d = desc(8, 2, 2, 2, DSX_MANUAL, 10.0);
    const long long N = 4000;
    Hub hub(2);
    std::vector<Ctx> ctx(2);
    std::vector<std::unique_ptr<dsx::ShardedGrid>> shards;
    for (int r = 0; r < 2; ++r) {
        ctx[r] = {&hub, r};
        Ctx* c = &ctx[r];
        dsx::Transport tr;
        tr.sum_i64 = [c](long long* v, long long n) { allreduce(c, c->hub->li, v, n); };
        tr.sum_f64 = [c](double* v, long long n) { allreduce(c, c->hub->ld, v, n); };
        tr.messages = [c](const std::vector<dsx::Message>& out, const std::vector<dsx::Message>& in,
                          void* stream) {
            std::vector<int> to, from;
            std::vector<const void*> sb;
            std::vector<void*> rb;
            std::vector<long long> sn, rn;
            for (const auto& m : out) {
                to.push_back(m.peer);
                sb.push_back(m.data);
                sn.push_back(m.bytes);
            }
            for (const auto& m : in) {
                from.push_back(m.peer);
                rb.push_back(m.data);
                rn.push_back(m.bytes);
            }
            if (exchange(c, static_cast<int>(to.size()), to.data(), sb.data(), sn.data(),
                         static_cast<int>(from.size()), from.data(), rb.data(), rn.data(), stream) != DSX_OK)
                throw std::runtime_error("exchange");
        };
        shards.push_back(std::make_unique<dsx::ShardedGrid>(d, std::vector<dsx::FieldSpec>{},
                                                            r == 0 ? N : 10, r, 2, tr));
    }
    const std::vector<int> owners = shards[0]->owners();
    if (dsx::ShardedGrid::plan_owners({2, 2, 2}, 2) != owners) expect(false, "planned owners (C++)", 0);
    int first = 0;
    while (owners[first] != 0) ++first;
    std::vector<double> x(N), y(N), z(N);
    std::vector<int> id(N);
    for (long long i = 0; i < N; ++i) {
        x[i] = 10.0 * unit(7 * i);
        y[i] = 10.0 * unit(7 * i + 1);
        z[i] = 10.0 * unit(7 * i + 2);
        id[i] = static_cast<int>(i);
    }
    std::vector<const void*> ptrs(13, nullptr);
    ptrs[0] = x.data();
    ptrs[1] = y.data();
    ptrs[2] = z.data();
    ptrs[12] = id.data();
    std::vector<long long> counts(8, 0);
    counts[first] = N;   // every particle in one subdomain of shard 0
    shards[0]->upload(counts, ptrs);
    counts[first] = 0;
    shards[1]->upload(counts, ptrs);
    std::vector<int> caught(2, 0);
    on_shards(2, [&](int r) {
        try {
            shards[r]->migrate();
        } catch (const std::length_error&) {
            caught[r] = 1;
        } catch (...) {
            caught[r] = 2;
        }
    });
    const bool ok = caught[0] == 1 && caught[1] == 1;
    expect(ok, "both shards raise length_error on a shortfall", 0);
    std::printf("storage shortfall: %s\n", ok ? "ok" : "FAILED");
}

dsx_grid_desc desc(int P, int d0, int d1, int d2, int policy, double L) {
    dsx_grid_desc d{};
    d.nranks = P;
    d.dims[0] = d0;
    d.dims[1] = d1;
    d.dims[2] = d2;
    d.policy = policy;
    for (int a = 0; a < 3; ++a) {
        d.lower[a] = 0.0;
        d.upper[a] = L;
        d.periodic[a] = 1;
    }
    d.halo_width = 1.0;
    d.edges_and_corners = 1;
    d.dyn_interval = 1.0;
    d.dyn_threshold = 1.05;
    d.dyn_relaxation = 0.5;
    d.dyn_min_fraction = 0.10;
    return d;
}

}  // namespace

int main() {
    run({"manual 4x4x2 over 4 shards", desc(32, 4, 4, 2, DSX_MANUAL, 16.0), 4, 60000});
    run({"dynamic 2x2x2 over 2 shards", desc(8, 0, 0, 0, DSX_DYNAMIC, 12.0), 2, 30000});
    shortfall();
    if (failures) return 1;
    std::printf("shard_sanity: ok\n");
    return 0;
}
