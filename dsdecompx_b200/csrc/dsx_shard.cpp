// Sharded virtual grid (include/dsx_shard.h): a grid of all P subdomains per
// process holding only this shard's block, one exchange step per collective
// call, and the assembly of this shard's subdomains in the reference's
// order.  Built on the public grid calls of dsx.h only; the same protocol as
// dsdecompx_b200/sharded.py (which serves it from Python).
//
// Orders (dsDecompX):
//   owned particles of t: retained, then the immigrants of every source
//     subdomain q in ascending q (src/migration.cpp:458-518);
//   ghosts of receiver t: its neighbor blocks m in order, block m the list
//     its neighbor sends toward -d_m, in the sender's owned order
//     (src/halo.cpp:609-649, src/runtime.cpp:951-957);
//   reverse sums: every owner's images in neighbor order (src/halo.cpp:956-1040),
//     which the local grid's own reverse keeps once each image's value is back
//     in the local slot of its list.
#include "dsx_shard.h"

#include "dsx_errors.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

constexpr int kNeighbors = 26;   // send lists per subdomain
constexpr int kArraySlots = 32;  // address table entries per source of dsx_grid_assemble

struct Error {
    int code;
    std::string message;   // empty: the failed grid call's message stands
};

void check(int status) {
    if (status != DSX_OK) throw Error{status, ""};
}

[[noreturn]] void fail(int code, const std::string& message) {
    throw Error{code, "dsDecompX: " + message};
}

void cuda(cudaError_t status, const char* what) {
    if (status != cudaSuccess) fail(DSX_E_RUNTIME, std::string(what) + ": " + cudaGetErrorString(status));
}

template <class F>
int guarded(F&& body) {
    try {
        body();
        return DSX_OK;
    } catch (const Error& e) {
        if (!e.message.empty()) dsx::set_last_error(e.message.c_str());
        return e.code;
    } catch (const std::bad_alloc&) {
        dsx::set_last_error("dsDecompX: host allocation failed");
        return DSX_E_LENGTH;
    } catch (const std::exception& e) {
        dsx::set_last_error((std::string("dsDecompX: ") + e.what()).c_str());
        return DSX_E_RUNTIME;
    }
}

long long align16(long long bytes) { return (bytes + 15) / 16 * 16; }

// A device buffer that only grows.
struct DeviceBuffer {
    void* data = nullptr;
    long long capacity = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { cudaFree(data); }
    void* ensure(long long bytes) {
        if (bytes > capacity) {
            cudaFree(data);
            data = nullptr;
            capacity = 0;
            cuda(cudaMalloc(&data, static_cast<std::size_t>(bytes)), "cudaMalloc message buffer");
            capacity = bytes;
        }
        return data;
    }
};

// (source index, destination index, count) rows; add() merges a row that
// continues the previous one in both source and destination.
struct Rows {
    std::vector<long long> src, dst, n;
    void add(long long s, long long d, long long c) {
        if (c <= 0) return;
        if (!n.empty() && src.back() + n.back() == s && dst.back() + n.back() == d) {
            n.back() += c;
            return;
        }
        src.push_back(s);
        dst.push_back(d);
        n.push_back(c);
    }
    bool empty() const { return n.empty(); }
};

}  // namespace

struct dsx_shard {
    dsx_grid* grid = nullptr;
    int P = 0, shard = 0, nshards = 1;
    dsx_transport tr{};
    bool dynamic = false;
    int dims[3] = {1, 1, 1};
    std::vector<int> owners, mine, nn;
    std::vector<long long> sender_of;   // [P * 26]: receiver t's block m -> entry q * 26 + n, or -1
    std::vector<int> bytes;             // bytes per record of every array (13 core + fields)

    // ghost plan of this shard's receivers
    bool planned = false;
    std::vector<long long> g, gbase;
    long long total = 0;
    Rows local;                              // engine ghost slot -> assembled slot
    std::map<int, Rows> recv, send;          // buffer offset -> assembled slot; engine slot -> buffer offset
    std::map<int, long long> recv_n, send_n;

    // the assembled ghost region and its view tables
    std::vector<void*> assembled;
    long long assembled_cap = 0;
    int* d_g = nullptr;        // [P]
    int* d_gbase = nullptr;    // [P + 1]
    int* d_totals = nullptr;   // {ghosts, 0}

    std::map<int, std::unique_ptr<DeviceBuffer>> sendbuf, recvbuf;
    long long launches = 0;   // kernels of this library launched for this shard
    long long capacity = 0;   // owned particles the local grid can hold

    ~dsx_shard() {
        for (void* p : assembled) cudaFree(p);
        cudaFree(d_g);
        cudaFree(d_gbase);
        cudaFree(d_totals);
        if (grid) dsx_grid_destroy(grid);
    }

    int narrays() const { return static_cast<int>(bytes.size()); }

    std::vector<int> all_arrays() const {
        std::vector<int> a(bytes.size());
        for (std::size_t k = 0; k < a.size(); ++k) a[k] = static_cast<int>(k);
        return a;
    }

    long long packed_bytes(long long n, const std::vector<int>& arrays) const {
        long long b = 0;
        for (int a : arrays) b += align16(n * bytes[static_cast<std::size_t>(a)]);
        return b;
    }

    // address of element 0 of every listed array in a packed buffer of n records
    std::vector<unsigned char*> sections(void* buffer, long long n, const std::vector<int>& arrays) const {
        std::vector<unsigned char*> out;
        long long at = 0;
        for (int a : arrays) {
            out.push_back(static_cast<unsigned char*>(buffer) + at);
            at += align16(n * bytes[static_cast<std::size_t>(a)]);
        }
        return out;
    }

    dsx_grid_view view() const {
        dsx_grid_view v{};
        check(dsx_grid_view_get(grid, &v));
        return v;
    }

    std::vector<unsigned char*> owned_bases(const std::vector<int>& arrays) const {
        const dsx_grid_view v = view();
        std::vector<unsigned char*> out;
        for (int a : arrays)
            out.push_back(static_cast<unsigned char*>(v.base[a]) + v.owned_offset * bytes[static_cast<std::size_t>(a)]);
        return out;
    }

    std::vector<unsigned char*> ghost_bases(const std::vector<int>& arrays) const {
        const dsx_grid_view v = view();
        std::vector<unsigned char*> out;
        for (int a : arrays)
            out.push_back(static_cast<unsigned char*>(v.base[a]) + v.ghost_offset * bytes[static_cast<std::size_t>(a)]);
        return out;
    }

    std::vector<unsigned char*> assembled_bases(const std::vector<int>& arrays) const {
        std::vector<unsigned char*> out;
        for (int a : arrays) out.push_back(static_cast<unsigned char*>(assembled[static_cast<std::size_t>(a)]));
        return out;
    }

    // every row of `rows` for every listed array, in one copy kernel;
    // swap: the rows read as (destination, source, count)
    void copy(const std::vector<unsigned char*>& dst, const std::vector<unsigned char*>& src,
              const Rows& rows, const std::vector<int>& arrays, bool swap, cudaStream_t s) const {
        std::vector<dsx_copy> list;
        for (std::size_t j = 0; j < arrays.size(); ++j) {
            const long long b = bytes[static_cast<std::size_t>(arrays[j])];
            for (std::size_t r = 0; r < rows.n.size(); ++r) {
                const long long si = swap ? rows.dst[r] : rows.src[r];
                const long long di = swap ? rows.src[r] : rows.dst[r];
                list.push_back({src[j] + si * b, dst[j] + di * b, rows.n[r] * b});
            }
        }
        if (list.empty()) return;
        check(dsx_copy_segments(list.data(), static_cast<long long>(list.size()), s));
        ++const_cast<dsx_shard*>(this)->launches;
    }

    // one message per peer each way through the transport
    void exchange(const std::map<int, void*>& out, const std::map<int, long long>& out_bytes,
                  const std::map<int, void*>& in, const std::map<int, long long>& in_bytes,
                  cudaStream_t s) {
        std::vector<int> to, from;
        std::vector<const void*> sb;
        std::vector<void*> rb;
        std::vector<long long> sn, rn;
        for (const auto& kv : out_bytes)
            if (kv.second > 0) {
                to.push_back(kv.first);
                sb.push_back(out.at(kv.first));
                sn.push_back(kv.second);
            }
        for (const auto& kv : in_bytes)
            if (kv.second > 0) {
                from.push_back(kv.first);
                rb.push_back(in.at(kv.first));
                rn.push_back(kv.second);
            }
        if (!tr.exchange) fail(DSX_E_INVALID, "the transport has no exchange");
        const int st = tr.exchange(tr.user, static_cast<int>(to.size()), to.data(), sb.data(), sn.data(),
                                   static_cast<int>(from.size()), from.data(), rb.data(), rn.data(), s);
        if (st != DSX_OK) fail(DSX_E_RUNTIME, "transport exchange failed");
    }

    void allreduce(std::vector<long long>& v) {
        if (!tr.allreduce_i64 || tr.allreduce_i64(tr.user, v.data(), static_cast<long long>(v.size())) != DSX_OK)
            fail(DSX_E_RUNTIME, "transport all-reduce failed");
    }

    void allreduce(std::vector<double>& v) {
        if (!tr.allreduce_f64 || tr.allreduce_f64(tr.user, v.data(), static_cast<long long>(v.size())) != DSX_OK)
            fail(DSX_E_RUNTIME, "transport all-reduce failed");
    }

    std::vector<long long> owned_counts(cudaStream_t s) const {
        std::vector<long long> o(static_cast<std::size_t>(P)), gh(static_cast<std::size_t>(P));
        check(dsx_grid_counts(grid, o.data(), gh.data(), s));
        return o;
    }

    // ------------------------------------------------------------ migrate

    // After a local migrate (res: P x 6): the particles placed into other
    // shards' subdomains go there; this shard's subdomains are assembled.
    void redistribute(const std::vector<long long>& res, cudaStream_t s, long long* results) {
        // one all-reduce carries the (destination, source) counts, every
        // subdomain's retained particles and every shard's storage, so that
        // all shards see any shard's shortfall before data moves and fail
        // together (the reference agrees on errors the same way,
        // src/runtime.cpp:214-230)
        const std::size_t PP = static_cast<std::size_t>(P) * P;
        std::vector<long long> pairs(PP + static_cast<std::size_t>(P) + static_cast<std::size_t>(nshards), 0);
        check(dsx_grid_migration_pairs(grid, pairs.data(), s));
        ++launches;
        for (int t : mine) pairs[PP + t] = res[static_cast<std::size_t>(6 * t + 2)];
        pairs[PP + P + shard] = capacity;
        allreduce(pairs);
        const auto M = [&](int t, int q) { return pairs[static_cast<std::size_t>(t) * P + q]; };
        {
            std::vector<long long> need(static_cast<std::size_t>(nshards), 0);
            for (int t = 0; t < P; ++t) {
                long long n = pairs[PP + t];
                for (int q = 0; q < P; ++q) n += M(t, q);
                need[static_cast<std::size_t>(owners[t])] += n;
            }
            for (int r = 0; r < nshards; ++r)
                if (need[r] > pairs[PP + P + r]) {
                    planned = false;
                    fail(DSX_E_LENGTH, "particle storage of shard " + std::to_string(r) +
                                           " is smaller than its subdomains' particles after migration");
                }
        }
        std::vector<long long> local_n(static_cast<std::size_t>(P)), obase(static_cast<std::size_t>(P) + 1, 0);
        for (int t = 0; t < P; ++t) {
            local_n[t] = res[static_cast<std::size_t>(6 * t + 5)];
            obase[t + 1] = obase[t] + local_n[t];
        }
        const std::vector<int> all = all_arrays();
        std::map<int, void*> out, in;
        std::map<int, long long> out_bytes, in_bytes, from_peer;
        const std::vector<unsigned char*> owned = owned_bases(all);
        bool leaving = false;
        for (int p = 0; p < nshards; ++p) {
            if (p == shard) continue;
            Rows rows;
            long long n = 0;
            for (int t = 0; t < P; ++t)
                if (owners[t] == p && local_n[t] > 0) {
                    rows.add(obase[t], n, local_n[t]);
                    n += local_n[t];
                }
            if (n > 0) {
                leaving = true;
                void* buf = sendbuf.emplace(p, std::make_unique<DeviceBuffer>()).first->second->ensure(packed_bytes(n, all));
                copy(sections(buf, n, all), owned, rows, all, false, s);
                out[p] = buf;
                out_bytes[p] = packed_bytes(n, all);
            }
            long long m = 0;
            for (int t : mine)
                for (int q = 0; q < P; ++q)
                    if (owners[q] == p) m += M(t, q);
            from_peer[p] = m;
            if (m > 0) {
                in[p] = recvbuf.emplace(p, std::make_unique<DeviceBuffer>()).first->second->ensure(packed_bytes(m, all));
                in_bytes[p] = packed_bytes(m, all);
            }
        }
        exchange(out, out_bytes, in, in_bytes, s);
        // new layout: retained, then every source's group in ascending order
        std::vector<long long> counts(static_cast<std::size_t>(P), 0);
        std::vector<int> peers;
        for (const auto& kv : in_bytes) peers.push_back(kv.first);
        std::map<int, int> source_of;
        for (std::size_t k = 0; k < peers.size(); ++k) source_of[peers[k]] = static_cast<int>(k);
        std::map<int, long long> peer_at;
        std::vector<dsx_segment> segs;
        for (int t : mine) {
            const long long retained = res[static_cast<std::size_t>(6 * t + 2)];
            long long received = 0;
            for (int q = 0; q < P; ++q) received += M(t, q);
            counts[t] = retained + received;
            auto push = [&](int source, long long from, long long at, long long c) {
                if (c <= 0) return;
                if (!segs.empty()) {
                    dsx_segment& b = segs.back();
                    if (b.source == source && b.dst_rank == t && b.src_index + b.count == from &&
                        b.dst_index + b.count == at) {
                        b.count += c;
                        return;
                    }
                }
                segs.push_back({source, from, t, at, c});
            };
            push(-1, obase[t], 0, retained);
            long long at = retained, local_at = obase[t] + retained;
            for (int q = 0; q < P; ++q) {
                const long long c = M(t, q);
                if (!c) continue;
                const int p = owners[q];
                if (p == shard) {
                    push(-1, local_at, at, c);
                    local_at += c;
                } else {
                    push(source_of.at(p), peer_at[p], at, c);
                    peer_at[p] += c;
                }
                at += c;
            }
            if (results) {
                long long* o = results + 6 * t;
                const long long sent = res[static_cast<std::size_t>(6 * t + 3)];
                o[0] = (sent != 0 || received != 0) ? 1 : 0;
                o[1] = res[static_cast<std::size_t>(6 * t + 1)];
                o[2] = retained;
                o[3] = sent;
                o[4] = received;
                o[5] = counts[t];
            }
        }
        planned = false;
        if (peers.empty() && !leaving) return;   // the local layout is final
        std::vector<const void*> sources(peers.size() * kArraySlots, nullptr);
        for (std::size_t k = 0; k < peers.size(); ++k) {
            const std::vector<unsigned char*> sec = sections(in.at(peers[k]), from_peer.at(peers[k]), all);
            for (std::size_t a = 0; a < sec.size(); ++a) sources[k * kArraySlots + a] = sec[a];
        }
        launches += 2;   // the copies and the new layout
        check(dsx_grid_assemble(grid, counts.data(), static_cast<int>(peers.size()),
                                sources.empty() ? nullptr : sources.data(),
                                static_cast<long long>(segs.size()), segs.empty() ? nullptr : segs.data(), s));
    }

    void migrate(cudaStream_t s, long long* results) {
        if (dynamic) {
            const std::vector<long long> o = owned_counts(s);
            std::vector<double> w(o.begin(), o.end());
            allreduce(w);
            check(dsx_grid_set_rebalance_work(grid, w.data()));
        }
        std::vector<long long> res(static_cast<std::size_t>(6) * P);
        check(dsx_grid_migrate(grid, s, res.data()));
        // classify, scan, layout, move, emigrant histogram / scan / placement
        // (and the rebalance kernel of a Dynamic grid)
        launches += 7 + (dynamic ? 1 : 0);
        redistribute(res, s, results);
    }

    void rebalance(const double* work, bool force, cudaStream_t s, long long* results, double* imbalance) {
        std::vector<double> w(static_cast<std::size_t>(P), 0.0);
        const std::vector<long long> before = owned_counts(s);
        for (int t : mine) w[t] = work ? work[t] : static_cast<double>(before[t]);
        allreduce(w);
        std::vector<long long> flags(static_cast<std::size_t>(3) * P);
        std::vector<double> imb(static_cast<std::size_t>(P), 1.0);
        check(dsx_grid_rebalance(grid, w.data(), force ? 1 : 0, s, flags.data(), imb.data()));
        launches += 8 + 1;   // the rebalance, its migrate, the pair counts
        // the migrate inside the rebalance, in migrate's result format
        std::vector<long long> pairs(static_cast<std::size_t>(P) * P);
        check(dsx_grid_migration_pairs(grid, pairs.data(), s));
        const std::vector<long long> now = owned_counts(s);
        std::vector<long long> res(static_cast<std::size_t>(6) * P, 0);
        for (int t = 0; t < P; ++t) {
            long long sent = 0, received = 0;
            for (int q = 0; q < P; ++q) {
                sent += pairs[static_cast<std::size_t>(q) * P + t];
                received += pairs[static_cast<std::size_t>(t) * P + q];
            }
            long long* o = &res[static_cast<std::size_t>(6 * t)];
            o[0] = (sent != 0 || received != 0) ? 1 : 0;
            o[1] = before[t];
            o[2] = before[t] - sent;
            o[3] = sent;
            o[4] = received;
            o[5] = now[t];
        }
        std::vector<long long> mig(static_cast<std::size_t>(6) * P, 0);
        redistribute(res, s, mig.data());
        if (results)
            for (int t : mine) {
                results[3 * t + 0] = flags[static_cast<std::size_t>(3 * t + 0)];
                results[3 * t + 1] = flags[static_cast<std::size_t>(3 * t + 1)];
                results[3 * t + 2] = mig[static_cast<std::size_t>(6 * t + 5)];
            }
        if (imbalance) *imbalance = imb[0];
    }

    // -------------------------------------------------------------- halo

    void make_plan(const std::vector<long long>& length, const std::vector<int>& first) {
        g.assign(static_cast<std::size_t>(P), 0);
        gbase.assign(static_cast<std::size_t>(P) + 1, 0);
        local = Rows();
        recv.clear();
        send.clear();
        recv_n.clear();
        send_n.clear();
        long long at = 0;
        for (int t : mine) {
            gbase[t] = at;
            for (int m = 0; m < nn[t]; ++m) {
                const long long e = sender_of[static_cast<std::size_t>(t) * kNeighbors + m];
                if (e < 0 || length[static_cast<std::size_t>(e)] == 0) continue;
                const long long n = length[static_cast<std::size_t>(e)];
                const int p = owners[static_cast<std::size_t>(e / kNeighbors)];
                if (p == shard) {
                    local.add(first[static_cast<std::size_t>(e)], at, n);
                } else {
                    long long& off = recv_n[p];
                    recv[p].add(off, at, n);
                    off += n;
                }
                at += n;
            }
            g[t] = at - gbase[t];
        }
        total = at;
        gbase[static_cast<std::size_t>(P)] = at;
        for (int t = 0; t < P; ++t) {
            const int p = owners[t];
            if (p == shard) continue;
            for (int m = 0; m < nn[t]; ++m) {
                const long long e = sender_of[static_cast<std::size_t>(t) * kNeighbors + m];
                if (e < 0 || length[static_cast<std::size_t>(e)] == 0 ||
                    owners[static_cast<std::size_t>(e / kNeighbors)] != shard)
                    continue;
                const long long n = length[static_cast<std::size_t>(e)];
                long long& off = send_n[p];
                send[p].add(first[static_cast<std::size_t>(e)], off, n);
                off += n;
            }
        }
        planned = true;
    }

    // grows the assembled region (keeping its contents); true if it grew
    bool ensure_assembled(long long n, cudaStream_t s) {
        if (n <= assembled_cap && !assembled.empty()) return false;
        const long long cap = std::max<long long>(n + n / 4, 1024);
        std::vector<void*> next(bytes.size(), nullptr);
        cudaError_t e = cudaSuccess;
        for (std::size_t a = 0; a < bytes.size() && e == cudaSuccess; ++a) {
            e = cudaMalloc(&next[a], static_cast<std::size_t>(cap * bytes[a]));
            if (e == cudaSuccess && assembled_cap)
                e = cudaMemcpyAsync(next[a], assembled[a], static_cast<std::size_t>(assembled_cap * bytes[a]),
                                    cudaMemcpyDeviceToDevice, s);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            for (void* p : next) cudaFree(p);   // the old region stays in use
            cuda(e, "grow ghost region");
        }
        for (void* p : assembled) cudaFree(p);
        assembled = next;
        assembled_cap = cap;
        return true;
    }

    void publish_plan(cudaStream_t s) {
        std::vector<int> gi(static_cast<std::size_t>(P)), bi(static_cast<std::size_t>(P) + 1);
        for (int t = 0; t < P; ++t) gi[t] = static_cast<int>(g[t]);
        for (int t = 0; t <= P; ++t) bi[t] = static_cast<int>(gbase[t]);
        const int tot[2] = {static_cast<int>(total), 0};
        cuda(cudaMemcpyAsync(d_g, gi.data(), sizeof(int) * P, cudaMemcpyHostToDevice, s), "publish plan");
        cuda(cudaMemcpyAsync(d_gbase, bi.data(), sizeof(int) * (P + 1), cudaMemcpyHostToDevice, s), "publish plan");
        cuda(cudaMemcpyAsync(d_totals, tot, sizeof(tot), cudaMemcpyHostToDevice, s), "publish plan");
        cuda(cudaStreamSynchronize(s), "publish plan");
    }

    // lists of local senders: into the assembled region (own receivers) or
    // to the receivers' shards; lists from other shards into the region
    void ship(const std::vector<int>& arrays, cudaStream_t s) {
        std::map<int, void*> out, in;
        std::map<int, long long> out_bytes, in_bytes;
        const std::vector<unsigned char*> gh = ghost_bases(arrays);
        for (const auto& kv : send) {
            const long long n = send_n.at(kv.first);
            void* buf = sendbuf.emplace(kv.first, std::make_unique<DeviceBuffer>()).first->second->ensure(packed_bytes(n, arrays));
            copy(sections(buf, n, arrays), gh, kv.second, arrays, false, s);
            out[kv.first] = buf;
            out_bytes[kv.first] = packed_bytes(n, arrays);
        }
        for (const auto& kv : recv_n) {
            in[kv.first] = recvbuf.emplace(kv.first, std::make_unique<DeviceBuffer>()).first->second->ensure(packed_bytes(kv.second, arrays));
            in_bytes[kv.first] = packed_bytes(kv.second, arrays);
        }
        exchange(out, out_bytes, in, in_bytes, s);
        const std::vector<unsigned char*> asmb = assembled_bases(arrays);
        copy(asmb, gh, local, arrays, false, s);
        for (const auto& kv : recv)
            copy(asmb, sections(in.at(kv.first), recv_n.at(kv.first), arrays), kv.second, arrays, false, s);
    }

    // the inverse: assembled values back into the local slots of their
    // lists (own senders) or to the senders' shards
    void give_back(const std::vector<int>& arrays, cudaStream_t s) {
        std::map<int, void*> out, in;
        std::map<int, long long> out_bytes, in_bytes;
        const std::vector<unsigned char*> gh = ghost_bases(arrays);
        const std::vector<unsigned char*> asmb = assembled_bases(arrays);
        copy(gh, asmb, local, arrays, true, s);
        for (const auto& kv : recv) {
            const long long n = recv_n.at(kv.first);
            void* buf = sendbuf.emplace(kv.first, std::make_unique<DeviceBuffer>()).first->second->ensure(packed_bytes(n, arrays));
            copy(sections(buf, n, arrays), asmb, kv.second, arrays, true, s);
            out[kv.first] = buf;
            out_bytes[kv.first] = packed_bytes(n, arrays);
        }
        for (const auto& kv : send_n) {
            in[kv.first] = recvbuf.emplace(kv.first, std::make_unique<DeviceBuffer>()).first->second->ensure(packed_bytes(kv.second, arrays));
            in_bytes[kv.first] = packed_bytes(kv.second, arrays);
        }
        exchange(out, out_bytes, in, in_bytes, s);
        for (const auto& kv : send)
            copy(gh, sections(in.at(kv.first), send_n.at(kv.first), arrays), kv.second, arrays, true, s);
    }

    void exchange_halo(bool rebuild, bool positions_only, cudaStream_t s, long long* results) {
        const bool build = rebuild || !planned;
        const bool had_plan = planned;
        const std::vector<long long> prev_g = g;
        std::vector<long long> hres(static_cast<std::size_t>(4) * P);
        check(dsx_grid_exchange_halo(grid, build ? 1 : 0, (positions_only && !build) ? 1 : 0, s, hres.data()));
        launches += build ? 4 : 1;   // classify, scan, layout, scatter; or the refresh
        bool grew = false;
        if (build) {
            std::vector<int> len(static_cast<std::size_t>(P) * kNeighbors), first(len.size());
            check(dsx_grid_send_lists(grid, len.data(), first.data(), s));
            std::vector<long long> length(len.begin(), len.end());
            allreduce(length);
            make_plan(length, first);
            grew = ensure_assembled(total, s);
            publish_plan(s);
        }
        const std::vector<int> arrays = (positions_only && !build) ? std::vector<int>{0, 1, 2} : all_arrays();
        ship(arrays, s);
        if (results)
            for (int t : mine) {
                // layout_changed (src/runtime.cpp:966-980): a requested
                // rebuild, or another ghost count (none since a migrate)
                const long long gt = g[t];
                long long changed = 0;
                if (rebuild) changed = 1;
                else if (!had_plan) changed = gt != 0;
                else changed = prev_g[t] != gt;
                long long* o = results + 4 * t;
                o[0] = gt;
                o[1] = changed;
                o[2] = grew ? 1 : 0;
                o[3] = build ? 0 : 1;
            }
    }

    void reverse_halo(cudaStream_t s) {
        if (!planned) fail(DSX_E_LOGIC, "reverse_halo without a halo plan");
        give_back({6, 7, 8}, s);
        check(dsx_grid_reverse_halo(grid, s));
        ++launches;
    }

    std::vector<int> field_arrays(int nfields, const int* ids) const {
        std::vector<int> out;
        for (int k = 0; k < nfields; ++k) {
            if (ids[k] < 0 || 13 + ids[k] >= narrays()) fail(DSX_E_INVALID, "unknown field");
            out.push_back(13 + ids[k]);
        }
        return out;
    }
};

namespace {

// Contiguous Cartesian blocks of the process grid (the (a, b, c) with
// a * b * c = nshards that divides dims with the least cut area; ties: the
// first in (a, b, c) order), else contiguous runs of subdomain ranks.
std::vector<int> block_owners(const int* dims, int nshards) {
    const int P = dims[0] * dims[1] * dims[2];
    std::vector<int> owners(static_cast<std::size_t>(P), 0);
    long long best = -1;
    int ba = 0, bb = 0, bc = 0;
    for (int a = 1; a <= nshards; ++a) {
        if (nshards % a || dims[0] % a) continue;
        for (int b = 1; b <= nshards / a; ++b) {
            if ((nshards / a) % b || dims[1] % b) continue;
            const int c = nshards / a / b;
            if (dims[2] % c) continue;
            const long long cut = static_cast<long long>(a - 1) * dims[1] * dims[2] +
                                  static_cast<long long>(b - 1) * dims[0] * dims[2] +
                                  static_cast<long long>(c - 1) * dims[0] * dims[1];
            if (best < 0 || cut < best) {
                best = cut;
                ba = a;
                bb = b;
                bc = c;
            }
        }
    }
    for (int t = 0; t < P; ++t) {
        if (best < 0) {
            owners[t] = static_cast<int>(static_cast<long long>(t) * nshards / P);
            continue;
        }
        const int x = t / (dims[1] * dims[2]), y = (t / dims[2]) % dims[1], z = t % dims[2];
        owners[t] = ((x / (dims[0] / ba)) * bb + y / (dims[1] / bb)) * bc + z / (dims[2] / bc);
    }
    return owners;
}

std::size_t field_bytes(int type, int components) {
    switch (type) {
    case DSX_INT32: case DSX_UINT32: case DSX_FLOAT32: return 4u * static_cast<std::size_t>(components);
    default: return 8u * static_cast<std::size_t>(components);
    }
}

}  // namespace

extern "C" {

int dsx_shard_create(const dsx_grid_desc* desc, const dsx_field_desc* fields, int nfields,
                     long long particles, long long ghost_capacity, int shard, int nshards,
                     const int* owners, const dsx_transport* transport, dsx_shard** out) {
    return guarded([&] {
        if (!desc || !transport || !out || (nfields > 0 && !fields)) fail(DSX_E_INVALID, "null argument");
        if (nshards < 1 || shard < 0 || shard >= nshards) fail(DSX_E_INVALID, "shard out of range");
        *out = nullptr;
        auto sh = std::make_unique<dsx_shard>();
        check(dsx_grid_create(desc, fields, nfields, particles, ghost_capacity, &sh->grid));
        sh->P = desc->nranks;
        sh->shard = shard;
        sh->nshards = nshards;
        sh->tr = *transport;
        sh->dynamic = desc->policy == DSX_DYNAMIC;
        sh->capacity = particles;
        if (nshards > sh->P) fail(DSX_E_INVALID, "more shards than subdomains");
        int coords[3];
        double local[6];
        check(dsx_grid_topology(sh->grid, 0, sh->dims, coords, local));
        if (owners) {
            sh->owners.assign(owners, owners + sh->P);
            for (int o : sh->owners)
                if (o < 0 || o >= nshards) fail(DSX_E_INVALID, "owner out of range");
        } else {
            sh->owners = block_owners(sh->dims, nshards);
        }
        for (int t = 0; t < sh->P; ++t)
            if (sh->owners[t] == shard) sh->mine.push_back(t);
        // receiver t's block m holds the list its neighbor sends toward -d_m
        std::vector<std::vector<std::array<int, 4>>> topo(static_cast<std::size_t>(sh->P));
        for (int t = 0; t < sh->P; ++t) {
            int count = 0;
            int info[kNeighbors * 5];
            double shifts[kNeighbors * 3];
            check(dsx_grid_neighbors(sh->grid, t, &count, info, shifts));
            for (int n = 0; n < count; ++n)
                topo[t].push_back({info[5 * n], info[5 * n + 1], info[5 * n + 2], info[5 * n + 3]});
        }
        sh->nn.resize(static_cast<std::size_t>(sh->P));
        sh->sender_of.assign(static_cast<std::size_t>(sh->P) * kNeighbors, -1);
        for (int t = 0; t < sh->P; ++t) {
            sh->nn[t] = static_cast<int>(topo[t].size());
            for (std::size_t m = 0; m < topo[t].size(); ++m) {
                const int q = topo[t][m][0];
                if (q < 0) continue;
                for (std::size_t n = 0; n < topo[q].size(); ++n)
                    if (topo[q][n][1] == -topo[t][m][1] && topo[q][n][2] == -topo[t][m][2] &&
                        topo[q][n][3] == -topo[t][m][3]) {
                        sh->sender_of[static_cast<std::size_t>(t) * kNeighbors + m] =
                            static_cast<long long>(q) * kNeighbors + static_cast<long long>(n);
                        break;
                    }
            }
        }
        sh->bytes.assign(11, 8);
        sh->bytes.push_back(4);
        sh->bytes.push_back(4);
        for (int f = 0; f < nfields; ++f)
            sh->bytes.push_back(static_cast<int>(field_bytes(fields[f].type, fields[f].components)));
        cuda(cudaMalloc(reinterpret_cast<void**>(&sh->d_g), sizeof(int) * sh->P), "cudaMalloc");
        cuda(cudaMalloc(reinterpret_cast<void**>(&sh->d_gbase), sizeof(int) * (sh->P + 1)), "cudaMalloc");
        cuda(cudaMalloc(reinterpret_cast<void**>(&sh->d_totals), sizeof(int) * 2), "cudaMalloc");
        cuda(cudaMemset(sh->d_g, 0, sizeof(int) * sh->P), "cudaMemset");
        cuda(cudaMemset(sh->d_gbase, 0, sizeof(int) * (sh->P + 1)), "cudaMemset");
        cuda(cudaMemset(sh->d_totals, 0, sizeof(int) * 2), "cudaMemset");
        *out = sh.release();
    });
}

int dsx_shard_destroy(dsx_shard* shard) {
    delete shard;
    return DSX_OK;
}

int dsx_shard_plan_owners(const int* dims, int nshards, int* owners) {
    return guarded([&] {
        if (!dims || !owners) fail(DSX_E_INVALID, "null argument");
        long long P = 1;
        for (int a = 0; a < 3; ++a) {
            if (dims[a] < 1) fail(DSX_E_INVALID, "process grid dims must be positive");
            P *= dims[a];
            if (P > (1 << 20)) fail(DSX_E_INVALID, "process grid too large");
        }
        if (nshards < 1 || nshards > P) fail(DSX_E_INVALID, "shards must be in 1..P");
        const std::vector<int> planned = block_owners(dims, nshards);
        std::copy(planned.begin(), planned.end(), owners);
    });
}

int dsx_shard_owners(dsx_shard* shard, int* owners) {
    return guarded([&] {
        if (!shard || !owners) fail(DSX_E_INVALID, "null argument");
        std::copy(shard->owners.begin(), shard->owners.end(), owners);
    });
}

int dsx_shard_upload(dsx_shard* shard, const long long* counts, const void* const* arrays, void* stream) {
    return guarded([&] {
        if (!shard || !counts) fail(DSX_E_INVALID, "null argument");
        for (int t = 0; t < shard->P; ++t)
            if (counts[t] != 0 && shard->owners[t] != shard->shard)
                fail(DSX_E_INVALID, "particles outside this shard's subdomains");
        check(dsx_grid_upload(shard->grid, counts, arrays, stream));
        shard->planned = false;
    });
}

int dsx_shard_download(dsx_shard* shard, long long* counts, void* const* arrays, void* stream) {
    return guarded([&] {
        if (!shard || !counts) fail(DSX_E_INVALID, "null argument");
        check(dsx_grid_download(shard->grid, counts, arrays, stream));
    });
}

int dsx_shard_migrate(dsx_shard* shard, void* stream, long long* results) {
    return guarded([&] {
        if (!shard) fail(DSX_E_INVALID, "null shard");
        shard->migrate(static_cast<cudaStream_t>(stream), results);
    });
}

int dsx_shard_rebalance(dsx_shard* shard, const double* work, int force, void* stream,
                        long long* results, double* imbalance) {
    return guarded([&] {
        if (!shard) fail(DSX_E_INVALID, "null shard");
        shard->rebalance(work, force != 0, static_cast<cudaStream_t>(stream), results, imbalance);
    });
}

int dsx_shard_exchange_halo(dsx_shard* shard, int rebuild, int positions_only, void* stream,
                            long long* results) {
    return guarded([&] {
        if (!shard) fail(DSX_E_INVALID, "null shard");
        shard->exchange_halo(rebuild != 0, positions_only != 0, static_cast<cudaStream_t>(stream), results);
    });
}

int dsx_shard_reverse_halo(dsx_shard* shard, void* stream) {
    return guarded([&] {
        if (!shard) fail(DSX_E_INVALID, "null shard");
        shard->reverse_halo(static_cast<cudaStream_t>(stream));
    });
}

int dsx_shard_step(dsx_shard* shard, dsx_step_callback callback, void* user, void* stream,
                   unsigned* status) {
    return guarded([&] {
        if (!shard) fail(DSX_E_INVALID, "null shard");
        shard->planned = false;   // the per-call plan and the assembled region are stale
        check(dsx_grid_sharded_step(shard->grid, shard->owners.data(), shard->shard, shard->nshards,
                                    &shard->tr, callback, user, stream, status));
        // rebalance, classify + scan + export, bases, move, emigrant
        // histogram / scan / placement, immigrant masks / scan / scatter,
        // the reverse sum, and the message copies
        shard->launches += 12 + (shard->dynamic ? 1 : 0) + 6;
    });
}

int dsx_shard_forward_exchange(dsx_shard* shard, int nfields, const int* field_ids, void* stream) {
    return guarded([&] {
        if (!shard || (nfields > 0 && !field_ids)) fail(DSX_E_INVALID, "null argument");
        if (!shard->planned) fail(DSX_E_LOGIC, "forward_exchange without a halo plan");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        check(dsx_grid_forward_exchange(shard->grid, nfields, field_ids, s));
        ++shard->launches;
        shard->ship(shard->field_arrays(nfields, field_ids), s);
    });
}

int dsx_shard_reverse_exchange(dsx_shard* shard, int nfields, const int* field_ids, const int* ops,
                               void* stream) {
    return guarded([&] {
        if (!shard || (nfields > 0 && (!field_ids || !ops))) fail(DSX_E_INVALID, "null argument");
        if (!shard->planned) fail(DSX_E_LOGIC, "reverse_exchange without a halo plan");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        shard->give_back(shard->field_arrays(nfields, field_ids), s);
        check(dsx_grid_reverse_exchange(shard->grid, nfields, field_ids, ops, s));
        ++shard->launches;
    });
}

int dsx_shard_owned_view(dsx_shard* shard, dsx_grid_view* out) {
    return guarded([&] {
        if (!shard || !out) fail(DSX_E_INVALID, "null argument");
        check(dsx_grid_view_get(shard->grid, out));
    });
}

int dsx_shard_ghost_view(dsx_shard* shard, dsx_grid_view* out) {
    return guarded([&] {
        if (!shard || !out) fail(DSX_E_INVALID, "null argument");
        dsx_grid_view v{};
        check(dsx_grid_view_get(shard->grid, &v));
        dsx_grid_view g{};
        for (std::size_t a = 0; a < shard->assembled.size() && a < 32; ++a) g.base[a] = shard->assembled[a];
        g.owned_offset = 0;
        g.ghost_offset = 0;
        g.n = v.n;
        g.obase = v.obase;
        g.g = shard->d_g;
        g.gbase = shard->d_gbase;
        g.halo_totals = shard->d_totals;
        g.particles = v.particles;
        g.ghost_capacity = shard->assembled_cap;
        g.nranks = shard->P;
        *out = g;
    });
}

int dsx_shard_totals(dsx_shard* shard, long long* out4, void* stream) {
    return guarded([&] {
        if (!shard || !out4) fail(DSX_E_INVALID, "null argument");
        check(dsx_grid_totals(shard->grid, out4, stream));
    });
}

int dsx_shard_launches(dsx_shard* shard, long long* count) {
    return guarded([&] {
        if (!shard || !count) fail(DSX_E_INVALID, "null argument");
        *count = shard->launches;
    });
}

int dsx_shard_counts(dsx_shard* shard, long long* owned, long long* ghosts, void* stream) {
    return guarded([&] {
        if (!shard || !owned || !ghosts) fail(DSX_E_INVALID, "null argument");
        const std::vector<long long> o = shard->owned_counts(static_cast<cudaStream_t>(stream));
        // after a fused step (dsx_shard_step) the grid's own ghost blocks
        // are this shard's receivers' ghosts
        std::vector<long long> gg(static_cast<std::size_t>(shard->P), 0), oo(gg.size(), 0);
        if (!shard->planned) check(dsx_grid_counts(shard->grid, oo.data(), gg.data(), stream));
        for (int t = 0; t < shard->P; ++t) {
            const bool mine = shard->owners[t] == shard->shard;
            owned[t] = mine ? o[t] : 0;
            ghosts[t] = !mine ? 0 : shard->planned ? shard->g[t] : gg[static_cast<std::size_t>(t)];
        }
    });
}

}  // extern "C"
