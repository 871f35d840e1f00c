// Thread-per-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE ONLY: it is
// linked into the oracle build of the reference Host path and into nothing
// else.
#include "mpi.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <memory>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>
#include <vector>

namespace {

struct CommState {
    int handle = 0;
    bool cartesian = false;
    int ndims = 0;
    int dims[8] = {0};
    int periods[8] = {0};
    // collective rendezvous
    std::mutex mutex;
    std::condition_variable cv;
    int arrived = 0;
    std::uint64_t generation = 0;
    std::vector<const void*> slot_a, slot_b, slot_c;
};

struct RequestState {
    bool receive = false;
    void* buffer = nullptr;
    std::size_t capacity = 0;
    int source = 0;
    int tag = 0;
    int comm = 0;
};

using MailKey = std::tuple<int, int, int, int>;  // comm, source, dest, tag

// One mailbox per destination rank: a send wakes only the rank it is
// addressed to (a single shared condition variable would wake every waiting
// rank on every message).
struct Mailbox {
    std::mutex mutex;
    std::condition_variable cv;
    std::map<MailKey, std::deque<std::vector<char>>> mail;
};

}  // namespace

struct shim_world_t {
    int size = 1;
    std::mutex mutex;
    std::map<int, CommState*> comms;
    std::map<int, int> creation_handle;   // creation sequence -> handle
    std::vector<int> creation_sequence;   // per rank
    int next_handle = 16;
    std::vector<std::unique_ptr<Mailbox>> boxes;   // per destination rank
};

namespace {

thread_local shim_world* tl_world = nullptr;
thread_local int tl_rank = 0;

std::mutex g_type_mutex;
std::map<int, std::size_t> g_type_size;
int g_next_type = 100;

shim_world* world() {
    if (!tl_world) {
        std::fprintf(stderr, "mpi shim: MPI call on a thread with no bound rank\n");
        std::abort();
    }
    return tl_world;
}

std::size_t type_size(MPI_Datatype type) {
    switch (type) {
    case MPI_BYTE: case MPI_CHAR: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_LONG_LONG: case MPI_UNSIGNED_LONG_LONG: case MPI_DOUBLE:
    case MPI_UINT64_T: case MPI_INT64_T: return 8;
    default: break;
    }
    std::lock_guard<std::mutex> lock(g_type_mutex);
    auto found = g_type_size.find(type);
    if (found == g_type_size.end()) {
        std::fprintf(stderr, "mpi shim: unknown datatype %d\n", type);
        std::abort();
    }
    return found->second;
}

CommState* comm_state(MPI_Comm comm) {
    shim_world* w = world();
    std::lock_guard<std::mutex> lock(w->mutex);
    auto found = w->comms.find(comm);
    if (found == w->comms.end()) {
        std::fprintf(stderr, "mpi shim: unknown communicator %d\n", comm);
        std::abort();
    }
    return found->second;
}

// Every rank calls the communicator constructors in the same order, so the
// k-th construction on each rank names the same communicator.
CommState* create_comm() {
    shim_world* w = world();
    std::lock_guard<std::mutex> lock(w->mutex);
    const int sequence = w->creation_sequence[static_cast<std::size_t>(tl_rank)]++;
    auto found = w->creation_handle.find(sequence);
    if (found != w->creation_handle.end()) return w->comms[found->second];
    auto* state = new CommState();
    state->handle = w->next_handle++;
    state->slot_a.assign(static_cast<std::size_t>(w->size), nullptr);
    state->slot_b.assign(static_cast<std::size_t>(w->size), nullptr);
    state->slot_c.assign(static_cast<std::size_t>(w->size), nullptr);
    w->comms[state->handle] = state;
    w->creation_handle[sequence] = state->handle;
    return state;
}

void barrier(CommState* c, int size) {
    std::unique_lock<std::mutex> lock(c->mutex);
    const std::uint64_t generation = c->generation;
    if (++c->arrived == size) {
        c->arrived = 0;
        ++c->generation;
        c->cv.notify_all();
    } else {
        c->cv.wait(lock, [&] { return c->generation != generation; });
    }
}

int comm_size(MPI_Comm comm) {
    if (comm == MPI_COMM_SELF) return 1;
    return world()->size;
}

template <class T>
void reduce_into(T* out, const T* in, int count, MPI_Op op) {
    for (int i = 0; i < count; ++i) {
        switch (op) {
        case MPI_SUM: out[i] = static_cast<T>(out[i] + in[i]); break;
        case MPI_MIN: out[i] = in[i] < out[i] ? in[i] : out[i]; break;
        case MPI_MAX: out[i] = out[i] < in[i] ? in[i] : out[i]; break;
        default: std::abort();
        }
    }
}

void reduce_typed(void* out, const void* in, int count, MPI_Datatype type,
                  MPI_Op op) {
    switch (type) {
    case MPI_INT: reduce_into(static_cast<int*>(out), static_cast<const int*>(in), count, op); break;
    case MPI_UNSIGNED: reduce_into(static_cast<unsigned*>(out), static_cast<const unsigned*>(in), count, op); break;
    case MPI_LONG_LONG: case MPI_INT64_T:
        reduce_into(static_cast<long long*>(out), static_cast<const long long*>(in), count, op); break;
    case MPI_UNSIGNED_LONG_LONG: case MPI_UINT64_T:
        reduce_into(static_cast<unsigned long long*>(out),
                    static_cast<const unsigned long long*>(in), count, op); break;
    case MPI_DOUBLE: reduce_into(static_cast<double*>(out), static_cast<const double*>(in), count, op); break;
    case MPI_FLOAT: reduce_into(static_cast<float*>(out), static_cast<const float*>(in), count, op); break;
    default:
        std::fprintf(stderr, "mpi shim: reduction on unsupported datatype %d\n", type);
        std::abort();
    }
}

// Posts up to three pointers, waits for everyone, runs `body` (which may read
// every rank's posted pointers), then waits again so the posted buffers stay
// valid until every rank is done reading.
template <class Body>
void collective(MPI_Comm comm, const void* a, const void* b, const void* c,
                Body body) {
    const int size = comm_size(comm);
    if (comm == MPI_COMM_SELF || size == 1) {
        std::vector<const void*> sa{a}, sb{b}, sc{c};
        body(sa, sb, sc);
        return;
    }
    CommState* state = comm_state(comm);
    state->slot_a[static_cast<std::size_t>(tl_rank)] = a;
    state->slot_b[static_cast<std::size_t>(tl_rank)] = b;
    state->slot_c[static_cast<std::size_t>(tl_rank)] = c;
    barrier(state, size);
    body(state->slot_a, state->slot_b, state->slot_c);
    barrier(state, size);
}

}  // namespace

extern "C" {

shim_world* shim_world_create(int size) {
    auto* w = new shim_world();
    w->size = size;
    w->creation_sequence.assign(static_cast<std::size_t>(size), 0);
    for (int r = 0; r < size; ++r) w->boxes.emplace_back(new Mailbox());
    auto* world_comm = new CommState();
    world_comm->handle = MPI_COMM_WORLD;
    world_comm->slot_a.assign(static_cast<std::size_t>(size), nullptr);
    world_comm->slot_b.assign(static_cast<std::size_t>(size), nullptr);
    world_comm->slot_c.assign(static_cast<std::size_t>(size), nullptr);
    w->comms[MPI_COMM_WORLD] = world_comm;
    return w;
}

void shim_world_destroy(shim_world* w) {
    if (!w) return;
    for (auto& entry : w->comms) delete entry.second;
    delete w;
}

void shim_bind_rank(shim_world* w, int rank) {
    tl_world = w;
    tl_rank = rank;
}

void shim_unbind_rank(void) {
    tl_world = nullptr;
    tl_rank = 0;
}

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int, int* provided) {
    if (provided) *provided = MPI_THREAD_MULTIPLE;
    return MPI_SUCCESS;
}
int MPI_Initialized(int* flag) { *flag = tl_world ? 1 : 0; return MPI_SUCCESS; }
int MPI_Finalized(int* flag) { *flag = 0; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Query_thread(int* provided) { *provided = MPI_THREAD_MULTIPLE; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "mpi shim: MPI_Abort(%d)\n", code);
    std::abort();
}
double MPI_Wtime(void) {
    using clock = std::chrono::steady_clock;
    return std::chrono::duration<double>(clock::now().time_since_epoch()).count();
}
int MPI_Get_processor_name(char* name, int* length) {
    std::strcpy(name, "localhost");
    *length = 9;
    return MPI_SUCCESS;
}
int MPI_Error_string(int code, char* text, int* length) {
    *length = std::snprintf(text, MPI_MAX_ERROR_STRING, "mpi shim error %d", code);
    return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int* rank) {
    *rank = comm == MPI_COMM_SELF ? 0 : (world(), tl_rank);
    return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int* size) {
    *size = comm_size(comm);
    return MPI_SUCCESS;
}
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) {
    if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
    CommState* created = create_comm();
    *out = created->handle;
    return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* comm) {
    // Communicators live as long as their world (they are few and tiny).
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}
int MPI_Comm_split_type(MPI_Comm comm, int, int, MPI_Info, MPI_Comm* out) {
    // All ranks share one node: the split keeps everyone, in the same order.
    return MPI_Comm_dup(comm, out);
}

int MPI_Dims_create(int nnodes, int ndims, int* dims) {
    int fixed = 1;
    int free_count = 0;
    for (int d = 0; d < ndims; ++d) {
        if (dims[d] > 0) fixed *= dims[d];
        else ++free_count;
    }
    if (free_count == 0) return fixed == nnodes ? MPI_SUCCESS : MPI_ERR_OTHER;
    if (fixed <= 0 || nnodes % fixed != 0) return MPI_ERR_OTHER;
    int remaining = nnodes / fixed;
    std::vector<int> factors;
    for (int f = 2; remaining > 1 && f * f <= remaining; ++f) {
        while (remaining % f == 0) { factors.push_back(f); remaining /= f; }
    }
    if (remaining > 1) factors.push_back(remaining);
    std::sort(factors.rbegin(), factors.rend());
    std::vector<int> grid(static_cast<std::size_t>(free_count), 1);
    for (int f : factors) {
        auto smallest = std::min_element(grid.begin(), grid.end());
        *smallest *= f;
    }
    std::sort(grid.rbegin(), grid.rend());
    std::size_t next = 0;
    for (int d = 0; d < ndims; ++d) {
        if (dims[d] <= 0) dims[d] = grid[next++];
    }
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm comm, int ndims, const int* dims,
                    const int* periods, int, MPI_Comm* out) {
    if (comm == MPI_COMM_NULL || ndims > 8) return MPI_ERR_OTHER;
    int product = 1;
    for (int d = 0; d < ndims; ++d) product *= dims[d];
    if (product != comm_size(comm)) return MPI_ERR_OTHER;
    CommState* created = create_comm();
    {
        std::lock_guard<std::mutex> lock(created->mutex);
        created->cartesian = true;
        created->ndims = ndims;
        for (int d = 0; d < ndims; ++d) {
            created->dims[d] = dims[d];
            created->periods[d] = periods[d];
        }
    }
    *out = created->handle;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int* coords) {
    CommState* c = comm_state(comm);
    int remainder = rank;
    for (int d = c->ndims - 1; d >= 0; --d) {
        if (d < maxdims) coords[d] = remainder % c->dims[d];
        remainder /= c->dims[d];
    }
    return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int* coords, int* rank) {
    CommState* c = comm_state(comm);
    int result = 0;
    for (int d = 0; d < c->ndims; ++d) {
        int coordinate = coords[d];
        if (coordinate < 0 || coordinate >= c->dims[d]) {
            if (!c->periods[d]) { *rank = MPI_PROC_NULL; return MPI_SUCCESS; }
            coordinate %= c->dims[d];
            if (coordinate < 0) coordinate += c->dims[d];
        }
        result = result * c->dims[d] + coordinate;
    }
    *rank = result;
    return MPI_SUCCESS;
}

int MPI_Get_address(const void* location, MPI_Aint* address) {
    *address = reinterpret_cast<MPI_Aint>(location);
    return MPI_SUCCESS;
}

int MPI_Type_create_struct(int count, const int* block_lengths,
                           const MPI_Aint* displacements,
                           const MPI_Datatype* types, MPI_Datatype* out) {
    std::size_t upper = 0;
    std::size_t alignment = 1;
    for (int i = 0; i < count; ++i) {
        const std::size_t element = type_size(types[i]);
        alignment = std::max(alignment, element);
        upper = std::max(upper, static_cast<std::size_t>(displacements[i]) +
                                    element * static_cast<std::size_t>(block_lengths[i]));
    }
    const std::size_t extent = (upper + alignment - 1) / alignment * alignment;
    std::lock_guard<std::mutex> lock(g_type_mutex);
    *out = g_next_type++;
    g_type_size[*out] = extent;
    return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype* type) { *type = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
int MPI_Type_size(MPI_Datatype type, int* size) {
    *size = static_cast<int>(type_size(type));
    return MPI_SUCCESS;
}

int MPI_Isend(const void* buffer, int count, MPI_Datatype type, int dest,
              int tag, MPI_Comm comm, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    const std::size_t bytes = static_cast<std::size_t>(count) * type_size(type);
    std::vector<char> payload(bytes);
    if (bytes) std::memcpy(payload.data(), buffer, bytes);
    shim_world* w = world();
    if (dest < 0 || dest >= w->size) {
        std::fprintf(stderr, "mpi shim: send to rank %d of %d\n", dest, w->size);
        std::abort();
    }
    Mailbox& box = *w->boxes[static_cast<std::size_t>(dest)];
    {
        std::lock_guard<std::mutex> lock(box.mutex);
        box.mail[MailKey{comm, tl_rank, dest, tag}].push_back(std::move(payload));
    }
    box.cv.notify_all();
    return MPI_SUCCESS;
}

int MPI_Irecv(void* buffer, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request* request) {
    if (source == MPI_PROC_NULL) { *request = MPI_REQUEST_NULL; return MPI_SUCCESS; }
    auto* state = new RequestState();
    state->receive = true;
    state->buffer = buffer;
    state->capacity = static_cast<std::size_t>(count) * type_size(type);
    state->source = source;
    state->tag = tag;
    state->comm = comm;
    *request = reinterpret_cast<MPI_Request>(state);
    return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request* request, MPI_Status* status) {
    if (*request == MPI_REQUEST_NULL) return MPI_SUCCESS;
    auto* state = reinterpret_cast<RequestState*>(*request);
    shim_world* w = world();
    std::vector<char> payload;
    {
        Mailbox& box = *w->boxes[static_cast<std::size_t>(tl_rank)];
        std::unique_lock<std::mutex> lock(box.mutex);
        const MailKey key{state->comm, state->source, tl_rank, state->tag};
        box.cv.wait(lock, [&] {
            auto found = box.mail.find(key);
            return found != box.mail.end() && !found->second.empty();
        });
        auto& queue = box.mail[key];
        payload = std::move(queue.front());
        queue.pop_front();
    }
    if (payload.size() > state->capacity) {
        std::fprintf(stderr, "mpi shim: message truncated (%zu > %zu bytes)\n",
                     payload.size(), state->capacity);
        std::abort();
    }
    if (!payload.empty()) std::memcpy(state->buffer, payload.data(), payload.size());
    if (status) {
        status->MPI_SOURCE = state->source;
        status->MPI_TAG = state->tag;
        status->MPI_ERROR = MPI_SUCCESS;
        status->bytes = payload.size();
    }
    delete state;
    *request = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request* requests, MPI_Status* statuses) {
    for (int i = 0; i < count; ++i) {
        MPI_Wait(&requests[i], statuses ? &statuses[i] : MPI_STATUS_IGNORE);
    }
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    collective(comm, nullptr, nullptr, nullptr,
               [](auto&, auto&, auto&) {});
    return MPI_SUCCESS;
}

int MPI_Bcast(void* buffer, int count, MPI_Datatype type, int root,
              MPI_Comm comm) {
    const std::size_t bytes = static_cast<std::size_t>(count) * type_size(type);
    collective(comm, buffer, nullptr, nullptr,
               [&](auto& a, auto&, auto&) {
                   if (tl_rank != root && bytes)
                       std::memcpy(buffer, a[static_cast<std::size_t>(root)], bytes);
               });
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void* send, void* receive, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
    const std::size_t bytes = static_cast<std::size_t>(count) * type_size(type);
    std::vector<char> result(bytes);
    collective(comm, send, nullptr, nullptr, [&](auto& a, auto&, auto&) {
        if (bytes) std::memcpy(result.data(), a[0], bytes);
        for (std::size_t r = 1; r < a.size(); ++r)
            reduce_typed(result.data(), a[r], count, type, op);
    });
    if (bytes) std::memcpy(receive, result.data(), bytes);
    return MPI_SUCCESS;
}

int MPI_Reduce(const void* send, void* receive, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm) {
    const std::size_t bytes = static_cast<std::size_t>(count) * type_size(type);
    std::vector<char> result(bytes);
    collective(comm, send, nullptr, nullptr, [&](auto& a, auto&, auto&) {
        if (tl_rank != root) return;
        if (bytes) std::memcpy(result.data(), a[0], bytes);
        for (std::size_t r = 1; r < a.size(); ++r)
            reduce_typed(result.data(), a[r], count, type, op);
    });
    if (tl_rank == root && bytes) std::memcpy(receive, result.data(), bytes);
    return MPI_SUCCESS;
}

int MPI_Allgather(const void* send, int send_count, MPI_Datatype send_type,
                  void* receive, int, MPI_Datatype, MPI_Comm comm) {
    const std::size_t bytes = static_cast<std::size_t>(send_count) * type_size(send_type);
    collective(comm, send, nullptr, nullptr, [&](auto& a, auto&, auto&) {
        for (std::size_t r = 0; r < a.size(); ++r)
            if (bytes) std::memcpy(static_cast<char*>(receive) + r * bytes, a[r], bytes);
    });
    return MPI_SUCCESS;
}

int MPI_Allgatherv(const void* send, int send_count, MPI_Datatype send_type,
                   void* receive, const int* receive_counts,
                   const int* displacements, MPI_Datatype receive_type,
                   MPI_Comm comm) {
    const std::size_t element = type_size(receive_type);
    (void)send_count; (void)send_type;
    collective(comm, send, nullptr, nullptr, [&](auto& a, auto&, auto&) {
        for (std::size_t r = 0; r < a.size(); ++r) {
            const std::size_t bytes = static_cast<std::size_t>(receive_counts[r]) * element;
            if (bytes)
                std::memcpy(static_cast<char*>(receive) +
                                static_cast<std::size_t>(displacements[r]) * element,
                            a[r], bytes);
        }
    });
    return MPI_SUCCESS;
}

int MPI_Alltoall(const void* send, int send_count, MPI_Datatype send_type,
                 void* receive, int, MPI_Datatype, MPI_Comm comm) {
    const std::size_t bytes = static_cast<std::size_t>(send_count) * type_size(send_type);
    collective(comm, send, nullptr, nullptr, [&](auto& a, auto&, auto&) {
        const std::size_t me = static_cast<std::size_t>(comm == MPI_COMM_SELF ? 0 : tl_rank);
        for (std::size_t r = 0; r < a.size(); ++r)
            if (bytes)
                std::memcpy(static_cast<char*>(receive) + r * bytes,
                            static_cast<const char*>(a[r]) + me * bytes, bytes);
    });
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void* send, const int* send_counts,
                  const int* send_displacements, MPI_Datatype send_type,
                  void* receive, const int* receive_counts,
                  const int* receive_displacements, MPI_Datatype receive_type,
                  MPI_Comm comm) {
    const std::size_t send_element = type_size(send_type);
    const std::size_t receive_element = type_size(receive_type);
    collective(comm, send, send_counts, send_displacements,
               [&](auto& a, auto& b, auto& c) {
        const std::size_t me = static_cast<std::size_t>(comm == MPI_COMM_SELF ? 0 : tl_rank);
        for (std::size_t r = 0; r < a.size(); ++r) {
            const int* their_counts = static_cast<const int*>(b[r]);
            const int* their_displacements = static_cast<const int*>(c[r]);
            const std::size_t bytes = static_cast<std::size_t>(their_counts[me]) * send_element;
            if (bytes != static_cast<std::size_t>(receive_counts[r]) * receive_element) {
                std::fprintf(stderr, "mpi shim: Alltoallv count mismatch\n");
                std::abort();
            }
            if (bytes)
                std::memcpy(static_cast<char*>(receive) +
                                static_cast<std::size_t>(receive_displacements[r]) * receive_element,
                            static_cast<const char*>(a[r]) +
                                static_cast<std::size_t>(their_displacements[me]) * send_element,
                            bytes);
        }
    });
    return MPI_SUCCESS;
}

}  // extern "C"
