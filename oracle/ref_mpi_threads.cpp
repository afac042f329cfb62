// Thread-backed stand-ins for the MPI routines the reference's Index.cpp and
// node.cpp call, so that its multi-rank modes (GROUP: src/Index.cpp:1053-1187
// with src/node.cpp:679-1203) run inside one process with each rank on its
// own thread.  TEST INFRASTRUCTURE ONLY: the CPU baseline and the tests use
// it through oracle/ref_capi.cpp; the product never links it.
//
// Semantics kept from MPI: point-to-point messages between a pair of ranks
// with the same tag arrive in send order, and a receive matches the earliest
// message whose tag it names; receives posted first (MPI_Irecv, or a
// blocking MPI_Recv) are matched first.  Sends are buffered (the data is
// copied at the call), so MPI_Send and MPI_Isend complete at once.
// Collectives (MPI_Bcast, MPI_Barrier) use their own channels, so they never
// match point-to-point traffic.  Every wait gives up after WAIT_S seconds
// with an error rather than blocking forever (600 s, or HY_REF_MPI_WAIT_S).
//
// ref_mpi_threads_init(size) sets the number of ranks (1 before it is
// called: a single-rank world in which barriers pass and broadcasts are
// no-ops); ref_mpi_threads_bind(rank) tells the calling thread its rank.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <vector>

#include "mpi.h"

namespace {

// Seconds a wait gives up after (HY_REF_MPI_WAIT_S overrides).
double wait_s() {
    static const double s = [] {
        const char* e = std::getenv("HY_REF_MPI_WAIT_S");
        return e ? std::atof(e) : 600.0;
    }();
    return s;
}

size_t type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_BYTE: return 1;
        case MPI_INT: return 4;
        case MPI_FLOAT: return 4;
        case MPI_DOUBLE: return 8;
        case MPI_INT64_T: return 8;
        default:
            std::fprintf(stderr, "oracle MPI: unknown datatype %d\n", t);
            std::abort();
    }
}

struct Req {
    bool recv = false;
    void* buf = nullptr;
    size_t bytes = 0;
    int tag = 0;
    bool done = false;
};

struct Msg {
    int tag;
    std::vector<char> data;
};

// One direction between two ranks: messages not yet received and receives
// not yet matched, each in arrival / post order.
struct Channel {
    std::deque<Msg> unexpected;
    std::deque<Req*> posted;
};

struct World {
    int size = 1;
    std::mutex mu;
    std::condition_variable cv;
    std::vector<Channel> p2p, coll;  // [src * size + dst]
    // barrier
    int arrived = 0;
    unsigned long long generation = 0;
    // requests handed out as MPI_Request (int) handles
    std::vector<std::unique_ptr<Req>> reqs;
    std::vector<int> free_ids;
};

World g;
thread_local int t_rank = 0;

// Matching happens under g.mu, in order; the bytes are copied outside it so
// that ranks exchanging large buffers do not serialise on the lock.

// Send on chans[t_rank -> dst]: the data is copied first; a receive already
// posted with the tag takes it, else it queues.  Caller does not hold g.mu.
void post_send(std::vector<Channel>& chans, int dst, int tag, const void* buf, size_t bytes) {
    std::vector<char> data(bytes);
    if (bytes) std::memcpy(data.data(), buf, bytes);
    Req* match = nullptr;
    {
        std::lock_guard<std::mutex> lk(g.mu);
        Channel& c = chans[static_cast<size_t>(t_rank) * g.size + dst];
        for (auto it = c.posted.begin(); it != c.posted.end(); ++it)
            if ((*it)->tag == tag) {
                match = *it;
                c.posted.erase(it);
                break;
            }
        if (!match) {
            c.unexpected.push_back(Msg{tag, std::move(data)});
            g.cv.notify_all();
            return;
        }
    }
    std::memcpy(match->buf, data.data(), bytes < match->bytes ? bytes : match->bytes);
    std::lock_guard<std::mutex> lk(g.mu);
    match->done = true;
    g.cv.notify_all();
}

// Post receive r on chans[src -> t_rank]: the earliest queued message with
// its tag is copied in now, else r waits for a send.  Caller does not hold
// g.mu.
void post_recv(std::vector<Channel>& chans, int src, Req* r) {
    Msg m{0, {}};
    bool got = false;
    {
        std::lock_guard<std::mutex> lk(g.mu);
        Channel& c = chans[static_cast<size_t>(src) * g.size + t_rank];
        for (auto it = c.unexpected.begin(); it != c.unexpected.end(); ++it)
            if (it->tag == r->tag) {
                m = std::move(*it);
                c.unexpected.erase(it);
                got = true;
                break;
            }
        if (!got) {
            c.posted.push_back(r);
            return;
        }
    }
    std::memcpy(r->buf, m.data.data(), m.data.size() < r->bytes ? m.data.size() : r->bytes);
    std::lock_guard<std::mutex> lk(g.mu);
    r->done = true;
}

// Waits (caller holds g.mu through lk) until r is matched; on giving up,
// r is withdrawn from every channel so no later send writes through it.
int wait_done(std::unique_lock<std::mutex>& lk, Req* r) {
    const bool ok = g.cv.wait_for(lk, std::chrono::duration<double>(wait_s()), [&] { return r->done; });
    if (!ok) {
        for (auto* chans : {&g.p2p, &g.coll})
            for (Channel& c : *chans)
                for (auto it = c.posted.begin(); it != c.posted.end();)
                    it = (*it == r) ? c.posted.erase(it) : it + 1;
        std::fprintf(stderr, "oracle MPI: rank %d gave up waiting for a message (tag %d)\n", t_rank, r->tag);
        return 1;
    }
    return 0;
}

bool valid_rank(int r) { return r >= 0 && r < g.size; }

int new_request(Req** out) {
    int id;
    if (!g.free_ids.empty()) {
        id = g.free_ids.back();
        g.free_ids.pop_back();
        g.reqs[id] = std::make_unique<Req>();
    } else {
        id = static_cast<int>(g.reqs.size());
        g.reqs.push_back(std::make_unique<Req>());
    }
    *out = g.reqs[id].get();
    return id + 1;  // 0 is the null request
}

void release(MPI_Request* req) {
    const int id = *req - 1;
    g.reqs[id].reset();
    g.free_ids.push_back(id);
    *req = 0;
}

}  // namespace

extern "C" {

void ref_mpi_threads_init(int size) {
    std::lock_guard<std::mutex> lk(g.mu);
    g.size = size < 1 ? 1 : size;
    g.p2p.assign(static_cast<size_t>(g.size) * g.size, Channel{});
    g.coll.assign(static_cast<size_t>(g.size) * g.size, Channel{});
    g.arrived = 0;
    g.reqs.clear();
    g.free_ids.clear();
}

void ref_mpi_threads_bind(int rank) { t_rank = rank; }

int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "oracle MPI: MPI_Abort(%d) on rank %d\n", code, t_rank);
    std::abort();
}

int MPI_Comm_get_attr(MPI_Comm, int, void*, int* flag) {
    if (flag) *flag = 0;
    return 0;
}

int MPI_Barrier(MPI_Comm) {
    std::unique_lock<std::mutex> lk(g.mu);
    if (g.size <= 1) return 0;
    const unsigned long long gen = g.generation;
    if (++g.arrived == g.size) {
        g.arrived = 0;
        ++g.generation;
        g.cv.notify_all();
        return 0;
    }
    const bool ok = g.cv.wait_for(lk, std::chrono::duration<double>(wait_s()), [&] { return g.generation != gen; });
    if (!ok) std::fprintf(stderr, "oracle MPI: rank %d gave up at a barrier (%d of %d arrived)\n", t_rank, g.arrived,
                          g.size);
    return ok ? 0 : 1;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm) {
    const size_t bytes = static_cast<size_t>(count) * type_size(t);
    if (g.size <= 1) return 0;
    if (!valid_rank(root)) return 1;
    if (t_rank == root) {
        for (int r = 0; r < g.size; ++r)
            if (r != root) post_send(g.coll, r, 0, buf, bytes);
        return 0;
    }
    Req r;
    r.recv = true;
    r.buf = buf;
    r.bytes = bytes;
    post_recv(g.coll, root, &r);
    std::unique_lock<std::mutex> lk(g.mu);
    return wait_done(lk, &r);
}

int MPI_Send(const void* buf, int count, MPI_Datatype t, int dst, int tag, MPI_Comm) {
    if (!valid_rank(dst)) return 1;
    post_send(g.p2p, dst, tag, buf, static_cast<size_t>(count) * type_size(t));
    return 0;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dst, int tag, MPI_Comm, MPI_Request* req) {
    if (!valid_rank(dst)) return 1;
    post_send(g.p2p, dst, tag, buf, static_cast<size_t>(count) * type_size(t));
    std::lock_guard<std::mutex> lk(g.mu);
    Req* r;
    *req = new_request(&r);
    r->done = true;  // buffered
    return 0;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Request* req) {
    if (!valid_rank(src)) return 1;
    Req* r;
    {
        std::lock_guard<std::mutex> lk(g.mu);
        *req = new_request(&r);
    }
    r->recv = true;
    r->buf = buf;
    r->bytes = static_cast<size_t>(count) * type_size(t);
    r->tag = tag;
    post_recv(g.p2p, src, r);
    return 0;
}

int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status* st) {
    if (!valid_rank(src)) return 1;
    Req r;
    r.recv = true;
    r.buf = buf;
    r.bytes = static_cast<size_t>(count) * type_size(t);
    r.tag = tag;
    post_recv(g.p2p, src, &r);
    std::unique_lock<std::mutex> lk(g.mu);
    const int rc = wait_done(lk, &r);
    if (st) {
        st->MPI_SOURCE = src;
        st->MPI_TAG = tag;
        st->MPI_ERROR = rc;
    }
    return rc;
}

int MPI_Test(MPI_Request* req, int* flag, MPI_Status* st) {
    std::lock_guard<std::mutex> lk(g.mu);
    if (*req == 0) {
        *flag = 1;
        return 0;
    }
    Req* r = g.reqs[*req - 1].get();
    *flag = r->done ? 1 : 0;
    if (st) st->MPI_ERROR = 0;
    if (r->done) release(req);
    return 0;
}

int MPI_Wait(MPI_Request* req, MPI_Status* st) {
    std::unique_lock<std::mutex> lk(g.mu);
    if (*req == 0) return 0;
    Req* r = g.reqs[*req - 1].get();
    const int rc = wait_done(lk, r);
    if (st) st->MPI_ERROR = rc;
    if (rc == 0) release(req);
    return rc;
}

int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*) {
    int rc = 0;
    for (int i = 0; i < n; ++i) rc |= MPI_Wait(&reqs[i], MPI_STATUS_IGNORE);
    return rc;
}

}  // extern "C"
