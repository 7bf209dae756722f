// Single-node MPI shim used ONLY to compile and run the unmodified reference
// headers as a test oracle / CPU baseline (MPI is not installed on these
// machines).  It is test infrastructure: nothing in the product links it.
//
// It implements exactly the MPI surface the reference touches
// (mpi_util.hpp:21-157, distributed.hpp:37-237, timer.hpp:25-37, and the
// driver's own MPI_Allreduce of U as in main.cpp:62):
//   Init/Finalize/Finalized, Comm_size/rank/split_type/split/free, Barrier,
//   Allreduce, Scan, Bcast, Allgather, Allgatherv,
//   Win_allocate_shared/shared_query/free/sync.
//
// Ranks: MPI_Init forks SIMPLEFMM_SHIM_NP - 1 child processes (default 1 =
// no fork).  All ranks live on one node, so MPI_COMM_TYPE_SHARED splits give
// "all ranks" and the node-root split gives a one-member communicator.
// Shared windows and collective scratch live in one MAP_SHARED anonymous
// arena mapped before the fork; allocation is a deterministic bump pointer
// (every rank performs the same collective allocations in the same order).
// Collectives spin on process-shared atomics with a wall-clock limit and
// abort the job (never hang) when a peer disappears.
#ifndef SIMPLEFMM_MPI_SHIM_H
#define SIMPLEFMM_MPI_SHIM_H

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sched.h>
#include <sys/mman.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <unistd.h>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Win;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long MPI_Aint;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_WIN_NULL 0
#define MPI_INFO_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_COMM_TYPE_SHARED 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_IN_PLACE ((void*)1)

#define MPI_DATATYPE_NULL 0
#define MPI_INT 1
#define MPI_INT64_T 2
#define MPI_UNSIGNED_CHAR 3
#define MPI_UNSIGNED_SHORT 4
#define MPI_UNSIGNED 5
#define MPI_UNSIGNED_LONG 6
#define MPI_UNSIGNED_LONG_LONG 7
#define MPI_FLOAT 8
#define MPI_DOUBLE 9
#define MPI_LONG 10

namespace mpishim {

struct Shared {                       // lives at the start of the arena
    std::atomic<int> bar_count;
    std::atomic<int> bar_sense;
    std::atomic<int> abort_flag;
    int np;
    int64_t slot_i64[1024];           // per-rank integer exchange slots
};

struct State {
    int np = 1;
    int rank = 0;
    bool initialized = false;
    bool finalized = false;
    char* arena = nullptr;
    size_t arena_size = 0;
    size_t bump = 0;                  // identical on every rank
    int local_sense = 0;
    std::vector<pid_t> children;
    // communicators: id -> (size, rank); 1 = world; created ids are per-process
    // counters advanced identically on every rank.
    std::vector<std::pair<int, int>> comms;
    // windows: id -> (base offset of rank-0 segment, owned malloc ptr)
    struct Win { char* base0; void* owned; size_t off; size_t len; };
    std::vector<Win> wins;
};

inline State& st() { static State s; return s; }
inline Shared* sh() { return reinterpret_cast<Shared*>(st().arena); }

inline size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_INT64_T: return 8;
    case MPI_UNSIGNED_CHAR: return 1;
    case MPI_UNSIGNED_SHORT: return 2;
    case MPI_UNSIGNED: return 4;
    case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
    case MPI_UNSIGNED_LONG_LONG: return 8;
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_LONG: return sizeof(long);
    default: return 0;
    }
}

[[noreturn]] inline void die(const char* what)
{
    std::fprintf(stderr, "mpi shim: %s (rank %d)\n", what, st().rank);
    if (st().arena) sh()->abort_flag.store(1);
    std::_Exit(70);
}

inline double timeout_s()
{
    const char* e = std::getenv("SIMPLEFMM_SHIM_TIMEOUT");
    return e ? std::atof(e) : 3600.0;
}

inline void barrier_all()
{
    State& s = st();
    if (s.np == 1) return;
    Shared* h = sh();
    s.local_sense ^= 1;
    if (h->bar_count.fetch_add(1) + 1 == s.np) {
        h->bar_count.store(0);
        h->bar_sense.store(s.local_sense);
        return;
    }
    const auto t0 = std::chrono::steady_clock::now();
    long spins = 0;
    while (h->bar_sense.load() != s.local_sense) {
        if (h->abort_flag.load()) die("peer aborted");
        if (++spins % 1024 == 0) {
            sched_yield();
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (dt > timeout_s()) die("barrier timeout");
        }
    }
}

inline std::pair<int, int> comm_info(MPI_Comm c)
{
    State& s = st();
    if (c == MPI_COMM_WORLD) return {s.np, s.rank};
    if (c >= 2 && static_cast<size_t>(c - 2) < s.comms.size()) return s.comms[c - 2];
    die("invalid communicator");
}

inline MPI_Comm new_comm(int size, int rank)
{
    st().comms.push_back({size, rank});
    return static_cast<MPI_Comm>(st().comms.size() + 1);
}

// bump-allocate `len` bytes of arena (same offset on every rank)
inline size_t arena_alloc(size_t len)
{
    State& s = st();
    const size_t off = (s.bump + 4095) & ~size_t(4095);
    if (off + len > s.arena_size) die("arena exhausted (raise SIMPLEFMM_SHIM_ARENA_GB)");
    s.bump = off + len;
    return off;
}

template<typename T>
inline void reduce_into(T* dst, const T* src, size_t n, MPI_Op op)
{
    for (size_t i = 0; i < n; ++i) {
        if (op == MPI_SUM) dst[i] += src[i];
        else if (op == MPI_MAX) dst[i] = dst[i] < src[i] ? src[i] : dst[i];
        else if (op == MPI_MIN) dst[i] = dst[i] > src[i] ? src[i] : dst[i];
    }
}

inline void reduce_typed(void* dst, const void* src, size_t n, MPI_Datatype t, MPI_Op op)
{
    switch (t) {
    case MPI_INT: reduce_into((int*)dst, (const int*)src, n, op); break;
    case MPI_INT64_T: reduce_into((int64_t*)dst, (const int64_t*)src, n, op); break;
    case MPI_UNSIGNED: reduce_into((unsigned*)dst, (const unsigned*)src, n, op); break;
    case MPI_UNSIGNED_LONG: reduce_into((unsigned long*)dst, (const unsigned long*)src, n, op); break;
    case MPI_UNSIGNED_LONG_LONG: reduce_into((unsigned long long*)dst, (const unsigned long long*)src, n, op); break;
    case MPI_LONG: reduce_into((long*)dst, (const long*)src, n, op); break;
    case MPI_FLOAT: reduce_into((float*)dst, (const float*)src, n, op); break;
    case MPI_DOUBLE: reduce_into((double*)dst, (const double*)src, n, op); break;
    default: die("unsupported reduction type");
    }
}

}  // namespace mpishim

inline int MPI_Init(int*, char***)
{
    using namespace mpishim;
    State& s = st();
    const char* e = std::getenv("SIMPLEFMM_SHIM_NP");
    s.np = e ? std::atoi(e) : 1;
    if (s.np < 1 || s.np > 1024) s.np = 1;
    s.initialized = true;
    if (s.np == 1) return MPI_SUCCESS;
    const char* g = std::getenv("SIMPLEFMM_SHIM_ARENA_GB");
    s.arena_size = static_cast<size_t>(g ? std::atof(g) : 256.0) << 30;
    void* a = mmap(nullptr, s.arena_size, PROT_READ | PROT_WRITE,
                   MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (a == MAP_FAILED) die("arena mmap failed");
    s.arena = static_cast<char*>(a);
    Shared* h = sh();
    h->bar_count.store(0);
    h->bar_sense.store(0);
    h->abort_flag.store(0);
    h->np = s.np;
    s.bump = sizeof(Shared);
    std::fflush(nullptr);
    for (int r = 1; r < s.np; ++r) {
        const pid_t pid = fork();
        if (pid < 0) die("fork failed");
        if (pid == 0) {
            s.rank = r;
            s.children.clear();
            return MPI_SUCCESS;
        }
        s.children.push_back(pid);
    }
    return MPI_SUCCESS;
}

inline int MPI_Finalized(int* flag)
{
    *flag = mpishim::st().finalized ? 1 : 0;
    return MPI_SUCCESS;
}

inline int MPI_Finalize()
{
    using namespace mpishim;
    State& s = st();
    barrier_all();
    s.finalized = true;
    if (s.np > 1) {
        if (s.rank != 0) {
            std::fflush(nullptr);
            std::_Exit(0);
        }
        int bad = 0;
        for (pid_t pid : s.children) {
            int status = 0;
            waitpid(pid, &status, 0);
            if (!WIFEXITED(status) || WEXITSTATUS(status) != 0) bad = 1;
        }
        if (bad) die("a child rank failed");
    }
    return MPI_SUCCESS;
}

inline int MPI_Comm_size(MPI_Comm c, int* size) { *size = mpishim::comm_info(c).first; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm c, int* rank) { *rank = mpishim::comm_info(c).second; return MPI_SUCCESS; }

inline int MPI_Comm_split_type(MPI_Comm c, int, int, MPI_Info, MPI_Comm* out)
{
    // one node: the shared-memory communicator has the parent's membership
    const auto ci = mpishim::comm_info(c);
    *out = mpishim::new_comm(ci.first, ci.second);
    return MPI_SUCCESS;
}

inline int MPI_Barrier(MPI_Comm c)
{
    const auto ci = mpishim::comm_info(c);
    if (ci.first > 1) mpishim::barrier_all();
    return MPI_SUCCESS;
}

// Exchange one int64 per rank of an all-ranks communicator.
inline std::vector<int64_t> mpishim_allgather_i64(int64_t v)
{
    using namespace mpishim;
    State& s = st();
    std::vector<int64_t> out(s.np);
    if (s.np == 1) { out[0] = v; return out; }
    barrier_all();
    sh()->slot_i64[s.rank] = v;
    barrier_all();
    for (int r = 0; r < s.np; ++r) out[r] = sh()->slot_i64[r];
    barrier_all();
    return out;
}

inline int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm* out)
{
    using namespace mpishim;
    const auto ci = comm_info(c);
    if (ci.first == 1) {
        *out = color == MPI_UNDEFINED ? MPI_COMM_NULL : new_comm(1, 0);
        return MPI_SUCCESS;
    }
    if (ci.first != st().np) die("split of a partial communicator is unsupported");
    const auto colors = mpishim_allgather_i64(color);
    const auto keys = mpishim_allgather_i64(key);
    int size = 0, rank = 0;
    for (int r = 0; r < st().np; ++r) {
        if (colors[r] == color && color != MPI_UNDEFINED) {
            if (keys[r] < key || (keys[r] == key && r < st().rank)) ++rank;
            ++size;
        }
    }
    if (color == MPI_UNDEFINED) {
        st().comms.push_back({0, 0});          // keep ids aligned across ranks
        *out = MPI_COMM_NULL;
        return MPI_SUCCESS;
    }
    if (size != 1 && size != st().np) die("split into partial groups is unsupported");
    *out = new_comm(size, rank);
    return MPI_SUCCESS;
}

inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }

inline int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    using namespace mpishim;
    const size_t ts = type_size(t);
    const size_t bytes = ts * static_cast<size_t>(count);
    if (sendbuf != MPI_IN_PLACE) std::memmove(recvbuf, sendbuf, bytes);
    const auto ci = comm_info(c);
    if (ci.first == 1 || count == 0) return MPI_SUCCESS;
    State& s = st();
    // chunked reduce-scatter + allgather through the arena
    const size_t chunk = size_t(8) << 20;
    const size_t saved = s.bump;
    const size_t slots = arena_alloc(chunk * s.np);
    const size_t res = arena_alloc(chunk);
    char* base = s.arena;
    for (size_t done = 0; done < bytes; done += chunk) {
        const size_t len = bytes - done < chunk ? bytes - done : chunk;
        std::memcpy(base + slots + chunk * s.rank, static_cast<char*>(recvbuf) + done, len);
        barrier_all();
        const size_t n = len / ts;
        const size_t b = n * s.rank / s.np, e = n * (s.rank + 1) / s.np;
        char* out = base + res + b * ts;
        std::memcpy(out, base + slots + b * ts, (e - b) * ts);
        for (int r = 1; r < s.np; ++r)
            reduce_typed(out, base + slots + chunk * r + b * ts, e - b, t, op);
        barrier_all();
        std::memcpy(static_cast<char*>(recvbuf) + done, base + res, len);
        barrier_all();
    }
    madvise(base + slots, chunk * (s.np + 1) + 4096, MADV_REMOVE);
    s.bump = saved;
    return MPI_SUCCESS;
}

inline int MPI_Scan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    using namespace mpishim;
    const size_t ts = type_size(t);
    std::memmove(recvbuf, sendbuf, ts * count);
    const auto ci = comm_info(c);
    if (ci.first == 1) return MPI_SUCCESS;
    if (count != 1 || (t != MPI_INT && t != MPI_INT64_T)) die("MPI_Scan: only scalar ints supported");
    int64_t v = t == MPI_INT ? *static_cast<int*>(recvbuf) : *static_cast<int64_t*>(recvbuf);
    const auto all = mpishim_allgather_i64(v);
    int64_t acc = all[0];
    for (int r = 1; r <= st().rank; ++r) {
        if (op == MPI_SUM) acc += all[r];
        else if (op == MPI_MAX) acc = acc < all[r] ? all[r] : acc;
        else acc = acc > all[r] ? all[r] : acc;
    }
    if (t == MPI_INT) *static_cast<int*>(recvbuf) = static_cast<int>(acc);
    else *static_cast<int64_t*>(recvbuf) = acc;
    return MPI_SUCCESS;
}

inline int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm c)
{
    using namespace mpishim;
    const auto ci = comm_info(c);
    if (ci.first == 1) return MPI_SUCCESS;
    State& s = st();
    const size_t bytes = type_size(t) * static_cast<size_t>(count);
    const size_t saved = s.bump;
    const size_t off = arena_alloc(bytes);
    barrier_all();
    if (s.rank == root) std::memcpy(s.arena + off, buf, bytes);
    barrier_all();
    if (s.rank != root) std::memcpy(buf, s.arena + off, bytes);
    barrier_all();
    s.bump = saved;
    return MPI_SUCCESS;
}

inline int MPI_Allgatherv(const void* sendbuf, int, MPI_Datatype, void* recvbuf, const int* counts,
                          const int* displs, MPI_Datatype t, MPI_Comm c)
{
    using namespace mpishim;
    const auto ci = comm_info(c);
    const size_t ts = type_size(t);
    State& s = st();
    if (ci.first == 1) {
        if (sendbuf != MPI_IN_PLACE) std::memmove(static_cast<char*>(recvbuf) + displs[0] * ts, sendbuf, counts[0] * ts);
        return MPI_SUCCESS;
    }
    size_t total = 0;
    for (int r = 0; r < s.np; ++r) total = total > size_t(displs[r] + counts[r]) ? total : size_t(displs[r] + counts[r]);
    const size_t saved = s.bump;
    const size_t off = arena_alloc(total * ts);
    const char* mine = sendbuf == MPI_IN_PLACE ? static_cast<char*>(recvbuf) + displs[s.rank] * ts
                                               : static_cast<const char*>(sendbuf);
    barrier_all();
    std::memcpy(s.arena + off + displs[s.rank] * ts, mine, counts[s.rank] * ts);
    barrier_all();
    std::memcpy(recvbuf, s.arena + off, total * ts);
    barrier_all();
    s.bump = saved;
    return MPI_SUCCESS;
}

inline int MPI_Allgather(const void* sendbuf, int count, MPI_Datatype t, void* recvbuf, int, MPI_Datatype, MPI_Comm c)
{
    const auto ci = mpishim::comm_info(c);
    std::vector<int> counts(ci.first, count), displs(ci.first);
    for (int r = 0; r < ci.first; ++r) displs[r] = r * count;
    return MPI_Allgatherv(sendbuf, count, t, recvbuf, counts.data(), displs.data(), t, c);
}

inline int MPI_Win_allocate_shared(MPI_Aint size, int, MPI_Info, MPI_Comm c, void* baseptr, MPI_Win* win)
{
    using namespace mpishim;
    State& s = st();
    const auto ci = comm_info(c);
    State::Win w{nullptr, nullptr, 0, 0};
    if (ci.first == 1) {
        const size_t len = size > 0 ? static_cast<size_t>(size) : 1;
        w.owned = std::aligned_alloc(64, (len + 63) & ~size_t(63));
        if (!w.owned) die("window allocation failed");
        w.base0 = static_cast<char*>(w.owned);
        *static_cast<void**>(baseptr) = w.owned;
    } else {
        if (ci.first != s.np) die("window over a partial communicator is unsupported");
        const auto sizes = mpishim_allgather_i64(size);
        size_t total = 0;
        std::vector<size_t> offs(s.np);
        for (int r = 0; r < s.np; ++r) { offs[r] = total; total += (static_cast<size_t>(sizes[r]) + 63) & ~size_t(63); }
        const size_t off = arena_alloc(total ? total : 64);
        w.off = off;
        w.len = total;
        w.base0 = s.arena + off + offs[0];
        *static_cast<void**>(baseptr) = s.arena + off + offs[s.rank];
        barrier_all();
    }
    s.wins.push_back(w);
    *win = static_cast<MPI_Win>(s.wins.size());
    return MPI_SUCCESS;
}

inline int MPI_Win_shared_query(MPI_Win win, int rank, MPI_Aint* size, int* disp, void* baseptr)
{
    using namespace mpishim;
    if (win <= 0 || static_cast<size_t>(win) > st().wins.size()) die("invalid window");
    if (rank != 0) die("shared_query of a non-root segment is unsupported");
    *size = 0;
    *disp = 1;
    *static_cast<void**>(baseptr) = st().wins[win - 1].base0;
    return MPI_SUCCESS;
}

inline int MPI_Win_free(MPI_Win* win)
{
    using namespace mpishim;
    State& s = st();
    if (*win > 0 && static_cast<size_t>(*win) <= s.wins.size()) {
        State::Win& w = s.wins[*win - 1];
        if (w.owned) {
            std::free(w.owned);
        } else if (w.len) {
            barrier_all();                    // MPI_Win_free is collective
            if (s.rank == 0) madvise(s.arena + w.off, w.len, MADV_REMOVE);
            barrier_all();
        }
        w = State::Win{nullptr, nullptr, 0, 0};
    }
    *win = MPI_WIN_NULL;
    return MPI_SUCCESS;
}

inline int MPI_Win_sync(MPI_Win) { std::atomic_thread_fence(std::memory_order_seq_cst); return MPI_SUCCESS; }

#endif
