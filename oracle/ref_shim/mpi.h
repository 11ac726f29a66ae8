/*
 * Single-rank MPI stand-in used ONLY to compile the reference's own walk engine
 * (include/walk.hpp, graph.hpp, path.hpp) and SGNS trainer (include/dsgl.hpp)
 * into the CPU checker binaries under oracle/_ref/.  Test infrastructure: nothing
 * in the shipped library includes it.
 *
 * Semantics (rank 0 of a world of size 1):
 *  - collectives copy send buffer to receive buffer (MPI_IN_PLACE is a no-op);
 *  - point-to-point messages go through one thread-safe FIFO per tag, so the
 *    reference's send/recv helper threads (graph.hpp:859-1148, path.hpp:303-358)
 *    exchange self-messages exactly as a one-process mpiexec would;
 *  - Isend is eager (the payload is copied at post time), Irecv/Recv block until
 *    a matching message exists, Probe blocks without consuming it.
 */
#ifndef DG_REF_SHIM_MPI_H
#define DG_REF_SHIM_MPI_H

#include <cstddef>
#include <cstring>
#include <cstdint>
#include <deque>
#include <map>
#include <vector>
#include <mutex>
#include <condition_variable>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; int count; };
struct MPI_Request { int done; };

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

enum { MPI_THREAD_SINGLE = 0, MPI_THREAD_FUNNELED, MPI_THREAD_SERIALIZED, MPI_THREAD_MULTIPLE };
enum { MPI_CHAR = 1, MPI_UNSIGNED_CHAR, MPI_INT, MPI_UNSIGNED, MPI_LONG, MPI_UNSIGNED_LONG,
       MPI_FLOAT, MPI_DOUBLE, MPI_LONG_LONG, MPI_UNSIGNED_LONG_LONG };
enum { MPI_SUM = 1, MPI_MAX, MPI_MIN };

namespace dg_mpi_shim {

inline size_t type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_CHAR: case MPI_UNSIGNED_CHAR: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    default: return 8;
    }
}

struct Mailbox {
    std::mutex mu;
    std::condition_variable cv;
    std::map<int, std::deque<std::vector<char> > > by_tag;
};

inline Mailbox &box() {
    static Mailbox b;
    return b;
}

inline void post(const void *buf, size_t bytes, int tag) {
    Mailbox &b = box();
    std::vector<char> msg((const char *)buf, (const char *)buf + bytes);
    {
        std::lock_guard<std::mutex> g(b.mu);
        b.by_tag[tag].push_back(std::move(msg));
    }
    b.cv.notify_all();
}

inline size_t take(void *buf, size_t cap_bytes, int tag) {
    Mailbox &b = box();
    std::unique_lock<std::mutex> g(b.mu);
    b.cv.wait(g, [&] { return !b.by_tag[tag].empty(); });
    std::vector<char> msg = std::move(b.by_tag[tag].front());
    b.by_tag[tag].pop_front();
    size_t n = msg.size() < cap_bytes ? msg.size() : cap_bytes;
    if (n) memcpy(buf, msg.data(), n);
    return n;
}

inline size_t peek(int tag) {
    Mailbox &b = box();
    std::unique_lock<std::mutex> g(b.mu);
    b.cv.wait(g, [&] { return !b.by_tag[tag].empty(); });
    return b.by_tag[tag].front().size();
}

}  // namespace dg_mpi_shim

inline int MPI_Init_thread(int *, char ***, int required, int *provided) { if (provided) *provided = required; return 0; }
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Get_processor_name(char *name, int *len) { strcpy(name, "localhost"); *len = 9; return 0; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (send != MPI_IN_PLACE && count > 0) memmove(recv, send, (size_t)count * dg_mpi_shim::type_size(t));
    return 0;
}

inline int MPI_Send(const void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm) {
    dg_mpi_shim::post(buf, (size_t)count * dg_mpi_shim::type_size(t), tag);
    return 0;
}

inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request *req) {
    MPI_Send(buf, count, t, dst, tag, c);
    req->done = 1;
    return 0;
}

inline int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status *st) {
    size_t n = dg_mpi_shim::take(buf, (size_t)count * dg_mpi_shim::type_size(t), tag);
    if (st) { st->MPI_SOURCE = src; st->MPI_TAG = tag; st->MPI_ERROR = 0; st->count = (int)n; }
    return 0;
}

inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req) {
    MPI_Recv(buf, count, t, src, tag, c, MPI_STATUS_IGNORE);
    req->done = 1;
    return 0;
}

inline int MPI_Probe(int src, int tag, MPI_Comm, MPI_Status *st) {
    size_t n = dg_mpi_shim::peek(tag);
    if (st) { st->MPI_SOURCE = src; st->MPI_TAG = tag; st->MPI_ERROR = 0; st->count = (int)n; }
    return 0;
}

inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
    *count = (int)(st->count / dg_mpi_shim::type_size(t));
    return 0;
}

inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }

#endif
