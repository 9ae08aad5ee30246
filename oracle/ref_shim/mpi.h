// Single-rank stand-in for the part of the MPI API that the reference's grid,
// halo-buffer and execution-manager headers call, so that those headers
// compile unmodified into the parity checker (oracle/_ref).  Test
// infrastructure only: one process is rank 0 of a world of size 1, and every
// point-to-point message goes to a process-local queue that the matching
// receive drains (the reference exchanges periodic halos with itself this
// way).  Collectives copy the send buffer to the receive buffer.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Op;
// A datatype is its size in bytes: the queue only copies bytes.
typedef int MPI_Datatype;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE (reinterpret_cast<void*>(static_cast<std::intptr_t>(-1)))

#define MPI_CHAR ((MPI_Datatype)sizeof(char))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_LONG_DOUBLE ((MPI_Datatype)sizeof(long double))
#define MPI_CXX_BOOL ((MPI_Datatype)sizeof(bool))
#define MPI_INT8_T ((MPI_Datatype)1)
#define MPI_UINT8_T ((MPI_Datatype)1)
#define MPI_INT16_T ((MPI_Datatype)2)
#define MPI_UINT16_T ((MPI_Datatype)2)
#define MPI_INT32_T ((MPI_Datatype)4)
#define MPI_UINT32_T ((MPI_Datatype)4)
#define MPI_INT64_T ((MPI_Datatype)8)
#define MPI_UINT64_T ((MPI_Datatype)8)
#define MPI_LONG_LONG_INT ((MPI_Datatype)sizeof(long long))
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)sizeof(unsigned long long))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LAND 4

struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    std::size_t bytes;
};
#define MPI_STATUS_IGNORE (static_cast<MPI_Status*>(nullptr))
#define MPI_STATUSES_IGNORE (static_cast<MPI_Status*>(nullptr))

namespace dare_ref_shim {
struct Message {
    int tag;
    std::vector<char> bytes;
};
struct PendingRecv {
    void* buf;
    std::size_t cap;
    int tag;
};
inline std::deque<Message>& queue() {
    static std::deque<Message> q;
    return q;
}
inline bool take(int tag, void* buf, std::size_t cap, MPI_Status* st) {
    auto& q = queue();
    for (auto it = q.begin(); it != q.end(); ++it) {
        if (tag != MPI_ANY_TAG && it->tag != tag) continue;
        if (it->bytes.size() > cap) {
            std::fprintf(stderr, "mpi shim: message of %zu bytes for a %zu-byte buffer\n", it->bytes.size(), cap);
            std::abort();
        }
        if (!it->bytes.empty()) std::memcpy(buf, it->bytes.data(), it->bytes.size());
        if (st) {
            st->MPI_SOURCE = 0;
            st->MPI_TAG = it->tag;
            st->MPI_ERROR = MPI_SUCCESS;
            st->bytes = it->bytes.size();
        }
        q.erase(it);
        return true;
    }
    return false;
}
}  // namespace dare_ref_shim

// A request is either a completed send (nullptr) or a pending receive.
typedef dare_ref_shim::PendingRecv* MPI_Request;

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Initialized(int* flag) {
    *flag = 1;
    return MPI_SUCCESS;
}
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}
[[noreturn]] inline int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "mpi shim: MPI_Abort(%d)\n", code);
    std::abort();
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Dims_create(int, int ndims, int* dims) {
    for (int d = 0; d < ndims; d++)
        if (dims[d] == 0) dims[d] = 1;
    return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm = 0) {
    if (send != MPI_IN_PLACE && count > 0) std::memmove(recv, send, (std::size_t)count * type);
    return MPI_SUCCESS;
}
inline int MPI_Allgather(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype,
                         MPI_Comm) {
    if (send != MPI_IN_PLACE && scount > 0) std::memmove(recv, send, (std::size_t)scount * stype);
    return MPI_SUCCESS;
}
inline int MPI_Send(const void* buf, int count, MPI_Datatype type, int, int tag, MPI_Comm) {
    const char* p = static_cast<const char*>(buf);
    dare_ref_shim::queue().push_back({tag, std::vector<char>(p, p + (std::size_t)count * type)});
    return MPI_SUCCESS;
}
inline int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
                     MPI_Request* req) {
    *req = nullptr;
    return MPI_Send(buf, count, type, dest, tag, comm);
}
inline int MPI_Recv(void* buf, int count, MPI_Datatype type, int, int tag, MPI_Comm, MPI_Status* st) {
    if (!dare_ref_shim::take(tag, buf, (std::size_t)count * type, st)) {
        std::fprintf(stderr, "mpi shim: receive with tag %d has no message (single rank)\n", tag);
        std::abort();
    }
    return MPI_SUCCESS;
}
inline int MPI_Irecv(void* buf, int count, MPI_Datatype type, int, int tag, MPI_Comm, MPI_Request* req) {
    *req = new dare_ref_shim::PendingRecv{buf, (std::size_t)count * type, tag};
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request* req, MPI_Status* st) {
    if (*req) {
        if (!dare_ref_shim::take((*req)->tag, (*req)->buf, (*req)->cap, st)) {
            std::fprintf(stderr, "mpi shim: wait on a receive with tag %d that has no message\n", (*req)->tag);
            std::abort();
        }
        delete *req;
        *req = nullptr;
    }
    return MPI_SUCCESS;
}
inline int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* st) {
    for (int i = 0; i < count; i++) MPI_Wait(&reqs[i], st ? &st[i] : MPI_STATUS_IGNORE);
    return MPI_SUCCESS;
}
inline int MPI_Probe(int, int tag, MPI_Comm, MPI_Status* st) {
    for (const auto& m : dare_ref_shim::queue())
        if (tag == MPI_ANY_TAG || m.tag == tag) {
            if (st) {
                st->MPI_SOURCE = 0;
                st->MPI_TAG = m.tag;
                st->MPI_ERROR = MPI_SUCCESS;
                st->bytes = m.bytes.size();
            }
            return MPI_SUCCESS;
        }
    std::fprintf(stderr, "mpi shim: probe for tag %d finds no message (single rank)\n", tag);
    std::abort();
}
inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype type, int* count) {
    *count = (int)(st->bytes / (std::size_t)type);
    return MPI_SUCCESS;
}
