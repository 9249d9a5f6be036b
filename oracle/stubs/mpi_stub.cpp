// Single-rank, self-messaging MPI implementation for the pinning oracle build.
// Test infrastructure only: it lets the reference's unmodified sources run as
// one periodic rank so their outputs pin the oracle restatement.
#include "mpi.h"

#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct Pending {
    void *buf;
    const void *cbuf;
    size_t bytes;
    int tag;
    bool is_send;
};

std::vector<Pending> g_pending;
int g_periods[3] = {0, 0, 0};

}  // namespace

struct ns3d_mpi_abort : std::runtime_error {
    explicit ns3d_mpi_abort(int code)
        : std::runtime_error("MPI_Abort(" + std::to_string(code) + ")") {}
};

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }

int MPI_Dims_create(int, int ndims, int dims[]) {
    for (int d = 0; d < ndims; ++d) dims[d] = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm, int ndims, const int *, const int periods[], int, MPI_Comm *cart) {
    for (int d = 0; d < ndims && d < 3; ++d) g_periods[d] = periods[d];
    *cart = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm, int, int maxdims, int coords[]) {
    for (int d = 0; d < maxdims; ++d) coords[d] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm, int direction, int, int *src, int *dst) {
    int nb = g_periods[direction] ? 0 : MPI_PROC_NULL;
    *src = nb;
    *dst = nb;
    return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm,
              MPI_Request *req) {
    *req = 0;
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    g_pending.push_back({nullptr, buf, (size_t)count * (size_t)dt, tag, true});
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm,
              MPI_Request *req) {
    *req = 0;
    if (source == MPI_PROC_NULL) return MPI_SUCCESS;
    g_pending.push_back({buf, nullptr, (size_t)count * (size_t)dt, tag, false});
    return MPI_SUCCESS;
}

int MPI_Waitall(int, MPI_Request *, MPI_Status *) {
    for (const Pending &r : g_pending) {
        if (r.is_send) continue;
        bool matched = false;
        for (const Pending &s : g_pending) {
            if (s.is_send && s.tag == r.tag) {
                if (s.bytes != r.bytes) throw std::runtime_error("stub MPI: size mismatch");
                std::memcpy(r.buf, s.cbuf, r.bytes);
                matched = true;
                break;
            }
        }
        if (!matched) throw std::runtime_error("stub MPI: unmatched receive");
    }
    g_pending.clear();
    return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *, MPI_Status *) { return MPI_Waitall(0, nullptr, nullptr); }

int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
    throw std::runtime_error("stub MPI: blocking send on a single rank");
}
int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
    throw std::runtime_error("stub MPI: blocking receive on a single rank");
}
int MPI_Send_init(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
    throw std::runtime_error("stub MPI: persistent requests unsupported");
}
int MPI_Recv_init(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
    throw std::runtime_error("stub MPI: persistent requests unsupported");
}

int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype dt, MPI_Op, MPI_Comm) {
    std::memmove(r, s, (size_t)count * (size_t)dt);
    return MPI_SUCCESS;
}
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype dt, MPI_Op, int, MPI_Comm) {
    std::memmove(r, s, (size_t)count * (size_t)dt);
    return MPI_SUCCESS;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Gatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *, const int *,
                MPI_Datatype, int, MPI_Comm) {
    std::memmove(r, s, (size_t)sc * (size_t)st);
    return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { throw ns3d_mpi_abort(code); }

double MPI_Wtime(void) {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"
