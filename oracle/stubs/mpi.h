/*
 * Single-rank MPI stand-in used ONLY to compile the reference's own sources
 * into the pinning oracle (oracle/_ref). Test infrastructure, not product.
 *
 * Semantics (implemented in mpi_stub.cpp):
 *   - one rank (rank 0, size 1); MPI_Dims_create gives {1,1,1};
 *   - MPI_Cart_shift returns self (0) on a periodic axis, MPI_PROC_NULL otherwise,
 *     which is what a 1x1x1 periodic Cartesian communicator returns;
 *   - MPI_Isend/MPI_Irecv are queued; MPI_Waitall copies each posted send
 *     buffer into the receive buffer posted with the same tag (self-messaging),
 *     which reproduces the periodic halo exchange of field_structures.h:736-853;
 *   - collectives (Allreduce/Reduce/Bcast) copy send to receive;
 *   - MPI_Abort throws ns3d_mpi_abort (caught by the oracle driver).
 */
#ifndef NS3D_ORACLE_MPI_STUB_H
#define NS3D_ORACLE_MPI_STUB_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_NULL        (-1)
#define MPI_COMM_WORLD       (0)
#define MPI_PROC_NULL        (-2)
#define MPI_DOUBLE           (8)
#define MPI_INT              (4)
#define MPI_BYTE             (1)
#define MPI_SUM              (1)
#define MPI_MIN              (2)
#define MPI_MAX              (3)
#define MPI_STATUSES_IGNORE  ((MPI_Status *)0)
#define MPI_STATUS_IGNORE    ((MPI_Status *)0)
#define MPI_SUCCESS          (0)

#ifdef __cplusplus
extern "C" {
#endif

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm);
int MPI_Dims_create(int nnodes, int ndims, int dims[]);
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *src, int *dst);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status stats[]);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
             MPI_Status *st);
int MPI_Send_init(const void *buf, int count, MPI_Datatype dt, int dest, int tag,
                  MPI_Comm comm, MPI_Request *req);
int MPI_Recv_init(void *buf, int count, MPI_Datatype dt, int source, int tag,
                  MPI_Comm comm, MPI_Request *req);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt,
                  MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt,
               MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                const int recvcounts[], const int displs[], MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif

#endif
