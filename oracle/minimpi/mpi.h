/*
 * minimpi: the subset of the MPI C API that the camille reference solver calls,
 * implemented for the oracle build only (test infrastructure, never shipped).
 *
 * The container and the GPU box have no MPI library. The reference solver uses
 * about twenty MPI entry points (src/parallel/parallel.cpp:41-96, the halo
 * exchange in src/solver/spatial_discretization.cpp:1010-1074, the overset
 * exchange in src/overset/overset.cpp:1094-1221, and setup broadcasts in
 * src/io/plot3d.cpp and src/io/overture.cpp). This header declares them with
 * plain integer handles.
 *
 * Two transports:
 *   - one process (MINIMPI_SIZE unset or 1): every message to self goes
 *     through an in-process mailbox, so overset self-donation works;
 *   - several processes started by `minimpi_run -n N prog args...`: each rank is
 *     a forked child connected to every other rank by a socketpair. A reader
 *     thread per rank drains all sockets into per-source queues, so a blocking
 *     send never deadlocks and every receive waits with a time limit
 *     (MINIMPI_TIMEOUT_S, default 600 s) after which the rank exits non-zero.
 */
#ifndef MINIMPI_MPI_H
#define MINIMPI_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;

typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_bytes;
} MPI_Status;

typedef struct {
  int kind;      /* 0 = completed send, 1 = pending receive */
  void *buf;
  int count;
  MPI_Datatype type;
  int source;
  int tag;
  MPI_Comm comm;
} MPI_Request;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_GROUP_NULL (-1)
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_CHAR 3
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_UNDEFINED (-32766)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int errorcode);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_group(MPI_Comm comm, MPI_Group *group);
int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm *newcomm);
int MPI_Group_incl(MPI_Group group, int n, const int ranks[], MPI_Group *newgroup);
int MPI_Group_rank(MPI_Group group, int *rank);
int MPI_Group_size(MPI_Group group, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op op, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
             MPI_Status *status);
int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm,
              MPI_Request *request);
int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
              MPI_Request *request);
int MPI_Wait(MPI_Request *request, MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
