/*
 * Single-rank MPI stand-in used ONLY to compile the reference solver's own
 * C sources as the CPU oracle (test infrastructure, never the product path).
 *
 * It covers exactly the MPI surface the reference uses (enumerated by grep over
 * src/*.c): rank/size queries, derived datatypes (contiguous, vector), user
 * reduction ops, Sendrecv, Allreduce, Reduce, Bcast, Allgather(v), the
 * Cartesian helpers and the timers.  With one rank every neighbour is rank 0,
 * so Sendrecv is a strided self copy: the send region is packed with the send
 * datatype and unpacked into the receive region with the receive datatype.
 * That self copy is what builds the periodic halos of the reference
 * (src/lb.c:771-784 sendrecv_borders_pop with NEW_SENDRECV, src/grid.c:609-1182).
 */
#ifndef CH4_ORACLE_MPI_SHIM_H
#define CH4_ORACLE_MPI_SHIM_H

#include <stddef.h>

typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Comm;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef void (MPI_User_function)(void *invec, void *inoutvec, int *len, MPI_Datatype *datatype);

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

/* predefined datatypes: handles 1..5 are reserved by the shim */
#define MPI_DOUBLE 1
#define MPI_FLOAT 2
#define MPI_INT 3
#define MPI_LONG_DOUBLE 4
#define MPI_CHAR 5

/* predefined op */
#define MPI_SUM 1

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
double MPI_Wtime(void);
double MPI_Wtick(void);
int MPI_Barrier(MPI_Comm comm);

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Op_create(MPI_User_function *fn, int commute, MPI_Op *op);

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void *buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                  void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                   void *recvbuf, const int *recvcounts, const int *displs, MPI_Datatype recvtype, MPI_Comm comm);

int MPI_Dims_create(int nnodes, int ndims, int *dims);
int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank);

#endif
