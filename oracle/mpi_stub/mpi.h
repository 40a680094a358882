/* One-rank MPI for the oracle builds (test infrastructure only): the
 * declarations the reference's C++ sources use, so that its Thomas solvers
 * (00_C/PaScaL_TDMA/src/tdmas.cpp) and its Poisson solve
 * (00_C/examples/module_solve_poisson.cpp with the topology, subdomain and
 * global modules) compile and run as a single rank.  mpi_stub.cpp gives
 * every routine its MPI-standard meaning for a communicator of one rank:
 * collectives copy the caller's own block, point-to-point messages to self
 * are matched by (communicator, tag) in posting order, MPI_PROC_NULL
 * neighbours are no-ops, and subarray datatypes move their elements in C
 * order of the subarray. */
#ifndef PPF_ORACLE_MPI_STUB_H
#define PPF_ORACLE_MPI_STUB_H

typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Op;
struct ppf_mpi_type;
typedef struct ppf_mpi_type* MPI_Datatype;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

extern struct ppf_mpi_type ppf_mpi_double, ppf_mpi_double_complex, ppf_mpi_int;
#define MPI_DOUBLE (&ppf_mpi_double)
#define MPI_DOUBLE_COMPLEX (&ppf_mpi_double_complex)
#define MPI_INT (&ppf_mpi_int)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_PROC_NULL (-2)
#define MPI_REQUEST_NULL (-1)
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);

int MPI_Cart_create(MPI_Comm comm, int ndims, const int* dims, const int* periods, int reorder, MPI_Comm* cart);
int MPI_Cart_sub(MPI_Comm comm, const int* remain_dims, MPI_Comm* sub);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int* source, int* dest);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* comm);

int MPI_Type_create_subarray(int ndims, const int* sizes, const int* subsizes, const int* starts, int order,
                             MPI_Datatype oldtype, MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* statuses);

int MPI_Alltoallw(const void* sendbuf, const int* sendcounts, const int* sdispls, const MPI_Datatype* sendtypes,
                  void* recvbuf, const int* recvcounts, const int* rdispls, const MPI_Datatype* recvtypes,
                  MPI_Comm comm);
int MPI_Ialltoallw(const void* sendbuf, const int* sendcounts, const int* sdispls, const MPI_Datatype* sendtypes,
                   void* recvbuf, const int* recvcounts, const int* rdispls, const MPI_Datatype* recvtypes,
                   MPI_Comm comm, MPI_Request* req);
int MPI_Ialltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm, MPI_Request* req);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
               MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Igather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                MPI_Datatype recvtype, int root, MPI_Comm comm, MPI_Request* req);
int MPI_Iscatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm, MPI_Request* req);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm);

#endif
