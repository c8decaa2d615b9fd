/* A minimal, thread-based stand-in for the MPI calls the HPCG 3.1 reference
 * makes (ExchangeHalo.cpp, ComputeDotProduct_ref.cpp, ComputeResidual.cpp,
 * GenerateProblem_ref.cpp, mytimer.cpp). TEST INFRASTRUCTURE ONLY.
 *
 * Every "rank" is a thread of one process, started by shim_run(); the calling
 * thread's rank is thread-local. Point-to-point messages are buffered (MPI_Send
 * copies and returns; a receive completes in MPI_Wait), matched by (source,
 * tag) in send order as MPI's non-overtaking rule requires. MPI_Allreduce folds
 * the ranks' contributions in rank order 0, 1, ..., so its result is
 * deterministic. Only MPI_COMM_WORLD exists. */
#ifndef HPCG_ORACLE_MPI_SHIM_H
#define HPCG_ORACLE_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_LONG_LONG_INT 3
#define MPI_LONG_LONG 3
#define MPI_DOUBLE 4
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);

/* Runs fn(rank, arg) on nranks threads, one per rank, and joins them. */
void shim_run(int nranks, void (*fn)(int rank, void* arg), void* arg);

#ifdef __cplusplus
}
#endif

#endif
