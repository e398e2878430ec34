/*
 * mpi.h -- minimal MPI surface for building the NUC3d reference as a CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference solver (src/*.cpp of juncas/NUC3d)
 * uses exactly these MPI names (see src/MPICommunicator.cpp:55-115,
 * src/PDEData3d.cpp:78,121, src/postproc.cpp:828-830, src/NUC3d.cpp:5-9).
 * No MPI library exists in the build container, so this header declares them
 * and mpi_shim.cpp implements them, either as a single rank (self send/recv)
 * or, when NUC_SHIM_NP > 1, as N forked processes that exchange messages
 * through a shared-memory arena (the reference keeps per-process static state,
 * e.g. src/PDEData3d.cpp:100, so ranks must be processes, not threads).
 */
#ifndef NUC3D_ORACLE_MPI_SHIM_H
#define NUC3D_ORACLE_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest,
              int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src,
              int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
