/*
 * In-process stand-in for the MPI subset the reference's zmodel sources call.
 *
 * TEST INFRASTRUCTURE ONLY: it lets the unmodified reference pipeline
 * (zmodel/transforms/fft.cu, fft3d.cu, zmodel/stencils/laplace.cu, laplace3d.cu)
 * run with one host thread per MPI rank inside one process on one GPU, so that its
 * outputs and timings can be compared with the B200 library.  The product library
 * never includes or links this file.
 *
 * Semantics: every collective is a rendezvous of the calling communicator's member
 * threads (post pointers, barrier, copy, barrier).  Copies use cudaMemcpy with
 * cudaMemcpyDefault, so both the host-staged path and the __GPU__AWARE__MPI__ path
 * (device pointers) work.  Only the calls, datatypes and ops used by the reference
 * are provided (zmodel/transforms/fft.cu:221-305, fft3d.cu:260-378,
 * zmodel/stencils/laplace.cu:194-256, laplace3d.cu:265-361, the TIME_MPI_MAX_NS macro).
 */
#ifndef ZR_MPI_STANDIN_H
#define ZR_MPI_STANDIN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zr_comm* MPI_Comm;
typedef int MPI_Datatype;      /* element size in bytes */
typedef int MPI_Op;
typedef int MPI_Info;
typedef struct { int source, tag; } MPI_Status;

#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)16)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_LONG_LONG ((MPI_Datatype)8)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_MAX ((MPI_Op)1)
#define MPI_SUM ((MPI_Op)2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_COMM_TYPE_SHARED 1
#define MPI_SUCCESS 0

MPI_Comm zr_comm_world(void);
#define MPI_COMM_WORLD (zr_comm_world())

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_split_type(MPI_Comm comm, int split_type, int key, MPI_Info info, MPI_Comm* newcomm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm);

/* Driver side: run fn(rank, arg) on `nranks` threads, each one MPI rank of a fresh
 * MPI_COMM_WORLD.  Returns 0, or -1 if a rendezvous timed out (a rank missing). */
int zr_run_ranks(int nranks, void (*fn)(int rank, void* arg), void* arg);

#ifdef __cplusplus
}
#endif

#endif
