/*
 * Single-rank stand-in for the MPI interface, used only to build the
 * reference ZLLBM sources as the CPU oracle (test infrastructure).
 *
 * The reference includes <mpi.h> unconditionally (source/defs_libs.h:22) and
 * its committed source/config.h defines ENABLE_MPI, but no MPI library is
 * installed here.  Every call below behaves as MPI would on a communicator of
 * exactly one rank: rank 0, size 1, collectives copy the local contribution,
 * point-to-point calls are never issued by the reference at size 1 (its send
 * loops run over the other ranks only, e.g. mpi_grid_communication.cpp:230)
 * and abort loudly if they are.  File calls map onto POSIX pread/pwrite.
 */
#ifndef ZLLBM_ORACLE_MPI_SHIM_H_
#define ZLLBM_ORACLE_MPI_SHIM_H_
#include <cstddef>
#include <cstdint>

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* index into a size table kept by the shim */
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef long long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_INFO_NULL 0
#define MPI_SUM 1
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_TYPECLASS_INTEGER 1
#define MPI_TYPECLASS_REAL 2

/* predefined datatypes: the value indexes the shim's size table */
#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_INT32_T 5
#define MPI_DOUBLE 6
#define MPI_FLOAT 7
#define MPI_INT64_T 8
#define MPI_UINT64_T 9

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Alltoall(const void* send, int scount, MPI_Datatype stype, void* recv, int rcount,
                 MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allgather(const void* send, int scount, MPI_Datatype stype, void* recv, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm);
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm, MPI_Status* st);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* sts);
int MPI_Type_size(MPI_Datatype type, int* size);
int MPI_Type_free(MPI_Datatype* type);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_match_size(int typeclass, int size, MPI_Datatype* type);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out);
int MPI_Type_create_struct(int count, const int* blocklens, const MPI_Aint* disps,
                           const MPI_Datatype* types, MPI_Datatype* out);
int MPI_File_open(MPI_Comm comm, const char* name, int mode, MPI_Info info, MPI_File* fh);
int MPI_File_close(MPI_File* fh);
int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void* buf, int count, MPI_Datatype type,
                          MPI_Status* st);
int MPI_File_read_at_all(MPI_File fh, MPI_Offset off, void* buf, int count, MPI_Datatype type,
                         MPI_Status* st);
#endif  // ZLLBM_ORACLE_MPI_SHIM_H_
