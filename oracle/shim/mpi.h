/*
 * Single-rank MPI shim: test infrastructure for building the reference solver
 * (MHD2DCFDFFTW) from its own, unmodified sources in a container that has no
 * MPI.  It implements exactly the MPI identifiers those sources use, with the
 * semantics of a one-process MPI_COMM_WORLD:
 *   - point-to-point calls copy between the caller's own buffers (a rank
 *     sending to itself), honouring subarray / contiguous datatypes;
 *   - collectives (Bcast, Allreduce MIN/MAX, Barrier) are copies or no-ops;
 *   - MPI-IO writes go through stdio at the view displacement.
 * Only the oracle build and the drop-in demo link this; the GPU product does
 * not use MPI at all.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int source, tag, error; } MPI_Status;
typedef struct oracle_mpi_type *MPI_Datatype;
typedef struct oracle_mpi_file *MPI_File;

extern struct oracle_mpi_type oracle_mpi_double, oracle_mpi_int,
    oracle_mpi_uchar, oracle_mpi_ushort, oracle_mpi_unsigned,
    oracle_mpi_ulong, oracle_mpi_ulonglong;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE (&oracle_mpi_double)
#define MPI_INT (&oracle_mpi_int)
#define MPI_UNSIGNED_CHAR (&oracle_mpi_uchar)
#define MPI_UNSIGNED_SHORT (&oracle_mpi_ushort)
#define MPI_UNSIGNED (&oracle_mpi_unsigned)
#define MPI_UNSIGNED_LONG (&oracle_mpi_ulong)
#define MPI_UNSIGNED_LONG_LONG (&oracle_mpi_ulonglong)
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_ORDER_C 0
#define MPI_MODE_WRONLY 4
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm,
                 MPI_Status *status);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype old,
                             MPI_Datatype *newtype);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info,
                  MPI_File *fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype,
                      MPI_Datatype filetype, const char *datarep, MPI_Info info);
int MPI_File_write_all(MPI_File fh, const void *buf, int count,
                       MPI_Datatype type, MPI_Status *status);
int MPI_File_close(MPI_File *fh);

#ifdef __cplusplus
}
#endif
#endif
