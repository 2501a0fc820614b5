/*
 * Single-rank MPI subset -- TEST INFRASTRUCTURE ONLY (oracle build).
 *
 * The reference channel-flow code (nasilemakbox/ubiquitous-spoon) is written
 * against OpenMPI.  Neither mpi.h nor libmpi exists on this machine, so the
 * oracle build compiles the reference's .c files unmodified against this
 * header.  It implements exactly the calls the reference makes, with the
 * semantics they have on a communicator of size one:
 *   - Cartesian topology queries (every neighbour is rank 0),
 *   - derived datatypes: contiguous and C-order subarrays of basic types,
 *   - Alltoallw / Isend / Recv as local pack+unpack copies,
 *   - Allreduce / Gather(v) as copies (identity at one rank),
 *   - MPI-IO with subarray file views, through stdio.
 * Call sites: transpose.c:409-448, ghostz.c:107-149, get.c:281-302,
 * io.c:211-297, chanfast.c:85-99.
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct shim_dtype *MPI_Datatype;
typedef struct shim_request *MPI_Request;
typedef struct shim_file *MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; int count; } MPI_Status;

extern struct shim_dtype shim_mpi_double, shim_mpi_int, shim_mpi_char;

#define MPI_COMM_WORLD ((MPI_Comm) 0)
#define MPI_DOUBLE (&shim_mpi_double)
#define MPI_INT (&shim_mpi_int)
#define MPI_CHAR (&shim_mpi_char)
#define MPI_SUM ((MPI_Op) 1)
#define MPI_MAX ((MPI_Op) 2)
#define MPI_MIN ((MPI_Op) 3)
#define MPI_IN_PLACE ((void *) 1)
#define MPI_INFO_NULL ((MPI_Info) 0)
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_EXCL 64
#define MPI_MODE_DELETE_ON_CLOSE 16
#define MPI_MODE_APPEND 128

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Initialized(int *flag);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int errorcode);

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *comm_cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *src, int *dst);

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype oldtype,
                             MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);

int MPI_Alltoallw(const void *sendbuf, const int sendcounts[], const int sdispls[],
                  const MPI_Datatype sendtypes[], void *recvbuf, const int recvcounts[],
                  const int rdispls[], const MPI_Datatype recvtypes[], MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *request);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Wait(MPI_Request *request, MPI_Status *status);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
               void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, const int recvcounts[], const int displs[],
                MPI_Datatype recvtype, int root, MPI_Comm comm);

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype,
                      MPI_Datatype filetype, const char *datarep, MPI_Info info);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype type,
                       MPI_Status *status);
int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype type,
                      MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
