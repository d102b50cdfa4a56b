/*
 * Single-rank MPI stand-in used only to compile and run the reference DRPT
 * sources (cpp/src/**) on one host process.  Test infrastructure: the product
 * never links it.
 *
 * Every collective has its one-rank meaning: the send buffer is copied to the
 * receive buffer (or nothing happens for MPI_IN_PLACE / Bcast / Barrier).
 * MPI-IO maps onto pread/pwrite.  Only the subset the reference calls exists
 * (main.cpp:137-139,192,243-256; mdrpt.cpp:308,411-413,432-745;
 * drpt_global.cpp:405-485,655,762; math_operations.cpp:153,197,328-329;
 * file_reader.cpp:376-446; file_writer.cpp:72,123,166-175).
 */
#ifndef DRPT_ORACLE_MPI_SINGLE_RANK_H
#define DRPT_ORACLE_MPI_SINGLE_RANK_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct drpt_mpi_file_s *MPI_File;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; long long count; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_FILE 27
#define MPI_COMM_WORLD 0x44000000
#define MPI_INFO_NULL 0

#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_FLOAT_INT 5
#define MPI_LONG 6

#define MPI_SUM 1

#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1

#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                  int rcount, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                   const int *rcounts, const int *displs, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                 int rcount, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls,
                  MPI_Datatype stype, void *recvbuf, const int *rcounts,
                  const int *rdispls, MPI_Datatype rtype, MPI_Comm comm);

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info,
                  MPI_File *fh);
int MPI_File_get_size(MPI_File fh, MPI_Offset *size);
int MPI_File_read_at_all(MPI_File fh, MPI_Offset offset, void *buf, int count,
                         MPI_Datatype type, MPI_Status *status);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype,
                      MPI_Datatype filetype, const char *datarep, MPI_Info info);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype type,
                       MPI_Status *status);
int MPI_File_close(MPI_File *fh);

#ifdef __cplusplus
}
#endif

#endif
