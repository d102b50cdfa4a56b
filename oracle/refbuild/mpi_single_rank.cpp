// One-rank implementations of the MPI calls declared in mpi.h.  Test
// infrastructure for building the reference sources; never part of the
// product.  With one rank every collective reduces to a copy of the caller's
// own contribution, which is what MPICH/Open MPI return at world size 1.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

struct drpt_mpi_file_s {
  int fd;
  long long view_disp;
  long long write_pos;
};

static size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return 4;
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_FLOAT_INT: return 8;  // struct { float; int; }
    case MPI_LONG: return 8;
    default:
      std::fprintf(stderr, "mpi_single_rank: unknown datatype %d\n", t);
      std::abort();
  }
}

static void copy_elems(void *dst, const void *src, long long n, MPI_Datatype t) {
  if (n <= 0 || dst == src) return;
  std::memmove(dst, src, (size_t)n * type_size(t));
}

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE) copy_elems(recvbuf, sendbuf, count, type);
  return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                  int, MPI_Datatype, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE) copy_elems(recvbuf, sendbuf, scount, stype);
  return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                   const int *, const int *displs, MPI_Datatype, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE)
    copy_elems((char *)recvbuf + (size_t)displs[0] * type_size(stype), sendbuf, scount,
               stype);
  return MPI_SUCCESS;
}

int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                 int, MPI_Datatype, MPI_Comm) {
  copy_elems(recvbuf, sendbuf, scount, stype);
  return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls,
                  MPI_Datatype stype, void *recvbuf, const int *, const int *rdispls,
                  MPI_Datatype, MPI_Comm) {
  size_t es = type_size(stype);
  copy_elems((char *)recvbuf + (size_t)rdispls[0] * es,
             (const char *)sendbuf + (size_t)sdispls[0] * es, scounts[0], stype);
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm, const char *filename, int amode, MPI_Info, MPI_File *fh) {
  int flags = (amode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;  // no O_TRUNC, as MPI-IO
  int fd = open(filename, flags, 0644);
  if (fd < 0) { *fh = nullptr; return MPI_ERR_FILE; }
  *fh = new drpt_mpi_file_s{fd, 0, 0};
  return MPI_SUCCESS;
}

int MPI_File_get_size(MPI_File fh, MPI_Offset *size) {
  if (!fh) return MPI_ERR_FILE;
  struct stat st;
  if (fstat(fh->fd, &st) != 0) return MPI_ERR_FILE;
  *size = (MPI_Offset)st.st_size;
  return MPI_SUCCESS;
}

int MPI_File_read_at_all(MPI_File fh, MPI_Offset offset, void *buf, int count,
                         MPI_Datatype type, MPI_Status *) {
  if (!fh) return MPI_ERR_FILE;
  size_t want = (size_t)count * type_size(type), got = 0;
  while (got < want) {
    ssize_t r = pread(fh->fd, (char *)buf + got, want - got, offset + (off_t)got);
    if (r <= 0) break;
    got += (size_t)r;
  }
  return MPI_SUCCESS;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype, MPI_Datatype,
                      const char *, MPI_Info) {
  if (!fh) return MPI_ERR_FILE;
  fh->view_disp = disp;
  fh->write_pos = 0;
  return MPI_SUCCESS;
}

int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype type,
                       MPI_Status *) {
  if (!fh) return MPI_ERR_FILE;
  size_t want = (size_t)count * type_size(type), put = 0;
  while (put < want) {
    ssize_t w = pwrite(fh->fd, (const char *)buf + put, want - put,
                       fh->view_disp + fh->write_pos + (off_t)put);
    if (w <= 0) return MPI_ERR_FILE;
    put += (size_t)w;
  }
  fh->write_pos += (long long)want;
  return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh) {
  if (fh && *fh) {
    close((*fh)->fd);
    delete *fh;
    *fh = nullptr;
  }
  return MPI_SUCCESS;
}

}  // extern "C"
