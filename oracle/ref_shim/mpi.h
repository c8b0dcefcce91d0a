/* Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * sources for the reference harness (oracle/ref_cuda_harness.cu). Every
 * collective is the identity on one rank; file I/O entry points report
 * failure (the harness never writes or reads Tecplot files). */
#ifndef OSTC_REF_MPI_SHIM_H
#define OSTC_REF_MPI_SHIM_H
#include <cstdlib>
#include <cstring>
#include <chrono>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
struct ostc_mpi_status_s { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };
typedef ostc_mpi_status_s MPI_Status;
struct ostc_mpi_file_s { int fd; };
typedef ostc_mpi_file_s *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_ORDER_FORTRAN 57
#define MPI_ORDER_C 56
enum { MPI_CHAR = 1, MPI_INT = 4, MPI_FLOAT = 5, MPI_DOUBLE = 8, MPI_C_BOOL = 9, MPI_INT32_T = 10,
       MPI_INT64_T = 11, MPI_OFFSET = 12, MPI_UINT8_T = 13 };
enum { MPI_SUM = 1, MPI_MIN = 2, MPI_MAX = 3 };

inline int ostc_shim_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_C_BOOL: case MPI_UINT8_T: return 1;
    case MPI_INT: case MPI_FLOAT: case MPI_INT32_T: return 4;
    default: return 8;
  }
}
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
inline double MPI_Wtime() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) std::memmove(r, s, (size_t)n * ostc_shim_size(t));
  return 0;
}
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != r) std::memmove(r, s, (size_t)n * ostc_shim_size(t));
  return 0;
}
inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
  std::memmove(r, s, (size_t)n * ostc_shim_size(t));
  return 0;
}
inline int MPI_Allgatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *d, MPI_Datatype,
                          MPI_Comm) {
  std::memmove((char *)r + (size_t)d[0] * ostc_shim_size(t), s, (size_t)n * ostc_shim_size(t));
  return 0;
}
inline int MPI_Scatter(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) {
  std::memmove(r, s, (size_t)n * ostc_shim_size(t));
  return 0;
}
inline int MPI_Scatterv(const void *s, const int *, const int *d, MPI_Datatype t, void *r, int n, MPI_Datatype, int,
                        MPI_Comm) {
  std::memmove(r, (const char *)s + (size_t)d[0] * ostc_shim_size(t), (size_t)n * ostc_shim_size(t));
  return 0;
}
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_OTHER; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_OTHER; }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
inline int MPI_File_open(MPI_Comm, const char *, int, MPI_Info, MPI_File *) { return MPI_ERR_OTHER; }
inline int MPI_File_close(MPI_File *) { return 0; }
inline int MPI_File_read_at(MPI_File, MPI_Offset, void *, int, MPI_Datatype, MPI_Status *) { return MPI_ERR_OTHER; }
inline int MPI_File_write_at(MPI_File, MPI_Offset, const void *, int, MPI_Datatype, MPI_Status *) {
  return MPI_ERR_OTHER;
}
inline int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char *, MPI_Info) {
  return MPI_ERR_OTHER;
}
inline int MPI_File_read_all(MPI_File, void *, int, MPI_Datatype, MPI_Status *) { return MPI_ERR_OTHER; }
inline int MPI_File_write_all(MPI_File, const void *, int, MPI_Datatype, MPI_Status *) { return MPI_ERR_OTHER; }
inline int MPI_Type_create_subarray(int, const int *, const int *, const int *, int, MPI_Datatype, MPI_Datatype *o) {
  *o = MPI_DOUBLE;
  return 0;
}
inline int MPI_Type_commit(MPI_Datatype *) { return 0; }
inline int MPI_Type_free(MPI_Datatype *) { return 0; }
#endif
