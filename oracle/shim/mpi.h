// Single-rank stand-in for the MPI C API, used only to compile the
// reference simulator's own sources in place as a CPU test oracle.
//
// Test infrastructure: nothing in the product library includes this file.
// Every collective is the identity copy it reduces to at world size 1;
// point-to-point calls only ever see MPI_PROC_NULL at size 1 and do nothing.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef int MPI_Datatype;

struct MPI_Status {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
};

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_DATATYPE_NULL 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_LONG_LONG 3
#define MPI_LONG 4
#define MPI_UNSIGNED_LONG 5
#define MPI_CHAR 6

namespace pcc_mpi_shim {
// Byte extents of the predefined types plus any committed struct types.
inline std::vector<long>& extents() {
  static std::vector<long> e = {0, (long)sizeof(int), (long)sizeof(double), (long)sizeof(long long),
                                (long)sizeof(long), (long)sizeof(unsigned long), 1};
  return e;
}
inline long extent(MPI_Datatype t) { return extents().at((size_t)t); }
inline void copy(const void* src, void* dst, long count, MPI_Datatype t) {
  if (src != dst && count > 0) std::memmove(dst, src, (size_t)(count * extent(t)));
}
}  // namespace pcc_mpi_shim

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) { std::fprintf(stderr, "MPI_Abort(%d)\n", code); std::abort(); }
inline double MPI_Wtime() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  pcc_mpi_shim::copy(s, r, n, t);
  return MPI_SUCCESS;
}
inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  pcc_mpi_shim::copy(s, r, n, t);
  return MPI_SUCCESS;
}
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
  pcc_mpi_shim::copy(s, r, sn, st);
  return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
  pcc_mpi_shim::copy(s, r, sn, st);
  return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*,
                         const int* rd, MPI_Datatype, MPI_Comm) {
  long ext = pcc_mpi_shim::extent(st);
  if (sc[0] > 0)
    std::memmove((char*)r + (long)rd[0] * ext, (const char*)s + (long)sd[0] * ext, (size_t)(sc[0] * ext));
  return MPI_SUCCESS;
}
inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int, MPI_Comm,
                        MPI_Status*) {
  return MPI_SUCCESS;  // both peers are MPI_PROC_NULL at size 1
}
inline int MPI_Get_address(const void* p, MPI_Aint* a) { *a = (MPI_Aint)(uintptr_t)p; return MPI_SUCCESS; }
inline int MPI_Type_create_struct(int n, const int* bl, const MPI_Aint* disp, const MPI_Datatype* types,
                                  MPI_Datatype* out) {
  long ub = 0, align = 1;
  for (int i = 0; i < n; ++i) {
    long e = pcc_mpi_shim::extent(types[i]);
    if (disp[i] + bl[i] * e > ub) ub = disp[i] + bl[i] * e;
    if (e > align) align = e;
  }
  ub = (ub + align - 1) / align * align;
  pcc_mpi_shim::extents().push_back(ub);
  *out = (MPI_Datatype)(pcc_mpi_shim::extents().size() - 1);
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }
