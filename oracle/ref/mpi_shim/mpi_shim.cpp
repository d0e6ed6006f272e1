// Single-rank implementation of the MPI subset declared in mpi_shim/mpi.h.
// Test infrastructure only: lets the reference's own translation units run
// as one rank inside oracle/_ref.
#include "mpi.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace {
std::size_t typeSize(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_C_BOOL: return 1;
    case MPI_INT: case MPI_UNSIGNED: return 4;
    case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_LONG_LONG:
    case MPI_UNSIGNED_LONG_LONG: case MPI_DOUBLE: case MPI_UINT64_T: return 8;
    case MPI_LONG_DOUBLE: return sizeof(long double);
    case MPI_2INT: return 8;
    case MPI_DOUBLE_INT: return 16;
  }
  std::fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
  std::abort();
}
void copy(const void* s, void* r, int count, MPI_Datatype t) {
  if (s == MPI_IN_PLACE || s == r || count <= 0) return;
  std::memmove(r, s, static_cast<std::size_t>(count) * typeSize(t));
}
int pointToPoint(int partner) {
  if (partner == MPI_PROC_NULL) return MPI_SUCCESS;
  std::fprintf(stderr, "mpi shim: point-to-point with a real partner at one rank\n");
  std::abort();
}
}  // namespace

extern "C" {
int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int, int* provided) {
  if (provided) *provided = MPI_THREAD_FUNNELED;
  return MPI_SUCCESS;
}
int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
int MPI_Finalized(int* flag) { *flag = 0; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Query_thread(int* provided) { *provided = MPI_THREAD_FUNNELED; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::fprintf(stderr, "MPI_Abort(%d)\n", code); std::abort(); }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
double MPI_Wtime(void) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { copy(s, r, n, t); return MPI_SUCCESS; }
int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) { copy(s, r, n, t); return MPI_SUCCESS; }
int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) { copy(s, r, n, t); return MPI_SUCCESS; }
int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) { copy(s, r, n, t); return MPI_SUCCESS; }
int MPI_Scatter(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) { copy(s, r, n, t); return MPI_SUCCESS; }
int MPI_Alltoall(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) { copy(s, r, n, t); return MPI_SUCCESS; }
int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r,
                  const int*, const int* rd, MPI_Datatype, MPI_Comm) {
  if (sc[0] > 0)
    std::memmove(static_cast<char*>(r) + static_cast<std::size_t>(rd[0]) * typeSize(st),
                 static_cast<const char*>(s) + static_cast<std::size_t>(sd[0]) * typeSize(st),
                 static_cast<std::size_t>(sc[0]) * typeSize(st));
  return MPI_SUCCESS;
}
int MPI_Sendrecv(const void*, int, MPI_Datatype, int dest, int, void*, int, MPI_Datatype,
                 int source, int, MPI_Comm, MPI_Status*) {
  pointToPoint(dest);
  return pointToPoint(source);
}
int MPI_Send(const void*, int, MPI_Datatype, int dest, int, MPI_Comm) { return pointToPoint(dest); }
int MPI_Recv(void*, int, MPI_Datatype, int source, int, MPI_Comm, MPI_Status*) { return pointToPoint(source); }
}
