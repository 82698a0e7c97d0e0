// Single-rank MPI stand-in so that Mesh.cpp compiles for the oracle build.
// Only the calls Mesh.cpp makes exist; none of them communicates.
#pragma once
#include <cstdlib>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int x; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_C_BOOL 3
#define MPI_SUM 0
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (t == MPI_INT) for (int i = 0; i < n; ++i) ((int *)r)[i] = ((const int *)s)[i];
  return 0;
}
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
