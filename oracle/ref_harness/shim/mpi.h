// Single-rank stand-in for the few MPI C calls in milupHPC's hot-path
// sources.  Test infrastructure only (oracle/ref_harness).
#pragma once
#include <cstring>
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Comm;
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_COMM_WORLD 0
#define MPI_IN_PLACE ((void*)1)
inline int MPI_Finalize() { return 0; }
inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (in != MPI_IN_PLACE && in != out) std::memcpy(out, in, (size_t)n * (size_t)t);
    return 0;
}
