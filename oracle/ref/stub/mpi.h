/* Single-process stand-in for the MPI calls the reference's hot path makes
 * (MPI_Barrier, MPI_Reduce, MPI_Bcast).  Test infrastructure only.
 *
 * MPI_Reduce copies send->recv (one rank holds everything) and, when a capture
 * hook is installed, hands each reduced double array to it.  The harness uses
 * the hook to read the current arrays that Currents.cpp reduces and then frees
 * (FERMIONS/WILSON/Currents.cpp:326-333, FERMIONS/OVERLAP/OverlapCurrents.cpp:246-247). */
#pragma once
#include <cstring>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_SUM 10
#define MPI_MAX 11
#define MPI_MIN 12

typedef void (*ovlref_reduce_hook_t)(const double *data, int count);
extern ovlref_reduce_hook_t ovlref_reduce_hook;

static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    size_t width = (type == MPI_DOUBLE) ? sizeof(double) : (type == MPI_LONG ? sizeof(long) : sizeof(int));
    std::memcpy(recv, send, width * (size_t)count);
    if (type == MPI_DOUBLE && ovlref_reduce_hook) ovlref_reduce_hook((const double *)recv, count);
    return 0;
}
