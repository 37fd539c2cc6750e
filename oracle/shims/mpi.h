/* Single-rank stand-in for the MPI calls the reference makes (test
 * infrastructure for the oracle build only; never linked into the product).
 *
 * The reference (src/*.cpp, include/parvec.hpp, include/DataCollection.hpp)
 * calls MPI_Init/Finalize/Comm_rank/Comm_size/Barrier/Alltoall/Irecv/Isend/
 * Waitall/Allreduce/Bcast/Gather on MPI_COMM_WORLD.  With one rank every
 * collective is a local copy and point-to-point traffic is always to self,
 * which ParVec never sends (parvec.hpp:236 skips k == mpirank) except as
 * zero-byte messages, so Irecv/Isend/Waitall can be no-ops.
 *
 * <stdlib.h> and <math.h> are included here on purpose: the reference calls
 * unqualified abs() on doubles (src/wave3d.cpp:50-53, include/vec3t.hpp:77);
 * with libstdc++ that resolves to the floating overload only when the C++
 * <stdlib.h>/<math.h> wrappers are visible, as they were with the MPI
 * headers the reference was written against.  Without them abs(double)
 * would truncate to int and nml2dir could not work. */
#ifndef DDFMM_ORACLE_MPI_STUB_H
#define DDFMM_ORACLE_MPI_STUB_H

#include <stdlib.h>
#include <math.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_SUM 1
#define MPI_MAX 2

static inline int ddfmm_mpi_size_of(MPI_Datatype t) { return (int)t; }

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Alltoall(const void* sb, int sc, MPI_Datatype st, void* rb, int, MPI_Datatype, MPI_Comm) {
    if (sc > 0 && sb != rb) memmove(rb, sb, (size_t)sc * ddfmm_mpi_size_of(st));
    return 0;
}
static inline int MPI_Allreduce(const void* sb, void* rb, int c, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (c > 0 && sb != rb) memmove(rb, sb, (size_t)c * ddfmm_mpi_size_of(t));
    return 0;
}
static inline int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int, MPI_Datatype, int, MPI_Comm) {
    if (sc > 0 && sb != rb) memmove(rb, sb, (size_t)sc * ddfmm_mpi_size_of(st));
    return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
/* Only self-messages exist with one rank; ParVec never serialises entries
 * for itself, so these carry zero bytes. */
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }

#endif
