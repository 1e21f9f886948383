/*
 * Single-rank stand-in for <mpi.h>, used only to build the reference's own
 * sources into oracle/_ref (this image has no MPI).  With one rank every
 * collective is the identity and no point-to-point message is ever posted
 * (CPM has no valid neighbour), so these definitions are complete for that use.
 */
#ifndef FALM_ORACLE_MPI_STUB_H
#define FALM_ORACLE_MPI_STUB_H
#include <string.h>

typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Comm;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR 1
#define MPI_SHORT 2
#define MPI_INT 3
#define MPI_LONG 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 6
#define MPI_LONG_DOUBLE 7
#define MPI_UNSIGNED_CHAR 8
#define MPI_UNSIGNED_SHORT 9
#define MPI_UNSIGNED 10
#define MPI_UNSIGNED_LONG 11
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_IN_PLACE ((void *)1)

static inline int mpi_stub_size(MPI_Datatype t) {
    switch (t) {
    case MPI_CHAR: case MPI_UNSIGNED_CHAR: return 1;
    case MPI_SHORT: case MPI_UNSIGNED_SHORT: return 2;
    case MPI_INT: case MPI_FLOAT: case MPI_UNSIGNED: return 4;
    case MPI_LONG_DOUBLE: return 16;
    default: return 8;
    }
}
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *sb, void *rb, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (sb != MPI_IN_PLACE) memcpy(rb, sb, (size_t)n * mpi_stub_size(t));
    return 0;
}
static inline int MPI_Allgather(const void *sb, int n, MPI_Datatype t, void *rb, int, MPI_Datatype, MPI_Comm) {
    memcpy(rb, sb, (size_t)n * mpi_stub_size(t));
    return 0;
}
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q) { *q = 0; return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q) { *q = 0; return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
#endif
