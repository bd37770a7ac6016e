/* TEST INFRASTRUCTURE ONLY — a single-rank stand-in for the MPI C interface, written for
 * this project so that the reference TetOpSplitP compiles and runs as `mpirun -n 1`
 * would run it.  Collectives over one rank are copies; point-to-point calls are never
 * reached with one rank (no neighbours) and abort if they are. */
#ifndef STEPS_SHIM_MPI_H
#define STEPS_SHIM_MPI_H
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* the element size in bytes, 0 = null */
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR, count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL 0

#define MPI_DATATYPE_NULL 0
#define MPI_CHAR ((int)sizeof(char))
#define MPI_UNSIGNED_CHAR ((int)sizeof(unsigned char))
#define MPI_SHORT ((int)sizeof(short))
#define MPI_UNSIGNED_SHORT ((int)sizeof(unsigned short))
#define MPI_INT ((int)sizeof(int))
#define MPI_UNSIGNED ((int)sizeof(unsigned))
#define MPI_LONG ((int)sizeof(long))
#define MPI_UNSIGNED_LONG ((int)sizeof(unsigned long))
#define MPI_LONG_LONG ((int)sizeof(long long))
#define MPI_UNSIGNED_LONG_LONG ((int)sizeof(unsigned long long))
#define MPI_FLOAT ((int)sizeof(float))
#define MPI_DOUBLE ((int)sizeof(double))
#define MPI_LONG_DOUBLE ((int)sizeof(long double))
#define MPI_C_BOOL ((int)sizeof(bool))
#define MPI_CXX_BOOL ((int)sizeof(bool))
#define MPI_DOUBLE_COMPLEX ((int)(2 * sizeof(double)))
#define MPI_INT64_T 8
#define MPI_UINT64_T 8
#define MPI_INT32_T 4
#define MPI_UINT32_T 4

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LAND 4
#define MPI_LOR 5
#define MPI_PROD 6

static inline void steps_shim_mpi_unreachable(const char* what) {
    fprintf(stderr, "single-rank MPI stand-in: %s is not available with one rank\n", what);
    abort();
}
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Initialized(int* f) { *f = 1; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Finalized(int* f) { *f = 0; return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != MPI_IN_PLACE && n > 0) memmove(r, s, (size_t)n * (size_t)t);
    return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (s != MPI_IN_PLACE && n > 0) memmove(r, s, (size_t)n * (size_t)t);
    return 0;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
    if (s != MPI_IN_PLACE && n > 0) memmove(r, s, (size_t)n * (size_t)t);
    return 0;
}
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* displs,
                                 MPI_Datatype rt, MPI_Comm) {
    if (s != MPI_IN_PLACE && n > 0) memmove((char*)r + (size_t)displs[0] * (size_t)rt, s, (size_t)n * (size_t)t);
    return 0;
}
static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
    steps_shim_mpi_unreachable("MPI_Isend");
    return 0;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    steps_shim_mpi_unreachable("MPI_Recv");
    return 0;
}
static inline int MPI_Iprobe(int, int, MPI_Comm, int* flag, MPI_Status*) { *flag = 0; return 0; }
static inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* c) {
    *c = t ? st->count_bytes / t : 0;
    return 0;
}
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
#endif
