/*
 * Single-rank stand-in for <mpi.h>, used only to build the reference GRE engine
 * as a CPU oracle on hosts without an MPI installation.
 *
 * TEST INFRASTRUCTURE: nothing in the product links this file.
 *
 * Semantics: exactly one process (MPI_COMM_WORLD size 1, rank 0).  At np=1 the
 * reference never sends to itself (every send loop skips p==procID, e.g.
 * Engine.hpp:496 and GraphIngress.hpp:520), so point-to-point calls only need
 * to exist: a posted receive never completes, MPI_Test reports "not done",
 * collectives copy the send buffer to the receive buffer.  Only the symbols the
 * reference names (Comm/CommUnderlying.hpp:1-256, Comm/BufferingComm.hpp) are
 * provided.
 */
#ifndef GRE_ORACLE_MPI_SHIM_H
#define GRE_ORACLE_MPI_SHIM_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

/* datatype codes double as element sizes in bytes */
#define MPI_BYTE 1
#define MPI_INT 4
#define MPI_LONG 8
#define MPI_DOUBLE 9
#define MPI_SUM 0

static inline int gre_shim_type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : t; }

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static inline int MPI_Allreduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    memmove(r, s, (size_t)count * (size_t)gre_shim_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    memmove(r, s, (size_t)count * (size_t)gre_shim_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    memmove(r, s, (size_t)sc * (size_t)gre_shim_type_size(st));
    return MPI_SUCCESS;
}

/* point-to-point: never exercised at np=1 (no peer exists) */
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) {
    *q = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) {
    *q = 0;
    return MPI_SUCCESS;
}
/* a send "completes" at once; a receive never does (nobody can send) */
static inline int MPI_Test(MPI_Request* q, int* flag, MPI_Status*) {
    *flag = (*q == 1);
    return MPI_SUCCESS;
}
static inline int MPI_Cancel(MPI_Request*) { return MPI_SUCCESS; }
static inline int MPI_Iprobe(int, int, MPI_Comm, int* flag, MPI_Status*) {
    *flag = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype, int* c) {
    *c = st ? st->count_ : 0;
    return MPI_SUCCESS;
}

#endif
