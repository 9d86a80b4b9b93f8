/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference MAPP
 * sources as a CPU oracle (test infrastructure; never linked into the product).
 *
 * Every call behaves as it would on a one-process communicator: reductions and
 * broadcasts copy their input, the Cartesian topology is a 1x1x1 grid whose
 * neighbours are the calling rank itself, and point-to-point calls are never
 * reached on one rank (the reference only takes its p2p branches when
 * tot_p_grid[d] != 1, atoms.cpp:380,1105,1225), so they report an error if hit.
 */
#ifndef MAPP_ORACLE_MPI_STUB_H
#define MAPP_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 64

/* datatype handles encode their size in bytes */
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)

#define MPI_SUM ((MPI_Op)0)
#define MPI_MAX ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)

static inline int mpistub_size(MPI_Datatype t) { return (int)t; }

static inline int mpistub_unreachable(const char* what)
{
    fprintf(stderr, "mpi stub: %s is not available on a single rank\n", what);
    abort();
    return 1;
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm*) { return MPI_SUCCESS; }
static inline int MPI_Get_processor_name(char* name, int* len)
{
    strcpy(name, "oracle");
    *len = 6;
    return MPI_SUCCESS;
}
static inline double MPI_Wtime()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    if (in != out) memmove(out, in, (size_t)n * (size_t)mpistub_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* c)
{
    *c = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_get(MPI_Comm, int nd, int* dims, int* periods, int* coords)
{
    for (int i = 0; i < nd; i++) { dims[i] = 1; periods[i] = 1; coords[i] = 0; }
    return MPI_SUCCESS;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int* src, int* dst)
{
    *src = 0;
    *dst = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return mpistub_unreachable("MPI_Send"); }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return mpistub_unreachable("MPI_Recv"); }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return mpistub_unreachable("MPI_Isend"); }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return mpistub_unreachable("MPI_Irecv"); }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return mpistub_unreachable("MPI_Wait"); }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return mpistub_unreachable("MPI_Waitall"); }
static inline int MPI_Sendrecv(const void* sb, int sn, MPI_Datatype st, int, int, void* rb, int rn, MPI_Datatype rt, int, int, MPI_Comm, MPI_Status*)
{
    /* a self-exchange copies the message; only size handshakes reach this on one rank */
    size_t n = (size_t)sn * (size_t)mpistub_size(st);
    size_t m = (size_t)rn * (size_t)mpistub_size(rt);
    memmove(rb, sb, n < m ? n : m);
    return MPI_SUCCESS;
}

#endif
