/*
 * Single-process stand-in for the handful of MPI calls the BiqBin C sources
 * make outside their main.c.  It exists only so the reference's own sources
 * compile into the serial CPU oracle (oracle/_ref/); it is test
 * infrastructure, never part of the GPU product.
 *
 * Semantics chosen so the reference worker routine worker_Bab_Main
 * (src/bab_functions.c:224-332) runs unchanged in one process:
 *   - MPI_Send / MPI_Bcast are no-ops (nobody listens);
 *   - MPI_Recv zero-fills the receive buffer, so "number of free workers"
 *     reads as 0 and a received lower bound reads as 0 (never an
 *     improvement, since the B&B lower bound starts at 0,
 *     src/bab_functions.c:26-35);
 *   - MPI_Abort reports and exits with the given code, as the reference's
 *     fatal path does (e.g. src/ipm_mc_pk.c:132-136).
 */
#ifndef BQB_ORACLE_MPI_STUB_H
#define BQB_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_ANY_SOURCE (-1)

static inline size_t bqb_stub_type_size(MPI_Datatype t)
{
    return t == MPI_INT ? sizeof(int) : (t == MPI_DOUBLE ? sizeof(double) : 0);
}

static inline int MPI_Abort(MPI_Comm c, int code)
{
    (void)c;
    fprintf(stderr, "MPI_Abort(%d) called (serial oracle)\n", code);
    fflush(stderr);
    exit(code);
}

static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c;
    return 0;
}

static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)s; (void)tag; (void)c;
    if (b && n > 0) memset(b, 0, (size_t)n * bqb_stub_type_size(t));
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = tag; st->MPI_ERROR = 0; }
    return 0;
}

static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)b; (void)n; (void)t; (void)root; (void)c;
    return 0;
}

static inline double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#endif
