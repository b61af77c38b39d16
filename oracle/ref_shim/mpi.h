/*
 * Single-rank stand-in for <mpi.h>, used only to build the reference
 * (dgQuEST) from its sources for the oracle. TEST INFRASTRUCTURE ONLY.
 * Rank 0 of 1: collectives copy or do nothing; point-to-point calls are
 * never reached with one rank (every page is local), so they fail loudly.
 */
#ifndef DGQ_REF_SHIM_MPI_H
#define DGQ_REF_SHIM_MPI_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_THREAD_MULTIPLE 3
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_C_DOUBLE_COMPLEX 3
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_ANY_SOURCE (-1)
#define MPI_REQUEST_NULL 0
#define MPI_IN_PLACE ((void *) 1)
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)

static inline size_t dgq_shim_size(MPI_Datatype t) {
    return t == MPI_INT ? sizeof(int) : (t == MPI_C_DOUBLE_COMPLEX ? 2 * sizeof(double) : sizeof(double));
}
static inline int dgq_shim_unreachable(const char *what) {
    fprintf(stderr, "single-rank MPI shim: %s is not expected with one rank\n", what);
    abort();
    return 1;
}
static inline int MPI_Initialized(int *f) { *f = 0; return 0; }
static inline int MPI_Init(int *a, char ***b) { (void) a; (void) b; return 0; }
static inline int MPI_Init_thread(int *a, char ***b, int req, int *prov) { (void) a; (void) b; *prov = req; return 0; }
static inline int MPI_Finalized(int *f) { *f = 0; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void) c; *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void) c; *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void) c; return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void) b; (void) n; (void) t; (void) root; (void) c; return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
    (void) o; (void) c;
    if (s != MPI_IN_PLACE) memcpy(r, s, (size_t) n * dgq_shim_size(t));
    return 0;
}
static inline int MPI_Test(MPI_Request *r, int *f, MPI_Status *s) { (void) r; (void) s; *f = 1; return 0; }
static inline int MPI_Testall(int n, MPI_Request *r, int *f, MPI_Status *s) { (void) n; (void) r; (void) s; *f = 1; return 0; }
static inline int MPI_Recv_init(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r) {
    (void) b; (void) n; (void) t; (void) src; (void) tag; (void) c; *r = 0; return 0;
}
static inline int MPI_Start(MPI_Request *r) { (void) r; return dgq_shim_unreachable("MPI_Start"); }
static inline int MPI_Wait(MPI_Request *r, MPI_Status *s) { (void) r; (void) s; return dgq_shim_unreachable("MPI_Wait"); }
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) { (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; return dgq_shim_unreachable("MPI_Send"); }
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st) { (void) b; (void) n; (void) t; (void) s; (void) tag; (void) c; (void) st; return dgq_shim_unreachable("MPI_Recv"); }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) { (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; (void) r; return dgq_shim_unreachable("MPI_Isend"); }
static inline int MPI_Issend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) { (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; (void) r; return dgq_shim_unreachable("MPI_Issend"); }
#endif
