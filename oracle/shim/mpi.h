/* Single-rank stand-in for the MPI calls ZuikakuCFD makes, so that the
 * unmodified reference sources build into the CPU oracle without an MPI
 * installation.  Test infrastructure only.
 *
 * Semantics: the job is rank 0 of 1.  Point-to-point calls only ever talk to
 * MPI_PROC_NULL at size 1 (src_WENO/fluid.cpp:166-167, src_DG/fluid.cpp:352-353)
 * and are no-ops; collectives copy send to receive (MPI_IN_PLACE leaves the
 * receive buffer as is); barriers, init and finalize do nothing. */
#ifndef ZK_ORACLE_MPI_STUB_H
#define ZK_ORACLE_MPI_STUB_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_MAX 1
#define MPI_SUM 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

static inline int zk_mpi_type_size(MPI_Datatype t) { return t; }

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

static inline int MPI_Sendrecv(const void* sb, int sc, MPI_Datatype st, int dst, int stag,
                               void* rb, int rc, MPI_Datatype rt, int src, int rtag,
                               MPI_Comm comm, MPI_Status* status) {
    (void)sb; (void)sc; (void)st; (void)stag; (void)rb; (void)rc; (void)rt; (void)rtag;
    (void)comm; (void)status;
    /* At size 1 both partners are MPI_PROC_NULL; anything else is a misuse. */
    return (dst == MPI_PROC_NULL && src == MPI_PROC_NULL) ? 0 : 1;
}

static inline int MPI_Allreduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op,
                                MPI_Comm comm) {
    (void)op; (void)comm;
    if (sb != MPI_IN_PLACE) memcpy(rb, sb, (size_t)n * zk_mpi_type_size(t));
    return 0;
}

static inline int MPI_Reduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op, int root,
                             MPI_Comm comm) {
    (void)op; (void)root; (void)comm;
    if (sb != MPI_IN_PLACE) memcpy(rb, sb, (size_t)n * zk_mpi_type_size(t));
    return 0;
}

static inline int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc,
                             MPI_Datatype rt, int root, MPI_Comm comm) {
    (void)rc; (void)rt; (void)root; (void)comm;
    if (sb != MPI_IN_PLACE) memcpy(rb, sb, (size_t)sc * zk_mpi_type_size(st));
    return 0;
}

#endif
