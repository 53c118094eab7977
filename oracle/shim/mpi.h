/* Single-rank stand-in for <mpi.h> -- TEST INFRASTRUCTURE ONLY.
 *
 * It lets the reference's PDE, domain and communicator sources
 * (src/pdes/pde.h, src/utils/comm/*, src/grids/domain.*) compile unmodified
 * in the oracle, where the path runs as one rank: rank 0 of a communicator of
 * size 1.  Collectives over one rank are local copies (MPI_Alltoallv moves the
 * rank's own send block to its receive block); point-to-point calls, which a
 * single rank never makes to itself on the path, report an error. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_UNSIGNED 5
#define MPI_FLOAT 6
#define MPI_DOUBLE 8
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

static inline size_t oracle_mpi_type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    default: return 0;
    }
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code)
{
    fprintf(stderr, "MPI_Abort(%d) on the single oracle rank\n", code);
    exit(code);
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm)
{
    fprintf(stderr, "MPI_Send on a single rank: no peer\n");
    return MPI_ERR_OTHER;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*)
{
    fprintf(stderr, "MPI_Recv on a single rank: no peer\n");
    return MPI_ERR_OTHER;
}
static inline int MPI_Alltoallv(const void* sbuf, const int* scounts, const int* sdispls, MPI_Datatype stype,
                                void* rbuf, const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm)
{
    size_t se = oracle_mpi_type_size(stype), re = oracle_mpi_type_size(rtype);
    if (!se || se * scounts[0] != re * rcounts[0]) return MPI_ERR_OTHER;
    if (scounts[0] > 0) memmove((char*)rbuf + re * rdispls[0], (const char*)sbuf + se * sdispls[0], se * scounts[0]);
    return MPI_SUCCESS;
}

#ifdef __cplusplus
namespace MPI {
static const MPI_Datatype CHAR = MPI_CHAR;
static const MPI_Datatype INT = MPI_INT;
static const MPI_Datatype UNSIGNED = MPI_UNSIGNED;
static const MPI_Datatype FLOAT = MPI_FLOAT;
static const MPI_Datatype DOUBLE = MPI_DOUBLE;
}
#endif

#endif
