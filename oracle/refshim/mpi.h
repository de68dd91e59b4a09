/* Oracle build shim (test infrastructure only): a type-level stand-in for
 * <mpi.h> so the reference correlator sources compile without an MPI
 * installation.  The oracle harness only uses the non-MPI Configuration
 * constructor and calls Core::processdata directly, so none of these
 * functions is reached on the checked path; each one aborts if it is. */
#ifndef GX_ORACLE_MPI_SHIM_H
#define GX_ORACLE_MPI_SHIM_H
#include <stdio.h>
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; int count; } MPI_Status;

#define MPI_COMM_WORLD    0
#define MPI_SUCCESS       0
#define MPI_INT           1
#define MPI_FLOAT         2
#define MPI_CHAR          3
#define MPI_UNSIGNED_CHAR 4
#define MPI_DOUBLE        5
#define MPI_ANY_TAG      (-1)
#define MPI_ANY_SOURCE   (-2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

static inline int gx_mpi_unreachable(const char *fn) {
  fprintf(stderr, "oracle mpi shim: %s reached\n", fn);
  abort();
  return 1;
}
#define MPI_Abort(c, e)            gx_mpi_unreachable("MPI_Abort")
#define MPI_Bcast(...)             gx_mpi_unreachable("MPI_Bcast")
#define MPI_Barrier(...)           gx_mpi_unreachable("MPI_Barrier")
#define MPI_Ssend(...)             gx_mpi_unreachable("MPI_Ssend")
#define MPI_Send(...)              gx_mpi_unreachable("MPI_Send")
#define MPI_Issend(...)            gx_mpi_unreachable("MPI_Issend")
#define MPI_Irecv(...)             gx_mpi_unreachable("MPI_Irecv")
#define MPI_Recv(...)              gx_mpi_unreachable("MPI_Recv")
#define MPI_Wait(...)              gx_mpi_unreachable("MPI_Wait")
#define MPI_Waitall(...)           gx_mpi_unreachable("MPI_Waitall")
#define MPI_Testall(...)           gx_mpi_unreachable("MPI_Testall")
#define MPI_Get_count(...)         gx_mpi_unreachable("MPI_Get_count")
#define MPI_Comm_dup(a, b)         (*(b) = (a), 0)
#define MPI_Comm_rank(c, r)        (*(r) = 0, 0)
#define MPI_Comm_size(c, s)        (*(s) = 1, 0)
#define MPI_Iprobe(...)            gx_mpi_unreachable("MPI_Iprobe")
#define MPI_Wtime()                0.0
#endif
