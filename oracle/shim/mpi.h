/* Test infrastructure (oracle only): a single-rank stand-in for the MPI calls
 * the reference TRITON sources make, so that the unmodified reference
 * `src/main.cpp` compiles into a one-process CPU oracle.
 *
 * With one rank every collective is a local copy (Gather/Gatherv/Allreduce)
 * or a no-op (Bcast/Barrier).  Point-to-point calls are only reached by the
 * reference when the communicator has more than one rank; here they fail
 * loudly.  Written from the public MPI function names and signatures only. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_ERROR_STRING 256
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

/* datatype handles encode their byte size */
#define MPI_INT ((MPI_Datatype)4)
#define MPI_INTEGER ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)(0x100 | 4))
#define MPI_DOUBLE ((MPI_Datatype)(0x100 | 8))
#define MPI_MIN ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_SUM ((MPI_Op)3)

static inline size_t oracle_mpi_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm*) { return 0; }
static inline int MPI_Error_string(int, char* s, int* len) { s[0] = 0; *len = 0; return 0; }

static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  memmove(r, s, (size_t)n * oracle_mpi_size(t));
  return 0;
}
static inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) {
  memmove(r, s, (size_t)sn * oracle_mpi_size(st));
  return 0;
}
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
  memmove(r, s, (size_t)sn * oracle_mpi_size(st));
  return 0;
}
static inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs,
                              MPI_Datatype rt, int, MPI_Comm) {
  memmove((char*)r + (size_t)displs[0] * oracle_mpi_size(rt), s, (size_t)sn * oracle_mpi_size(st));
  return 0;
}
static inline int oracle_mpi_p2p_unsupported(void) {
  fprintf(stderr, "oracle mpi shim: point-to-point MPI is not available in the single-rank oracle\n");
  abort();
  return 1;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
  return oracle_mpi_p2p_unsupported();
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
  return oracle_mpi_p2p_unsupported();
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }

#endif
