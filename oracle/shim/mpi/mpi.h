/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * src/lsrtm/inversion.cpp into the CPU oracle so that its per-shot geometry
 * members (getVel, getIgz, swapReord, swapModel, removeDirect) can be called
 * directly.  No message is ever exchanged: the oracle never runs the MPI
 * drivers, and every call here is a no-op on one rank.
 */
#ifndef SEIS_ORACLE_MPI_STUB_H
#define SEIS_ORACLE_MPI_STUB_H
#include <unistd.h>  /* the reference calls sleep() without including it */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_SUM 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
#endif
