/*
 * Single-rank MPI shim — test infrastructure for the oracle only.
 *
 * The reference MD engine (MDcode/*.c) is written against MPI, which is not
 * installed on this machine.  This header declares the 16 MPI entry points the
 * reference calls (MDcode/Parallel.c, time_evolve.c, active.c, print.c,
 * initialise.c, main.c) with single-process semantics: rank 0 of a
 * communicator of size 1.  Collectives are copies; a send to self is queued
 * and matched by the next receive (the z-direction halo exchange at
 * MDcode/Parallel.c:427-460 sends to itself even at one rank).
 *
 * Nothing in the product links this file.
 */
#ifndef ACG_ORACLE_MPI_SHIM_H
#define ACG_ORACLE_MPI_SHIM_H
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct { int count_bytes; int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_ANY_SOURCE (-1)
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void *)1)

/* predefined datatypes: the value is the element size in bytes, except
 * derived types which are registered by MPI_Type_create_struct */
#define MPI_INT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)9)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Get_count(const MPI_Status *status, MPI_Datatype type, int *count);
int MPI_Gather(const void *send, int scount, MPI_Datatype stype, void *recv,
               int rcount, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void *send, int scount, MPI_Datatype stype, void *recv,
                const int *rcounts, const int *displs, MPI_Datatype rtype,
                int root, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status *status);
int MPI_Type_create_struct(int count, const int *blocklens, const MPI_Aint *offsets,
                           const MPI_Datatype *types, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);

#endif
