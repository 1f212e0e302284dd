/*
 * Single-process stand-in for the subset of MPI that the DPSNN reference
 * calls (DPSNN_messagePassing.c, DPSNN_mainUnderMPI.c, DPSNN_chrono.c).
 * Test infrastructure only: it lets the unmodified reference sources build
 * and run as one rank (env_globH=1) on a machine without an MPI library.
 * Every collective is a self-copy; point-to-point calls are unreachable at
 * one rank and abort if reached.
 */
#ifndef DPSNN_ORACLE_MPI_STUB_H
#define DPSNN_ORACLE_MPI_STUB_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef long MPI_Datatype;   /* element size in bytes; structs get a registry id */
typedef intptr_t MPI_Aint;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count_bytes; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_SUCCESS 0
#define MPI_ANY_TAG (-1)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)8)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
int MPI_Get_address(const void *location, MPI_Aint *address);
int MPI_Type_create_struct(int count, const int blocklengths[],
                           const MPI_Aint displacements[],
                           const MPI_Datatype types[], MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_get_extent(MPI_Datatype type, MPI_Aint *lb, MPI_Aint *extent);
int MPI_Get_count(const MPI_Status *status, MPI_Datatype type, int *count);
int MPI_Alltoall(const void *sbuf, int scount, MPI_Datatype stype,
                 void *rbuf, int rcount, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoallv(const void *sbuf, const int scounts[], const int sdispls[],
                  MPI_Datatype stype, void *rbuf, const int rcounts[],
                  const int rdispls[], MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype stype,
                  void *rbuf, int rcount, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]);

#ifdef __cplusplus
}
#endif
#endif
