/* Single-rank MPI subset for building the DPSNN reference as the oracle.
 * Test infrastructure only (see mpi.h). */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define MAX_STRUCT_TYPES 16
static MPI_Aint g_struct_extent[MAX_STRUCT_TYPES];
static int g_struct_count = 0;

/* Struct types are encoded as negative ids so they never collide with the
 * byte sizes used for the basic types. */
static size_t type_size(MPI_Datatype t) {
  if (t < 0) return (size_t)g_struct_extent[-t - 1];
  return (size_t)t;
}

static void unreachable(const char *what) {
  fprintf(stderr, "mpi_stub: %s is not available in a single-rank run\n", what);
  abort();
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
double MPI_Wtime(void) {
  struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
int MPI_Get_address(const void *loc, MPI_Aint *addr) { *addr = (MPI_Aint)loc; return 0; }
int MPI_Type_create_struct(int count, const int bl[], const MPI_Aint disp[],
                           const MPI_Datatype types[], MPI_Datatype *nt) {
  /* extent padded to the largest member alignment, as MPI does */
  MPI_Aint ext = 0, align = 1;
  for (int i = 0; i < count; i++) {
    const MPI_Aint sz = (MPI_Aint)type_size(types[i]);
    MPI_Aint end = disp[i] + (MPI_Aint)bl[i] * sz;
    if (end > ext) ext = end;
    const MPI_Aint a = sz >= 8 ? 8 : (sz >= 4 ? 4 : (sz >= 2 ? 2 : 1));
    if (a > align) align = a;
  }
  ext = (ext + align - 1) & ~(align - 1);
  if (g_struct_count >= MAX_STRUCT_TYPES) unreachable("more struct types");
  g_struct_extent[g_struct_count] = ext;
  *nt = -(MPI_Datatype)(++g_struct_count);
  return 0;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_get_extent(MPI_Datatype t, MPI_Aint *lb, MPI_Aint *ext) {
  *lb = 0; *ext = (MPI_Aint)type_size(t); return 0;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
  *count = st ? (int)(st->count_bytes / (int)type_size(t)) : 0; return 0;
}
int MPI_Alltoall(const void *sb, int sc, MPI_Datatype st, void *rb, int rc,
                 MPI_Datatype rt, MPI_Comm c) {
  (void)rc; (void)rt; (void)c;
  if (sb != MPI_IN_PLACE) memmove(rb, sb, (size_t)sc * type_size(st));
  return 0;
}
int MPI_Alltoallv(const void *sb, const int sc[], const int sd[], MPI_Datatype st,
                  void *rb, const int rc[], const int rd[], MPI_Datatype rt,
                  MPI_Comm c) {
  (void)rc; (void)c;
  size_t es = type_size(st), er = type_size(rt);
  memmove((char *)rb + (size_t)rd[0] * er, (const char *)sb + (size_t)sd[0] * es,
          (size_t)sc[0] * es);
  return 0;
}
int MPI_Allgather(const void *sb, int sc, MPI_Datatype st, void *rb, int rc,
                  MPI_Datatype rt, MPI_Comm c) {
  (void)rc; (void)rt; (void)c;
  if (sb != MPI_IN_PLACE) memmove(rb, sb, (size_t)sc * type_size(st));
  return 0;
}
int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; unreachable("MPI_Send"); return 1;
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; (void)r; unreachable("MPI_Isend"); return 1;
}
int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; unreachable("MPI_Recv"); return 1;
}
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)r; unreachable("MPI_Irecv"); return 1;
}
int MPI_Wait(MPI_Request *r, MPI_Status *st) { (void)r; (void)st; return 0; }
int MPI_Waitall(int n, MPI_Request r[], MPI_Status st[]) { (void)n; (void)r; (void)st; return 0; }
