/* Multi-process MPI subset over shared memory, for running the DPSNN
 * reference with env_globH > 1 ranks on a machine without an MPI library.
 * Test infrastructure only: it implements the calls of oracle/mpi_stub/mpi.h
 * that the reference reaches with env_collectivesAlgo=0 (the collectives,
 * barrier, datatypes, timing); point-to-point calls abort.
 *
 * MPI_Init forks DPSNN_SHM_RANKS - 1 children; every process returns from
 * MPI_Init with its own rank, exactly as separate MPI processes would start
 * main().  Collectives go through one staging slot per rank in an anonymous
 * shared mapping (DPSNN_SHM_SLOT_MB MiB each, default 1024, reserved but not
 * committed): each rank writes its outgoing data into its own slot, all ranks
 * meet at a barrier, each copies what is addressed to it out of every slot,
 * and all meet again before the slots are reused.  Every wait is bounded
 * (DPSNN_SHM_TIMEOUT_S, default 1800 s), after which all ranks abort. */
#define _GNU_SOURCE
#include "mpi.h"
#include <sched.h>
#include <signal.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define MAX_RANKS 256

typedef struct {
  atomic_uint arrive;
  atomic_uint gen;
  atomic_int failed;
} shm_header;

/* per-rank slot: P counts and P offsets (bytes), then the payload */
typedef struct {
  size_t bytes[MAX_RANKS];
  size_t off[MAX_RANKS];
} slot_meta;

static int g_rank = 0, g_size = 1;
static pid_t g_child[MAX_RANKS];
static shm_header *g_hdr = NULL;
static char *g_slots = NULL;
static size_t g_slot_bytes = 0;
static double g_timeout_s = 1800.0;

/* Basic types are their byte size; struct types are minus their extent (the
 * reference creates a struct type on every exchange, so none is stored). */
static size_t type_size(MPI_Datatype t) { return (size_t)(t < 0 ? -t : t); }

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void fail(const char *what) {
  fprintf(stderr, "mpi_shm rank %d: %s\n", g_rank, what);
  if (g_hdr) atomic_store(&g_hdr->failed, 1);
  _exit(3);
}

static void barrier(void) {
  if (g_size == 1) return;
  const unsigned gen = atomic_load(&g_hdr->gen);
  if (atomic_fetch_add(&g_hdr->arrive, 1u) == (unsigned)g_size - 1u) {
    atomic_store(&g_hdr->arrive, 0u);
    atomic_fetch_add(&g_hdr->gen, 1u);
    return;
  }
  const double t0 = now_s();
  unsigned spins = 0;
  while (atomic_load(&g_hdr->gen) == gen) {
    if (atomic_load(&g_hdr->failed)) fail("another rank failed");
    if (++spins > 1000u) {
      sched_yield();
      if (g_rank == 0 && (spins & 0xFFu) == 0) {   /* a rank that left early */
        int st = 0;
        if (waitpid(-1, &st, WNOHANG) > 0) {
          char msg[96];
          snprintf(msg, sizeof msg, "a rank ended before the barrier (status 0x%x)", st);
          fail(msg);
        }
      }
      if ((spins & 0xFFFu) == 0 && now_s() - t0 > g_timeout_s) fail("barrier timed out");
    }
  }
}

static slot_meta *meta(int r) { return (slot_meta *)(g_slots + (size_t)r * g_slot_bytes); }
static char *payload(int r) { return g_slots + (size_t)r * g_slot_bytes + sizeof(slot_meta); }

int MPI_Init(int *argc, char ***argv) {
  (void)argc;
  (void)argv;
  const char *s = getenv("DPSNN_SHM_RANKS");
  const int n = s ? atoi(s) : 1;
  if (n < 1 || n > MAX_RANKS) fail("DPSNN_SHM_RANKS out of range");
  g_size = n;
  if (n == 1) return 0;
  s = getenv("DPSNN_SHM_SLOT_MB");
  g_slot_bytes = (size_t)(s ? atol(s) : 1024) << 20;
  s = getenv("DPSNN_SHM_TIMEOUT_S");
  if (s) g_timeout_s = atof(s);
  const size_t total = 4096 + (size_t)n * g_slot_bytes;
  void *p = mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
  if (p == MAP_FAILED) fail("mmap of the shared staging area failed");
  g_hdr = (shm_header *)p;
  atomic_init(&g_hdr->arrive, 0u);
  atomic_init(&g_hdr->gen, 0u);
  atomic_init(&g_hdr->failed, 0);
  g_slots = (char *)p + 4096;
  fflush(stdout);
  fflush(stderr);
  const pid_t parent = getpid();
  for (int r = 1; r < n; r++) {
    const pid_t pid = fork();
    if (pid < 0) fail("fork failed");
    if (pid == 0) {
      prctl(PR_SET_PDEATHSIG, SIGKILL);
      if (getppid() != parent) _exit(3);
      g_rank = r;
      return 0;
    }
    g_child[r] = pid;
  }
  g_rank = 0;
  return 0;
}

int MPI_Finalize(void) {
  barrier();
  if (g_rank == 0 && g_size > 1) {
    int bad = 0;
    for (int r = 1; r < g_size; r++) {
      int st = 0;
      if (waitpid(g_child[r], &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
    }
    if (bad) fprintf(stderr, "mpi_shm: a rank exited abnormally\n");
  }
  return 0;
}

int MPI_Abort(MPI_Comm c, int code) {
  (void)c;
  if (g_hdr) atomic_store(&g_hdr->failed, 1);
  exit(code);
}
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = g_rank; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = g_size; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; barrier(); return 0; }
double MPI_Wtime(void) { return now_s(); }
int MPI_Get_address(const void *loc, MPI_Aint *addr) { *addr = (MPI_Aint)loc; return 0; }
int MPI_Type_create_struct(int count, const int bl[], const MPI_Aint disp[], const MPI_Datatype types[],
                           MPI_Datatype *nt) {
  /* extent: the end of the last block, padded to the largest alignment of
   * the member types (an int aligns to 4, a double to 8), as MPI does */
  MPI_Aint ext = 0, align = 1;
  for (int i = 0; i < count; i++) {
    const MPI_Aint sz = (MPI_Aint)type_size(types[i]);
    MPI_Aint end = disp[i] + (MPI_Aint)bl[i] * sz;
    if (end > ext) ext = end;
    const MPI_Aint a = sz >= 8 ? 8 : (sz >= 4 ? 4 : (sz >= 2 ? 2 : 1));
    if (a > align) align = a;
  }
  ext = (ext + align - 1) & ~(align - 1);
  *nt = -(MPI_Datatype)ext;
  return 0;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_get_extent(MPI_Datatype t, MPI_Aint *lb, MPI_Aint *ext) {
  *lb = 0;
  *ext = (MPI_Aint)type_size(t);
  return 0;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
  *count = st ? (int)(st->count_bytes / (int)type_size(t)) : 0;
  return 0;
}

/* Generic exchange: rank g_rank sends seg_bytes[d] bytes starting at
 * src + seg_off[d] to every rank d and receives into dst + rd_off[s] at most
 * rd_cap[s] bytes from every rank s. */
static void exchange(const char *src, const size_t *seg_off, const size_t *seg_bytes, char *dst,
                     const size_t *rd_off, const size_t *rd_cap) {
  slot_meta *m = meta(g_rank);
  char *pl = payload(g_rank);
  size_t used = 0;
  for (int d = 0; d < g_size; d++) {
    if (sizeof(slot_meta) + used + seg_bytes[d] > g_slot_bytes) fail("staging slot too small (DPSNN_SHM_SLOT_MB)");
    m->off[d] = used;
    m->bytes[d] = seg_bytes[d];
    if (seg_bytes[d]) memcpy(pl + used, src + seg_off[d], seg_bytes[d]);
    used += (seg_bytes[d] + 15) & ~(size_t)15;
  }
  barrier();
  for (int s = 0; s < g_size; s++) {
    const slot_meta *ms = meta(s);
    const size_t b = ms->bytes[g_rank];
    if (b > rd_cap[s]) fail("receive buffer smaller than the message");
    if (b) memcpy(dst + rd_off[s], payload(s) + ms->off[g_rank], b);
  }
  barrier();
}

int MPI_Alltoall(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, MPI_Comm c) {
  (void)c;
  size_t so[MAX_RANKS], sbt[MAX_RANKS], ro[MAX_RANKS], rcap[MAX_RANKS];
  const size_t rbytes = (size_t)rc * type_size(rt);
  const char *src = (const char *)sb;
  size_t sbytes = (size_t)sc * type_size(st);
  char *tmp = NULL;
  if (sb == MPI_IN_PLACE) {   /* the send data is in the receive buffer */
    sbytes = rbytes;
    tmp = (char *)malloc(rbytes * (size_t)g_size + 1);
    memcpy(tmp, rb, rbytes * (size_t)g_size);
    src = tmp;
  }
  for (int r = 0; r < g_size; r++) {
    so[r] = (size_t)r * sbytes;
    sbt[r] = sbytes;
    ro[r] = (size_t)r * rbytes;
    rcap[r] = rbytes;
  }
  exchange(src, so, sbt, (char *)rb, ro, rcap);
  free(tmp);
  return 0;
}

int MPI_Alltoallv(const void *sb, const int sc[], const int sd[], MPI_Datatype st, void *rb, const int rc[],
                  const int rd[], MPI_Datatype rt, MPI_Comm c) {
  (void)c;
  size_t so[MAX_RANKS], sbt[MAX_RANKS], ro[MAX_RANKS], rcap[MAX_RANKS];
  const size_t es = type_size(st), er = type_size(rt);
  for (int r = 0; r < g_size; r++) {
    so[r] = (size_t)sd[r] * es;
    sbt[r] = (size_t)sc[r] * es;
    ro[r] = (size_t)rd[r] * er;
    rcap[r] = (size_t)rc[r] * er;
  }
  exchange((const char *)sb, so, sbt, (char *)rb, ro, rcap);
  return 0;
}

int MPI_Allgather(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, MPI_Comm c) {
  (void)c;
  size_t so[MAX_RANKS], sbt[MAX_RANKS], ro[MAX_RANKS], rcap[MAX_RANKS];
  const size_t rbytes = (size_t)rc * type_size(rt);
  const char *src = (const char *)sb;
  size_t sbytes = (size_t)sc * type_size(st);
  if (sb == MPI_IN_PLACE) {
    src = (const char *)rb + (size_t)g_rank * rbytes;
    sbytes = rbytes;
  }
  for (int r = 0; r < g_size; r++) {
    so[r] = 0;
    sbt[r] = sbytes;
    ro[r] = (size_t)r * rbytes;
    rcap[r] = rbytes;
  }
  exchange(src, so, sbt, (char *)rb, ro, rcap);
  return 0;
}

static int p2p(const char *what) {
  char msg[96];
  snprintf(msg, sizeof msg, "%s is not implemented (run with env_collectivesAlgo=0)", what);
  fail(msg);
  return 1;
}
int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c;
  return p2p("MPI_Send");
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; (void)r;
  return p2p("MPI_Isend");
}
int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st;
  return p2p("MPI_Recv");
}
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)r;
  return p2p("MPI_Irecv");
}
int MPI_Wait(MPI_Request *r, MPI_Status *st) { (void)r; (void)st; return 0; }
int MPI_Waitall(int n, MPI_Request r[], MPI_Status st[]) { (void)n; (void)r; (void)st; return 0; }
