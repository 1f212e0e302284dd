// localnet_run.cpp -- a single-process main over the DAL trio, as the
// reference's MPI main drives it (DPSNN_mainUnderMPI.c:51-85 with one rank):
// init, fire until it returns non-zero, finish, and the CHRONO lines with the
// init and fire times.  Run it in a directory holding the input files, with
// the env_* variables set.
#include <cstdio>
#include <ctime>
#include <unistd.h>

#include "dpsnn_localnet.h"

static double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main() {
  static DALProcess proc;
  char host[256] = "NULL";
  gethostname(host, sizeof host);
  double t0 = now_s();
  localNetProcess_init(&proc);
  printf("CHRONO:MPI-MAIN h=0 on node %s - localNetProcess_init = %f sec \n", host, now_s() - t0);
  double fire = 0;
  int laps = 0, stop = 0;
  do {
    double a = now_s();
    stop = localNetProcess_fire(&proc);
    fire += now_s() - a;
    laps++;
  } while (stop == 0);
  localNetProcess_finish(&proc);
  printf("CHRONO:MPI-MAIN h=0 on node %s - mean localNetProcess_fire = %f sec on %d samples total fire time = %f\n",
         host, fire / laps, laps, fire);
  return 0;
}
