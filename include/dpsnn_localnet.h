/*
 * dpsnn_localnet.h -- drop-in replacement of DPSNN's localNet process.
 *
 * libdpsnn_localnet.so exports the DAL process trio with the signatures and
 * C++ linkage of the reference (localNetProcess.h:72-74, compiled as C++ by
 * the reference Makefile:12), so that the reference's MPI main
 * (DPSNN_mainUnderMPI.c:51-85) links against it in place of its own
 * localNetProcess.o and engine objects:
 *
 *   localNetProcess_init   <- localNetProcess.c:42-96: getParameters, stat
 *                             preparation, localNetClass::init -- here
 *                             dpsnn_params_from_env + dpsnn_create
 *   localNetProcess_fire   <- localNetProcess.c:98-157: one 1 ms step
 *                             (localNetClass::completeTimeStep_ms), the spike
 *                             and rate files of that step (DPSNN_stat.c), the
 *                             stopWatch advance; returns 0, and 1 once
 *                             env_totalSimTime_ms steps are done
 *   localNetProcess_finish <- localNetProcess.c:159-172: the
 *                             FiringsInChronoWindow_h<h>.stat files; frees
 *                             the device memory
 *
 * The process simulates the whole network: all env_globH ranks' RNG streams
 * are emulated on one GPU, and the output files of every rank h are written
 * (spikes-sec<s>-C<C>-H<H>-h<hhh>.dat, ratesPerPop-..., as the env_globH
 * reference processes would write them together).  Run it as a single
 * process (MPI world size 1).
 *
 * p->local is not read or written: the engine state lives in the library
 * (one localNet per process, as in the reference, localNetProcess.h:52).
 * Errors print "ERROR ..." and exit(0), as the reference does.
 *
 * The device is CUDA device 0 unless DPSNN_DEVICE names another ordinal.
 */
#ifndef DPSNN_LOCALNET_H
#define DPSNN_LOCALNET_H

#include <stdint.h>
#include "dpsnn_b200.h"

#ifndef DAL_H
/* The process handle of the reference's dal.h:24-42, same layout and tag. */
typedef struct _local_states *LocalState;
struct _process;
typedef void (*ProcessInit)(struct _process *);
typedef void (*ProcessFinish)(struct _process *);
typedef int (*ProcessFire)(struct _process *);
typedef void *WPTR;
typedef struct _process {
  LocalState local;
  ProcessInit init;
  ProcessFire fire;
  ProcessFinish finish;
  WPTR wptr;
} DALProcess;
#endif

#ifdef __cplusplus
void localNetProcess_init(DALProcess *p);
int localNetProcess_fire(DALProcess *p);
void localNetProcess_finish(DALProcess *p);

/* Handle of the engine the trio drives (NULL before init / after finish),
 * for callers that also want the C ABI of dpsnn_b200.h. */
struct dpsnn_engine *localNetProcess_engine(void);

/* getParameters (DPSNN_getParameters.c:23-831, declared at
 * DPSNN_getParameters.h:7 with C++ linkage): the run's parameters from the
 * env_* variables and the input files of the current directory, by the
 * reference's rules; on an error it prints "ERROR ..." and exits with status
 * 0, as the reference does.  loc_h is accepted for the signature's sake: every
 * rank of a run reads the same parameters (the rank number only selects the
 * emulated rank's output files).  The result is the engine's parameter
 * block (dpsnn_b200.h), not the reference's struct DPSNN_parameters: a
 * caller compiled against the reference's header must not call this one. */
dpsnn_params getParameters(const uint32_t loc_h);
#endif

#endif
