/*
 * dpsnn_b200.h -- C ABI of the B200 engine for DPSNN's per-timestep loop.
 *
 * One engine simulates one DPSNN network (all env_globH ranks of it) on one
 * GPU.  Plain C types only; every call returns 0 on success or a negative
 * DPSNN_E_* code, with a message available from dpsnn_last_error().
 *
 * Correspondence with the reference interface each call replaces:
 *   dpsnn_params_from_env  <- getParameters()             DPSNN_getParameters.c:23-831
 *                             + describeConnectome() file parsing
 *                                                         DPSNN_LIFCAconnectome.cpp:16-487
 *                             + readPlasticityParametersFile()
 *                                                         DPSNN_getParameters.c:900-1053
 *   dpsnn_create           <- localNetClass::init()       DPSNN_localNet_init.c:43-307
 *                             (synapse generation, connectome sort, neuron init,
 *                              RNG seeding), one call for all ranks
 *   dpsnn_step             <- localNetClass::completeTimeStep_ms()
 *                                                         DPSNN_localNet_sim.c:22-307
 *                             (+ stopWatch advance, localNetProcess.c:120-137)
 *   dpsnn_spikes           <- the spike list handed to statSpikesClass::write
 *                                                         DPSNN_localNet_sim.c:222-226
 *   dpsnn_backward_synapses<- backwardSynList of rank h   DPSNN_localNet_init.c:591-617
 *   dpsnn_ltp_probe        <- the synPeriodicProbe_A/B records
 *                                                         DPSNN_localNet_sim.c:360-397
 *   dpsnn_stdp_events      <- the STDPevent records       DPSNN_neuron_sim.c:152-166,230-246
 *   dpsnn_destroy         <- process exit (the reference never frees)
 * The DAL process trio localNetProcess_init/fire/finish and getParameters
 * themselves, with C++ linkage as in the reference, are exported by
 * libdpsnn_localnet.so (dpsnn_localnet.h).
 */
#ifndef DPSNN_B200_H
#define DPSNN_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPSNN_MAX_SUBPOP 27

enum {
  DPSNN_OK = 0,
  DPSNN_E_PARAM = -1,      /* invalid or missing parameter / input file */
  DPSNN_E_CUDA = -2,       /* CUDA runtime error */
  DPSNN_E_NOMEM = -3,      /* device or host allocation failed */
  DPSNN_E_CAPACITY = -4,   /* a fixed capacity was exceeded */
  DPSNN_E_MODEL = -5,      /* a condition on which the reference exits */
  DPSNN_E_STATE = -6       /* call not valid in the engine's current state */
};

/* Everything the reference reads from env_* variables and its four input
 * files, already parsed (floats as atof() -> float gives them). */
typedef struct {
  /* grid and sub-populations (column.txt, env_CFX/env_CFY) */
  uint32_t cfx, cfy, nsub;
  uint32_t count[DPSNN_MAX_SUBPOP];
  float JExt[DPSNN_MAX_SUBPOP], DJExt[DPSNN_MAX_SUBPOP], NuExt[DPSNN_MAX_SUBPOP];
  float Tau[DPSNN_MAX_SUBPOP], Theta[DPSNN_MAX_SUBPOP], H[DPSNN_MAX_SUBPOP];
  float Tarp[DPSNN_MAX_SUBPOP], AlphaC[DPSNN_MAX_SUBPOP], TauC[DPSNN_MAX_SUBPOP];
  float gC[DPSNN_MAX_SUBPOP];
  /* connectivity.txt, [src*nsub + tgt] */
  float J[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP];
  float DJ[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP];
  float DMin[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP];
  float DMax[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP];
  uint32_t stencil_dim;           /* env_stencilDim (explicit stencil) */
  /* spec[((src*nsub + tgt)*stencil_dim + x)*stencil_dim + y] */
  const float *spec;
  /* bathEfficacy.txt, bath[x*stencil_dim + y] */
  const uint32_t *bath;
  /* env_* */
  uint32_t D;                     /* env_D */
  uint32_t glob_h;                /* env_globH: ranks whose RNG streams are emulated */
  uint32_t global_seed;           /* env_globalSeed */
  uint32_t total_sim_time_ms;     /* env_totalSimTime_ms */
  uint32_t start_plasticity_ms, stop_plasticity_ms;
  float min_syn_weight_f;         /* env_minSynWeight_f */
  /* plasticity.txt (Song STDP) */
  float stdp_antiCausalCoeff, stdp_multiplier, stdp_tau_ms;
  float stdp_causalMax, stdp_antiCausalMax, stdp_tauDecay_s, stdp_drift;
  /* output controls (env_*) used by the stat writers */
  uint32_t moduloSec, ratesSampling, startStatFiles_s, stopStatFiles_s;
  uint32_t startRatesPerPop_s, stopRatesPerPop_s;
  uint32_t spikes_writeDisable, statRatesPerPop_writeDisable, howManyOutputFiles;
  /* 0: getRandomDelay_UNI (reference built with -DDelayUniform);
   * 1: getRandomDelay_EXP (the reference Makefile's default).  The reference
   * selects it at compile time; here DPSNN_DELAY_DISTRIBUTION=exponential. */
  uint32_t delay_exponential;
} dpsnn_params;

/* Engine capacities (0 = default). */
typedef struct {
  uint32_t events_per_neuron;     /* per-target event slots per step (default
                                     1024, halved while they would exceed
                                     16 GiB; at most 4096) */
  uint32_t overflow_events;       /* events beyond that, per step (default 1<<22) */
  int device;                     /* CUDA device ordinal (default current) */
} dpsnn_options;

typedef struct dpsnn_engine dpsnn_engine;

/* Fill *p from the env_* variables and the input files in `workdir`
 * (NULL = current directory).  Arrays spec/bath point into storage owned by
 * the library until the next call of this function in the same thread. */
int dpsnn_params_from_env(const char *workdir, dpsnn_params *p);

/* Build the network on the GPU: synapse generation, connectome sort, neuron
 * and RNG initialisation.  opts may be NULL. */
int dpsnn_create(const dpsnn_params *p, const dpsnn_options *opts, dpsnn_engine **out);
void dpsnn_destroy(dpsnn_engine *e);

/* Run nsteps 1 ms steps (asynchronously; results are read by the calls below,
 * which synchronise). */
int dpsnn_step(dpsnn_engine *e, uint32_t nsteps);
/* Batched form: nsteps steps of each of n independent engines, queued one
 * step of every engine at a time, so that their kernels overlap on the
 * device; each engine's results are those of dpsnn_step on it alone.
 * Asynchronous like dpsnn_step.  If queuing fails for engine i in round k,
 * engines 0..i-1 have k+1 steps queued and engines i..n-1 have k:
 * dpsnn_time_ms tells each engine's count. */
int dpsnn_step_many(dpsnn_engine *const *engines, uint32_t n, uint32_t nsteps);
/* Block until all queued steps are done; reports a deferred device error. */
int dpsnn_sync(dpsnn_engine *e);

/* Graphs of batched steps.  dpsnn_graph_create records nsteps steps (a
 * positive multiple of 80) of the n engines, queued as dpsnn_step_many
 * queues them, into one CUDA graph; nothing runs.  Every engine must have run
 * its first step, with kernel timing, the STDP event log and the LTP probe
 * off.  dpsnn_graph_run advances every engine by nsteps steps in one launch,
 * after the work already queued on the engines; later work on them follows
 * it.  A graph encodes the engines' ring slots and step parities, so a run
 * is refused unless every engine is at the step (mod 80) it was recorded at.
 * The engines must outlive the graph.  No counterpart in the reference, whose
 * process runs one network per MPI job. */
typedef struct dpsnn_graph dpsnn_graph;
int dpsnn_graph_create(dpsnn_engine *const *engines, uint32_t n, uint32_t nsteps, dpsnn_graph **out);
int dpsnn_graph_run(dpsnn_graph *g);
void dpsnn_graph_destroy(dpsnn_graph *g);

/* Grid sizes (blocks) of the delivery, warp-sort and heavy-run kernels; 0
 * restores the default (8, 8 and 16 blocks per SM, sized for a network that
 * fills the GPU).  Every kernel loops over its work, so the results do not
 * depend on them; a small network stepped beside others runs faster on
 * smaller grids.  Takes effect for steps queued (or graphs recorded) after
 * the call.  No counterpart in the reference. */
int dpsnn_set_launch_shape(dpsnn_engine *e, uint32_t deliver_blocks, uint32_t heavy_sort_blocks,
                           uint32_t heavy_run_blocks);

/* Sizes. */
uint32_t dpsnn_glob_n(const dpsnn_engine *e);
uint32_t dpsnn_time_ms(const dpsnn_engine *e);        /* steps completed */
uint64_t dpsnn_synapse_count(const dpsnn_engine *e);
/* Synaptic events delivered since creation. */
uint64_t dpsnn_events_delivered(const dpsnn_engine *e);

/* Spike list detected at step t_ms (one of the last 80 steps): ascending
 * neuron index, with emission times.  *count receives the number of spikes;
 * at most cap are written.  Waits only until that step's list is final (its
 * compaction), so the rest of the step and any later queued steps keep
 * running; reports device errors raised so far. */
int dpsnn_spikes(dpsnn_engine *e, uint32_t t_ms, uint32_t *ids, double *te,
                 uint32_t cap, uint32_t *count);

/* Spike lists of the n consecutive steps t0 .. t0+n-1 (all among the last 80
 * steps), concatenated in step order into ids/te (cap entries each), with
 * counts[k] the spikes of step t0+k.  One wait for the whole run: for a
 * caller collecting a raster every few tens of steps (the served form).  No
 * counterpart in the reference, which writes each step's list to its spike
 * file (DPSNN_stat.c:290). */
int dpsnn_spikes_range(dpsnn_engine *e, uint32_t t0, uint32_t n, uint32_t *ids, double *te, uint64_t cap,
                       uint32_t *counts);
/* Device memory the engine holds (its network, state and buffers), for
 * callers that budget device memory (admission of served jobs). */
uint64_t dpsnn_device_bytes(const dpsnn_engine *e);

/* Backward synapse list of rank h in the reference's memory order (sorted by
 * delay, source rank, generation order), as dumped by synapticListReport.
 * Arrays of dpsnn_rank_synapse_count() entries; any pointer may be NULL. */
uint64_t dpsnn_rank_synapse_count(dpsnn_engine *e, uint32_t h);
int dpsnn_backward_synapses(dpsnn_engine *e, uint32_t h, uint32_t *pre, uint32_t *post,
                            uint8_t *delay, uint8_t *kind, int16_t *weight, float *tderiv);

/* LTP probe: the synapses just before and just after each once-per-second
 * plasticity update, the records statSynPeriodicProbeA/B write inside
 * longTermPlasticity (DPSNN_localNet_sim.c:360-364 and :391-397).
 * dpsnn_enable_ltp_probe allocates 10 B per synapse on the device; it is
 * called before the first step, on an engine with plasticity switched on.
 * dpsnn_ltp_probe waits for the queued steps, then returns, for the last
 * update run (its step in *t_ms), rank h's synapses in the order of
 * dpsnn_backward_synapses: the weight and time derivative before the update,
 * and the weight and time derivative after it, the latter before its
 * decay.  Any array pointer may be NULL. */
int dpsnn_enable_ltp_probe(dpsnn_engine *e);
int dpsnn_ltp_probe(dpsnn_engine *e, uint32_t h, uint32_t *t_ms, int16_t *w_before, float *td_before,
                    int16_t *w_after, float *td_after);

/* STDP event log: the records statSTDPevent writes on rank 0
 * (DPSNN_neuron_sim.c:152-166, causal, and :230-246, anti-causal): every
 * non-zero STDP contribution on a synapse of rank 0 whose presynaptic and
 * postsynaptic neurons are both rank-0 neurons.  dpsnn_enable_stdp_events
 * allocates the log (32 MiB, 2^21 records a step) before the first step, on an
 * engine with plasticity switched on.  The log holds the last step queued:
 * dpsnn_stdp_events waits for it and returns its step in *t_ms and its
 * records in the reference's order (causal events by ascending postsynaptic
 * neuron, each neuron's synapses in backward-list order; then anti-causal
 * events in delivery order); *count receives the number of records, at most
 * cap are written.  A step with more records fails with DPSNN_E_CAPACITY.
 * Read it after every dpsnn_step(e, 1) to see every step. */
#define DPSNN_STDP_LOG_CAP (1u << 21)
int dpsnn_enable_stdp_events(dpsnn_engine *e);
int dpsnn_stdp_events(dpsnn_engine *e, uint32_t *t_ms, uint32_t *pre, uint32_t *post, float *contribution,
                      uint32_t cap, uint32_t *count);

/* Neuron state, global neuron index order; any pointer may be NULL. */
int dpsnn_state(dpsnn_engine *e, double *v, double *c, double *tr, double *te, double *nb);
/* Per-neuron bath parameters (invNuExt, maxExternCurrentCount). */
int dpsnn_bath_params(dpsnn_engine *e, double *inv_nu_ext, uint32_t *max_ext);

/* Seconds of device time spent in each kernel since creation, and the
 * number of launches timed, in DPSNN_TIMING_SLOTS slots: 0 compaction,
 * 1 delivery, 2 bath, 3 neuron update (neurons with few events),
 * 4 plasticity, 5/6/7 heavy-neuron sort / update / single-block update.
 * Counted only while timing is enabled with dpsnn_set_timing(e, 1), which
 * records CUDA events around each launch without synchronising. */
#define DPSNN_TIMING_SLOTS 8
int dpsnn_set_timing(dpsnn_engine *e, int enable);
int dpsnn_kernel_times(dpsnn_engine *e, double *seconds, uint64_t *launches);
/* Kernels enqueued by dpsnn_step since creation. */
uint64_t dpsnn_kernel_launches(const dpsnn_engine *e);
/* The cudaStream_t all of the engine's work is enqueued on (for timing
 * with CUDA events by the caller). */
void *dpsnn_cuda_stream(const dpsnn_engine *e);

/* Spike list of emulated rank h at step t_ms (one of the last 80 steps):
 * the entries of dpsnn_spikes() whose neuron belongs to rank h, same order.
 * No counterpart in the reference: it is the spike list one reference rank
 * holds (spikingNeuronIdsInThisTimeStep, DPSNN_localNet_sim.c:222-226), read
 * without any device allocation, for callers that must not allocate -- a
 * real-time loop reading a rank's raster every 1 ms step (cudaMalloc and
 * cudaFree synchronise the whole device and can take longer than a step) or
 * a host that budgets every byte of device memory itself.  The gather goes
 * through a fixed scratch area in the library image holding
 * DPSNN_NOALLOC_MAX_SPIKES spikes (384 KiB); engines whose ranks hold more
 * neurons get DPSNN_E_CAPACITY.  Like dpsnn_spikes it waits only for the
 * compaction of step t_ms, so later queued steps keep running.  The first
 * call on a device looks up the scratch's device address (once per device),
 * so that call should come before any stream capture.  There is one scratch
 * per device and process: calls that overlap in time on the same device
 * (from several threads, or several engines on one device) race on it and
 * must be serialised by the caller. */
#define DPSNN_NOALLOC_MAX_SPIKES 32768
int dpsnn_rank_spikes_noalloc(dpsnn_engine *e, uint32_t t_ms, uint32_t h, uint32_t *ids, double *te,
                              uint32_t cap, uint32_t *count);

const char *dpsnn_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
