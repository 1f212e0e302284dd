/*
 * dpsnn_oracle -- CPU restatement of DPSNN's per-timestep LIFCA loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the parity
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg compare the
 * GPU engine against.  It is never linked into, loaded by or called from the
 * product.  It is pinned against the reference itself (oracle/_ref/dpsnn_ref,
 * built from the reference sources by oracle/Makefile) through the committed
 * fixtures under tests/golden/.
 *
 * It restates, in plain single-threaded C, the algorithm of the reference at
 * the cited lines, with the reference's float/double promotions kept
 * operation for operation (built with -ffp-contract=off, like the x86-64
 * SSE2 reference build):
 *   ran3 / SetRandomSeed / NormDev   randdev.c:116-196,477-502,584-606
 *   Gaussian LUT, roundr2i           erflib.c:41-181
 *   synapse generation               DPSNN_LIFCAcorticalModuleGen.cpp:62-220,
 *                                    :247-338; DPSNN_LIFCAconnectome.cpp:513-823,
 *                                    :871-887, :1079-1133
 *   connectome sort / offsets        DPSNN_localNet_init.c:311-740
 *   one 1 ms step                    DPSNN_localNet_sim.c:22-307, :620-999
 *   neuron update                    DPSNN_neuron_sim.c:289-300, :522-824, :844-865
 *   STDP                             DPSNN_neuron_sim.c:45-277,
 *                                    DPSNN_localNet_sim.c:312-414
 * Several MPI ranks (env_globH) are emulated in one process: each rank keeps
 * its own RNG state, its own backward synapse list and its own delay rings,
 * exactly as separate reference processes would.
 */
#ifndef DPSNN_ORACLE_H
#define DPSNN_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define DPO_MAX_SUB 27
#define DPO_MAX_STENCIL 8   /* stencilDim limit of this restatement */

typedef struct {
  uint32_t cfx, cfy;            /* env_CFX, env_CFY */
  uint32_t nsub;                /* rows of column.txt */
  uint32_t count[DPO_MAX_SUB];  /* column.txt col 1 */
  /* column.txt cols 2..11 as the float values atof()->float gives */
  float JExt[DPO_MAX_SUB], DJExt[DPO_MAX_SUB], NuExt[DPO_MAX_SUB];
  float Tau[DPO_MAX_SUB], Theta[DPO_MAX_SUB], H[DPO_MAX_SUB], Tarp[DPO_MAX_SUB];
  float AlphaC[DPO_MAX_SUB], TauC[DPO_MAX_SUB], gC[DPO_MAX_SUB];
  /* connectivity.txt, [src][tgt] */
  float J[DPO_MAX_SUB][DPO_MAX_SUB], DJ[DPO_MAX_SUB][DPO_MAX_SUB];
  float DMin[DPO_MAX_SUB][DPO_MAX_SUB], DMax[DPO_MAX_SUB][DPO_MAX_SUB];
  /* spec[src][tgt][x][y], x,y in 0..stencil_dim-1 */
  float spec[DPO_MAX_SUB][DPO_MAX_SUB][DPO_MAX_STENCIL][DPO_MAX_STENCIL];
  uint32_t stencil_dim;         /* env_stencilDim, explicit stencil */
  uint32_t bath[DPO_MAX_STENCIL][DPO_MAX_STENCIL]; /* bathEfficacy.txt [x][y] */
  uint32_t D;                   /* env_D */
  uint32_t glob_h;              /* env_globH: emulated ranks */
  uint32_t global_seed;         /* env_globalSeed */
  uint32_t start_plasticity_ms, stop_plasticity_ms;
  float min_syn_weight_f;       /* env_minSynWeight_f */
  /* plasticity.txt (defaults of readPlasticityParametersFile if absent) */
  float stdp_antiCausalCoeff, stdp_multiplier, stdp_tau_ms;
  float stdp_causalMax, stdp_antiCausalMax, stdp_tauDecay_s, stdp_drift;
  /* delay distribution: 0 = getRandomDelay_UNI (built with -DDelayUniform),
   * 1 = getRandomDelay_EXP (the reference Makefile's default) */
  uint32_t delay_exp;
} dpo_config;

typedef struct dpo_net dpo_net;

/* libm used by the restatement: 0 = the C library (what the reference
 * calls), 1 = correctly rounded exp()/log() (what the GPU engine computes). */
enum { DPO_LIBM_SYSTEM = 0, DPO_LIBM_CORRECTLY_ROUNDED = 1 };

dpo_net *dpo_create(const dpo_config *cfg, int libm_mode);
void dpo_destroy(dpo_net *n);
/* Synapses per (presynaptic neuron, delay slot), out[pre * D + delay]
 * (glob_n * D entries), by the generation alone: no synapse lists or delay
 * rings are built, so any network size fits.  0 on success. */
int dpo_outdegree_by_delay(const dpo_config *cfg, int libm_mode, uint16_t *out);
const char *dpo_last_error(void);

uint32_t dpo_glob_n(const dpo_net *n);
uint32_t dpo_loc_n(const dpo_net *n);
uint64_t dpo_total_synapses(const dpo_net *n);
/* Backward synapse list of rank h, in the reference's memory order. */
uint64_t dpo_rank_synapse_count(const dpo_net *n, uint32_t h);
void dpo_rank_synapses(const dpo_net *n, uint32_t h, uint32_t *pre, uint32_t *post,
                       uint8_t *delay, uint8_t *kind, int16_t *weight);
void dpo_rank_plasticity(const dpo_net *n, uint32_t h, float *tderiv, int32_t *last_act);
/* Per-neuron bath parameters set during generation. */
void dpo_bath_params(const dpo_net *n, double *inv_nu_ext, uint32_t *max_ext);
/* 256-entry bath LUT of sub-population s. */
void dpo_bath_lut(const dpo_net *n, uint32_t s, double *lut);
/* Write the BACKWARD dump of rank 0 exactly as synapticListReport does. */
int dpo_write_backward_dump(const dpo_net *n, const char *path);

/* Advance one 1 ms step (all ranks).  Returns the number of spikes detected
 * in this step, or -1 on an error the reference would exit on. */
int64_t dpo_step(dpo_net *n);
uint32_t dpo_time_ms(const dpo_net *n);
/* Spikes detected in the last step: rank-major, ascending neuron index. */
void dpo_last_spikes(const dpo_net *n, uint32_t *ids, double *times);
uint64_t dpo_last_event_count(const dpo_net *n);      /* synaptic events delivered */
uint64_t dpo_last_bath_count(const dpo_net *n);       /* bath events applied */
void dpo_state(const dpo_net *n, double *v, double *c, double *tr, double *te, double *nb);

/* Stand-alone restatements for known-answer tests. */
void dpo_ran3_sequence(int32_t seed, uint32_t n, double *out);
void dpo_normdev_sequence(int32_t seed, uint32_t n, double *out);
void dpo_gaussian_lut(double mu, double sigma, double xmin, double xmax, double *lut256);
uint32_t dpo_roundr2i(double r);
double dpo_exp_cr(double x);
double dpo_log_cr(double x);

#ifdef __cplusplus
}
#endif
#endif
