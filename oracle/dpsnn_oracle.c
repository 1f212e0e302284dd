/*
 * dpsnn_oracle.c -- CPU restatement of DPSNN's per-timestep LIFCA loop.
 * TEST INFRASTRUCTURE ONLY (see dpsnn_oracle.h): never part of the product.
 * Build: oracle/Makefile target `port` (gcc -ffp-contract=off, libquadmath).
 */
#define _GNU_SOURCE
#include "dpsnn_oracle.h"

#include <math.h>
#include <quadmath.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- errors */
static char g_err[512];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *dpo_last_error(void) { return g_err; }

/* ---------------------------------------------------------------- libm */
static int g_libm_mode = DPO_LIBM_SYSTEM;
double dpo_exp_cr(double x) { return (double)expq((__float128)x); }
double dpo_log_cr(double x) { return (double)logq((__float128)x); }
static double o_exp(double x) { return g_libm_mode ? dpo_exp_cr(x) : exp(x); }
static double o_log(double x) { return g_libm_mode ? dpo_log_cr(x) : log(x); }

/* ---------------------------------------------------------------- ran3
 * Knuth's subtractive generator as Numerical Recipes' ran3, with the
 * reference's |mj| tweak and its process-global state (randdev.c:116-196).
 * SetRandomSeed(s) sets idum=-s and draws once; for s=0 with an already
 * initialised table no re-initialisation happens (randdev.c:477-502).     */
typedef struct {
  int32_t ma[56];
  int32_t inext, inextp, iff, idum;
  int32_t nd_set;      /* NormDev's static Set   (randdev.c:588) */
  double nd_cache;     /* NormDev's static IIran (randdev.c:589) */
  uint64_t draws;
} o_rng;

#define MBIG 1000000000
#define MSEED 161803398
static double o_rand3(o_rng *g) {
  int32_t mj, mk;
  if (g->idum < 0 || g->iff == 0) {
    g->iff = 1;
    mj = MSEED - (g->idum < 0 ? -g->idum : g->idum);
    mj = (mj < 0 ? -mj : mj);
    mj %= MBIG;
    g->ma[55] = mj;
    mk = 1;
    for (int i = 1; i <= 54; i++) {
      int ii = (21 * i) % 55;
      g->ma[ii] = mk;
      mk = mj - mk;
      if (mk < 0) mk += MBIG;
      mj = g->ma[ii];
    }
    for (int k = 1; k <= 4; k++)
      for (int i = 1; i <= 55; i++) {
        g->ma[i] -= g->ma[1 + (i + 30) % 55];
        if (g->ma[i] < 0) g->ma[i] += MBIG;
      }
    g->inext = 0;
    g->inextp = 31;
    g->idum = 1;
  }
  if (++g->inext == 56) g->inext = 1;
  if (++g->inextp == 56) g->inextp = 1;
  mj = g->ma[g->inext] - g->ma[g->inextp];
  if (mj < 0) mj += MBIG;
  g->ma[g->inext] = mj;
  g->draws++;
  return mj * (1.0 / (double)MBIG);
}
static void o_seed(o_rng *g, int32_t s) {
  g->idum = -s;
  (void)o_rand3(g);
}
static double o_random(o_rng *g) { return o_rand3(g); }
/* Polar Box-Muller with the one-value cache (randdev.c:584-606). */
static double o_normdev(o_rng *g) {
  double fac, r, v1, v2;
  if (g->nd_set == 0) {
    do {
      v1 = (double)(2.0 * o_random(g) - 1.0);
      v2 = (double)(2.0 * o_random(g) - 1.0);
      r = v1 * v1 + v2 * v2;
    } while (r >= 1.0 || r == 0.0);
    fac = (double)sqrt(-2.0 * o_log(r) / r);
    g->nd_cache = v1 * fac;
    g->nd_set = 1;
    return v2 * fac;
  }
  g->nd_set = 0;
  return g->nd_cache;
}

void dpo_ran3_sequence(int32_t seed, uint32_t n, double *out) {
  o_rng g;
  memset(&g, 0, sizeof g);
  o_seed(&g, seed);
  for (uint32_t i = 0; i < n; i++) out[i] = o_random(&g);
}
void dpo_normdev_sequence(int32_t seed, uint32_t n, double *out) {
  o_rng g;
  memset(&g, 0, sizeof g);
  o_seed(&g, seed);
  for (uint32_t i = 0; i < n; i++) out[i] = o_normdev(&g);
}

/* ---------------------------------------------------------------- erflib
 * erfcc (NR rational Chebyshev fit), truncated-normal CDF bisection and the
 * midpoint LUT (erflib.c:41-181).  Runs on the host with the C library exp,
 * in both libm modes, as the reference does at init.                      */
static double o_erfcc(double x) {
  double t, z, ans;
  z = fabs(x);
  t = 1.0 / (1.0 + 0.5 * z);
  ans = t * exp(-z * z - 1.26551223 +
                t * (1.00002368 +
                     t * (0.37409196 +
                          t * (0.09678418 +
                               t * (-0.18628806 +
                                    t * (0.27886807 +
                                         t * (-1.13520398 +
                                              t * (1.48851587 +
                                                   t * (-0.82215223 + t * 0.17087277)))))))));
  return x >= 0.0 ? ans : 2.0 - ans;
}
static double o_normcum(double x, double mu, double sigma) {
  return 1 - 0.5 * o_erfcc((x - mu) / (sqrt(2.0) * sigma));
}
static double o_cutnormcum(double x, double mu, double sigma, double a, double b) {
  double n0 = o_normcum(a, mu, sigma);
  return (o_normcum(x, mu, sigma) - n0) / (o_normcum(b, mu, sigma) - n0);
}
static double o_findprob(double p, double mu, double sigma, double a, double b) {
  double err = 1e-6;
  int maxit = 256, i = 0;
  double x, xmin, xmax;
  if (p <= 0.0) return a;
  if (p >= 1.0) return b;
  xmin = a;
  xmax = b;
  while ((xmax - xmin) > err && i < maxit) {
    x = (xmax + xmin) * 0.5;
    if (o_cutnormcum(x, mu, sigma, a, b) < p)
      xmin = x;
    else
      xmax = x;
    i++;
  }
  return (xmax + xmin) * 0.5;
}
void dpo_gaussian_lut(double mu, double sigma, double xmin, double xmax, double *table) {
  if (sigma > 0.0) {
    double dp = 1.0 / 256.0, x0, x1 = xmin, p;
    int i;
    for (p = dp, i = 0; p <= 1.0; p += dp, i++) {
      x0 = x1;
      x1 = o_findprob(p, mu, sigma, xmin, xmax);
      table[i] = (x1 + x0) * 0.5;
    }
  } else {
    for (int i = 0; i < 256; i++) table[i] = mu;
  }
}
/* erflib.c:172-181; a negative result wraps modulo 2^32 as in the
 * reference's x86-64 build (truncation to 64 bits, low 32 bits kept). */
uint32_t dpo_roundr2i(double r) {
  double i = floor(r);
  if (i + 0.5 > r) return (uint32_t)(int64_t)i;
  return (uint32_t)(int64_t)(i + 1.0);
}

/* ---------------------------------------------------------------- network */
typedef struct {
  uint32_t pre, post;
  uint8_t delay, kind;
  int16_t weight;
  float tderiv;
  int32_t last_act;
} o_syn;

typedef struct {
  double t;       /* originalEmissionTime */
  uint32_t pre;
} o_axspike;

typedef struct {      /* one slot of axonalSpikeSchedulerClass::circBuffer */
  o_axspike *list;
  uint32_t count;
} o_slot;

#define O_RING 80     /* DSD__maxD */

typedef struct {
  o_rng rng;
  o_syn *syn;                 /* backward list */
  uint64_t nsyn;
  uint32_t *grp_count;        /* synDelaySourceHostDistribution [D][globH] */
  uint32_t *grp_offset;
  uint32_t *offset_by_delay;  /* [globN][D], 0xFFFFFFFF = none */
  uint32_t *src_syn_count;    /* synSourceHostDistribution.synCount[globH] */
  uint32_t *in_ptr, *in_idx;  /* per local neuron incoming synapses (STDP) */
  o_slot *ring;               /* [globH][O_RING] */
  int32_t read_index, next_free;
} o_rank;

struct dpo_net {
  dpo_config cfg;
  uint32_t nsub, npcm, glob_cft, glob_n, loc_n, glob_h, D, tab_neuron;
  uint32_t delay_min, delay_max, stencil;
  int32_t max_mod;
  uint32_t offset[DPO_MAX_SUB];
  double sp_Tau[DPO_MAX_SUB], sp_Theta[DPO_MAX_SUB], sp_H[DPO_MAX_SUB], sp_Tarp[DPO_MAX_SUB];
  double sp_AlphaC[DPO_MAX_SUB], sp_TauC[DPO_MAX_SUB], sp_gC[DPO_MAX_SUB], sp_NuExt[DPO_MAX_SUB];
  double sp_J[DPO_MAX_SUB][DPO_MAX_SUB], sp_DJ[DPO_MAX_SUB][DPO_MAX_SUB];
  double sp_DMin[DPO_MAX_SUB][DPO_MAX_SUB], sp_DMax[DPO_MAX_SUB][DPO_MAX_SUB];
  float *prob;                /* [s][t][2M+1][2M+1] */
  double lut[DPO_MAX_SUB][256];
  float f2w, w2f;             /* factorFloat_2_weightType, factorWeightType_2_Float */
  float causal_tab[128], anti_tab[128];
  /* neurons, global index */
  double *v, *c, *tr, *te, *nb, *inv_nu;
  uint32_t *max_ext;
  uint8_t *sub;
  uint8_t *fired;
  int32_t *last_spike_ms;
  uint32_t *fwd_hosts;        /* [globN][globH] forwardNeuralTargetDistrInHost */
  o_rank *rank;
  /* per-step scratch */
  uint32_t t;
  uint32_t *spk_ids;
  double *spk_t;
  uint32_t spk_n;
  uint32_t *rank_spk_start;   /* [globH+1] */
  float *in_w;                /* [locN][cap] delivered weights */
  double *in_frac;
  uint32_t *in_cnt;
  uint32_t in_cap;
  uint64_t last_events, last_bath;
  double *ev_time, *ev_val;   /* per-neuron merge scratch */
  uint32_t ev_cap;
};

uint32_t dpo_glob_n(const dpo_net *n) { return n->glob_n; }
uint32_t dpo_loc_n(const dpo_net *n) { return n->loc_n; }
uint32_t dpo_time_ms(const dpo_net *n) { return n->t; }

static float *prob_at(dpo_net *n, uint32_t s, uint32_t t, uint32_t x, uint32_t y) {
  return &n->prob[(((size_t)s * DPO_MAX_SUB + t) * n->stencil + x) * n->stencil + y];
}

static uint32_t subpop_of(const dpo_net *n, uint32_t in_cm) {
  for (uint32_t s = 0; s < n->nsub; s++)
    if (in_cm >= n->offset[s] && in_cm < n->offset[s] + n->cfg.count[s]) return s;
  return 0xFFFFFFFFu;
}

/* getEmptyRandomSynapses (DPSNN_LIFCAconnectome.cpp:1079-1133). */
static uint32_t empty_random_synapses(dpo_net *n, o_rng *g, float pf, uint32_t max_n) {
  double connectivity = (double)pf;
  double r = o_random(g);
  double P = connectivity, C = P;
  uint32_t k = 1;
  while ((C < r) && (k <= max_n)) {
    k++;
    P *= 1 - connectivity;
    C += P;
  }
  (void)n;
  return k;
}

/* getRandomDelay_UNI (DPSNN_LIFCAcorticalModuleGen.cpp:299-338). */
static uint32_t random_delay_uni(dpo_net *n, o_rng *g, uint32_t s, uint32_t t) {
  float outF, DMin, DMax, DelayMin, DelayMax, DelayStep, DelayNum;
  DMin = (float)n->sp_DMin[s][t];
  DMax = (float)n->sp_DMax[s][t];
  DelayMin = (float)n->delay_min;
  DelayMax = (float)n->delay_max;
  DelayNum = 80;
  DelayStep = (DelayMax - DelayMin) / DelayNum;
  DelayMax -= DelayStep / 2;
  DelayMin += DelayStep / 2;
  DMax = dpo_roundr2i((DMax - DelayMin) / DelayStep) * DelayStep + DelayMin;
  DMin = dpo_roundr2i((DMin - DelayMin) / DelayStep) * DelayStep + DelayMin;
  outF = ((o_random(g) * (DMax - DMin) + DMin - DelayMin) / DelayStep);
  (void)DelayMax;
  if (outF >= DelayNum) return 0xFFFFFFFFu;   /* the reference's exit at :322-326 */
  {
    const uint32_t outfunc = dpo_roundr2i(outF * DelayStep);
    if (outfunc > n->sp_DMax[s][t]) return 0xFFFFFFFFu;   /* :330-334 */
    return outfunc;
  }
}

/* getRandomDelay_EXP (DPSNN_LIFCAcorticalModuleGen.cpp:247-297): a truncated
 * exponential over [DMin, DMax), float/double promotions as written there.
 * The constant 1/log(0.05) is folded at compile time by the reference build,
 * i.e. correctly rounded.  Returns 0xFFFFFFFF on the reference's error exits. */
#define O_TAIL_NEGLECTED 0.05
static uint32_t random_delay_exp(dpo_net *n, o_rng *g, uint32_t s, uint32_t t) {
  float InvLogTN, outfuncF, DMin, DMax, DelayMin, DelayMax, DelayStep, DelayNum;
  uint32_t outfunc;
  DMin = (float)n->sp_DMin[s][t];
  DMax = (float)n->sp_DMax[s][t];
  DelayMin = (float)n->delay_min;
  DelayMax = (float)n->delay_max;
  DelayNum = 80;
  InvLogTN = (float)(1.0 / dpo_log_cr(O_TAIL_NEGLECTED));
  DelayStep = (DelayMax - DelayMin) / DelayNum;
  DelayMax -= DelayStep / 2;
  DelayMin += DelayStep / 2;
  DMax = dpo_roundr2i((DMax - DelayMin) / DelayStep) * DelayStep + DelayMin;
  DMin = dpo_roundr2i((DMin - DelayMin) / DelayStep) * DelayStep + DelayMin;
  outfuncF = (float)((((double)DMin + (double)(DMax - DMin - DelayStep) *
                       o_log(1.0 - o_random(g) * (1.0 - O_TAIL_NEGLECTED)) * (double)InvLogTN) -
                      (double)DelayMin) / (double)DelayStep);
  if (outfuncF >= DelayNum) return 0xFFFFFFFFu;
  outfunc = dpo_roundr2i(outfuncF * DelayStep);
  if (outfunc >= n->sp_DMax[s][t]) return 0xFFFFFFFFu;
  (void)DelayMax;
  return outfunc;
}

typedef struct { uint32_t glob, host, sub; } o_target;

static int generate(dpo_net *n, o_syn **gen_out, uint64_t **rank_gen_start_out, uint16_t *outdeg) {
  /* Returns all generated synapses in generation order (rank-major, since
   * each rank walks its own neurons) plus per-rank start offsets.  With
   * outdeg (count-only mode) nothing is stored: outdeg[pre * D + delay]
   * counts the synapses instead. */
  uint64_t cap = outdeg ? 1 : (1u << 20), cnt = 0;
  o_syn *gen = malloc(cap * sizeof *gen);
  uint64_t *rstart = calloc(n->glob_h + 1, sizeof *rstart);
  o_target *tl = malloc(sizeof(o_target) * 8192 * 4);
  uint32_t tl_cap = 8192 * 4;
  if (!gen || !rstart || !tl) { set_err("out of memory"); return -1; }
  for (uint32_t h = 0; h < n->glob_h; h++) {
    o_rng *g = &n->rank[h].rng;
    memset(g, 0, sizeof *g);
    o_seed(g, (int32_t)n->cfg.global_seed);          /* DPSNN_localNet_init.c:119 */
    rstart[h] = cnt;
    for (uint32_t i = 0; i < n->loc_n; i++) {
      uint32_t gn = i + n->loc_n * h;
      uint32_t cfy = (gn / n->npcm) / n->cfg.cfx, cfx = (gn / n->npcm) % n->cfg.cfx;
      uint32_t incm = gn % n->npcm, ssub = subpop_of(n, incm);
      n->sub[gn] = (uint8_t)ssub;
      /* initNeuralKind (DPSNN_neuron_init.c:99-115); Tr stays 0 (static storage) */
      n->v[gn] = n->sp_H[ssub];
      n->c[gn] = 0.0;
      n->te[gn] = -1000;
      n->nb[gn] = 0.0;
      n->tr[gn] = 0.0;
      n->fired[gn] = 0;
      if ((gn % n->tab_neuron) == 0) o_seed(g, (int32_t)(gn / n->tab_neuron));
      /* generateTargetNeuList, explicit stencil, no periodic boundaries */
      uint32_t tot = 0;
      for (uint32_t ts = 0; ts < n->nsub; ts++)
        for (uint32_t x = 0; x < n->stencil; x++)
          for (uint32_t y = 0; y < n->stencil; y++) {
            int32_t nx = (int32_t)cfx + (int32_t)x - n->max_mod;
            int32_t ny = (int32_t)cfy + (int32_t)y - n->max_mod;
            if (nx < 0 || nx >= (int32_t)n->cfg.cfx || ny < 0 || ny >= (int32_t)n->cfg.cfy) continue;
            float pf = *prob_at(n, ssub, ts, x, y);
            if (!(pf > 0)) continue;
            if (!(pf > 0.00001f)) {
              set_err("connection probability in (0, 1e-5] is not supported");
              return -1;
            }
            uint32_t in_cm = n->offset[ts] - 1;
            uint32_t last = n->offset[ts] + n->cfg.count[ts];
            uint32_t avail = last - in_cm;
            while ((in_cm += empty_random_synapses(n, g, pf, avail)) < last) {
              uint32_t tg = in_cm + (uint32_t)nx * n->npcm + (uint32_t)ny * n->npcm * n->cfg.cfx;
              if (tot >= tl_cap) {
                tl_cap *= 2;
                tl = realloc(tl, sizeof(o_target) * tl_cap);
              }
              tl[tot].glob = tg;
              tl[tot].host = tg / n->loc_n;
              tl[tot].sub = subpop_of(n, in_cm);
              tot++;
            }
          }
      if (tot >= 7500) { set_err("neuron %u generates %u >= DSD__maxM synapses", gn, tot); return -1; }
      for (uint32_t j = 0; j < tot; j++) {
        o_syn s;
        memset(&s, 0, sizeof s);
        s.pre = gn;
        s.post = tl[j].glob;
        if (!outdeg) n->fwd_hosts[(size_t)gn * n->glob_h + tl[j].host]++;
        uint32_t tsub = tl[j].sub;
        if (n->cfg.delay_exp) {
          const uint32_t dl = random_delay_exp(n, g, ssub, tsub);
          if (dl == 0xFFFFFFFFu) { set_err("ERROR: delay level generated beyond the allowed delays"); return -1; }
          s.delay = (uint8_t)dl;
        } else {
          const uint32_t dl = random_delay_uni(n, g, ssub, tsub);
          if (dl == 0xFFFFFFFFu) { set_err("ERROR: delay level generated beyond the allowed delays"); return -1; }
          s.delay = (uint8_t)dl;
        }
        s.kind = (uint8_t)ssub;
        float mean = (float)n->sp_J[ssub][tsub];
        float sigma = (float)n->sp_DJ[ssub][tsub] * mean;
        float wf;
        if (mean > 0.0) {
          do { wf = mean + o_normdev(g) * sigma; } while ((wf < 0.0) || (wf >= 2.0 * mean));
        } else {
          do { wf = mean + o_normdev(g) * sigma; } while ((wf <= 2.0 * mean) || (wf > 0));
        }
        if ((wf < n->cfg.min_syn_weight_f) || (wf > (-n->cfg.min_syn_weight_f))) {
          set_err("synaptic weight %f out of minSynWeight_f range", wf);
          return -1;
        }
        s.weight = (int16_t)(wf * n->f2w);
        if (outdeg) {
          outdeg[(size_t)gn * n->D + s.delay]++;
          continue;
        }
        if (cnt == cap) {
          cap *= 2;
          gen = realloc(gen, cap * sizeof *gen);
          if (!gen) { set_err("out of memory"); return -1; }
        }
        gen[cnt++] = s;
      }
      /* external bath (DPSNN_LIFCAcorticalModuleGen.cpp:201-211) */
      float nu = (float)n->sp_NuExt[ssub];
      uint32_t bx = cfx, by = cfy;
      if (bx >= n->cfg.cfx / 2) bx = -1 * (bx - n->cfg.cfx + 1);
      if (by >= n->cfg.cfy / 2) by = -1 * (by - n->cfg.cfy + 1);
      if (bx >= n->cfg.stencil_dim) bx = n->cfg.stencil_dim - 1;
      if (by >= n->cfg.stencil_dim) by = n->cfg.stencil_dim - 1;
      float cext = (float)n->cfg.bath[bx][by];
      if (cext != 0) {
        n->inv_nu[gn] = 1000.0 / (nu * cext);
        n->max_ext[gn] = (uint32_t)ceil(20 / n->inv_nu[gn]);
      } else {
        n->inv_nu[gn] = 0;
        n->max_ext[gn] = 0;
      }
    }
  }
  rstart[n->glob_h] = cnt;
  free(tl);
  if (outdeg) {
    free(gen);
    free(rstart);
    return 0;
  }
  *gen_out = gen;
  *rank_gen_start_out = rstart;
  return 0;
}

/* Backward list of rank hp: synapses aimed at hp, concatenated by source rank
 * (own local list in the middle, DPSNN_localNet_init.c:532-586), then the
 * stable counting sort by delay and the per-(pre,delay) offsets
 * (inflateIntermToBackwardSynList, :631-740, with D counters). */
static int build_rank(dpo_net *n, uint32_t hp, const o_syn *gen, const uint64_t *rstart) {
  o_rank *R = &n->rank[hp];
  uint64_t m = 0;
  for (uint64_t k = 0; k < rstart[n->glob_h]; k++)
    if (gen[k].post / n->loc_n == hp) m++;
  o_syn *interm = malloc((m ? m : 1) * sizeof *interm);
  R->syn = malloc((m ? m : 1) * sizeof *R->syn);
  R->src_syn_count = calloc(n->glob_h, sizeof(uint32_t));
  if (!interm || !R->syn || !R->src_syn_count) { set_err("out of memory"); return -1; }
  uint64_t w = 0;
  for (uint32_t h = 0; h < n->glob_h; h++)
    for (uint64_t k = rstart[h]; k < rstart[h + 1]; k++)
      if (gen[k].post / n->loc_n == hp) {
        interm[w++] = gen[k];
        R->src_syn_count[h]++;
      }
  R->nsyn = m;
  uint32_t D = n->D;
  uint64_t *cnt = calloc(D, sizeof *cnt), *off = calloc(D, sizeof *off), *act = calloc(D, sizeof *act);
  for (uint64_t k = 0; k < m; k++) {
    if (interm[k].delay >= D) { set_err("delay %u >= env_D", interm[k].delay); return -1; }
    cnt[interm[k].delay]++;
  }
  for (uint32_t d = 1; d < D; d++) off[d] = off[d - 1] + cnt[d - 1];
  R->grp_count = calloc((size_t)D * n->glob_h, sizeof(uint32_t));
  R->grp_offset = calloc((size_t)D * n->glob_h, sizeof(uint32_t));
  for (uint64_t k = 0; k < m; k++) {
    uint32_t d = interm[k].delay;
    uint64_t j = off[d] + act[d]++;
    R->syn[j] = interm[k];
    R->syn[j].last_act = 0;
    R->syn[j].tderiv = 0.0f;
    R->grp_count[(size_t)d * n->glob_h + interm[k].pre / n->loc_n]++;
  }
  for (uint32_t d = 0; d < D; d++) {
    R->grp_offset[(size_t)d * n->glob_h] = (uint32_t)off[d];
    for (uint32_t h = 1; h < n->glob_h; h++)
      R->grp_offset[(size_t)d * n->glob_h + h] =
          R->grp_offset[(size_t)d * n->glob_h + h - 1] + R->grp_count[(size_t)d * n->glob_h + h - 1];
  }
  R->offset_by_delay = malloc((size_t)n->glob_n * D * sizeof(uint32_t));
  memset(R->offset_by_delay, 0xFF, (size_t)n->glob_n * D * sizeof(uint32_t));
  for (uint32_t d = 0; d < D; d++) {
    uint64_t prev = (uint64_t)-1;
    for (uint64_t j = 0; j < cnt[d]; j++) {
      uint32_t p = R->syn[j + off[d]].pre;
      if (p != prev) {
        prev = p;
        R->offset_by_delay[(size_t)p * D + d] = (uint32_t)(off[d] + j);
      }
    }
  }
  /* incoming lists for causal STDP (DPSNN_localNet_init.c:225-237) */
  R->in_ptr = calloc(n->loc_n + 1, sizeof(uint32_t));
  R->in_idx = malloc((m ? m : 1) * sizeof(uint32_t));
  for (uint64_t k = 0; k < m; k++) R->in_ptr[R->syn[k].post % n->loc_n + 1]++;
  for (uint32_t i = 0; i < n->loc_n; i++) R->in_ptr[i + 1] += R->in_ptr[i];
  uint32_t *fill = calloc(n->loc_n, sizeof(uint32_t));
  for (uint64_t k = 0; k < m; k++) {
    uint32_t i = R->syn[k].post % n->loc_n;
    R->in_idx[R->in_ptr[i] + fill[i]++] = (uint32_t)k;
  }
  for (uint32_t i = 0; i < n->loc_n; i++)
    if (R->in_ptr[i + 1] - R->in_ptr[i] >= 2 * 7500) {
      set_err("too many synapses incoming on neuron %u", i + hp * n->loc_n);
      return -1;
    }
  free(fill);
  free(interm);
  free(cnt);
  free(off);
  free(act);
  /* delay rings (DPSNN_localNet_init.c:1073-1131, DPSNN_spike.c:193-207) */
  R->ring = calloc((size_t)n->glob_h * O_RING, sizeof(o_slot));
  for (uint32_t h = 0; h < n->glob_h; h++)
    for (uint32_t s = 0; s < O_RING; s++)
      R->ring[(size_t)h * O_RING + s].list = malloc(sizeof(o_axspike) * n->loc_n);
  R->read_index = -1;
  R->next_free = 0;
  return 0;
}

/* The configuration-derived tables of a network (sizes, sub-population
 * parameters, delay range, mirrored stencil probabilities, bath LUTs, STDP
 * tables); 0 on success. */
static int net_params(dpo_net *n, const dpo_config *cfg) {
  n->cfg = *cfg;
  n->nsub = cfg->nsub;
  if (n->nsub == 0 || n->nsub > DPO_MAX_SUB || cfg->stencil_dim == 0 ||
      cfg->stencil_dim > DPO_MAX_STENCIL || cfg->glob_h == 0 || cfg->D == 0 || cfg->D > O_RING) {
    set_err("configuration out of range");
    return -1;
  }
  n->npcm = 0;
  for (uint32_t s = 0; s < n->nsub; s++) {
    n->offset[s] = n->npcm;
    n->npcm += cfg->count[s];
  }
  n->glob_cft = cfg->cfx * cfg->cfy;
  if ((n->glob_cft % cfg->glob_h) != 0) {
    set_err("globCFT must be a multiple of globH");
    return -1;
  }
  float loc_cft = (float)n->glob_cft / (float)cfg->glob_h;
  n->loc_n = (uint32_t)(n->npcm * loc_cft);
  n->glob_h = cfg->glob_h;
  n->glob_n = n->loc_n * n->glob_h;
  n->D = cfg->D;
  n->tab_neuron = n->glob_n / n->glob_cft;   /* makeMaxCMFract=1 */
  n->f2w = -32767 / cfg->min_syn_weight_f;
  n->w2f = cfg->min_syn_weight_f / -32767;
  for (uint32_t s = 0; s < n->nsub; s++) {
    n->sp_Tau[s] = cfg->Tau[s];
    n->sp_Theta[s] = cfg->Theta[s];
    n->sp_H[s] = cfg->H[s];
    n->sp_Tarp[s] = cfg->Tarp[s];
    n->sp_AlphaC[s] = cfg->AlphaC[s];
    n->sp_TauC[s] = cfg->TauC[s];
    n->sp_gC[s] = cfg->gC[s];
    n->sp_NuExt[s] = cfg->NuExt[s];
    for (uint32_t t = 0; t < n->nsub; t++) {
      n->sp_J[s][t] = cfg->J[s][t];
      n->sp_DJ[s][t] = cfg->DJ[s][t];
      n->sp_DMin[s][t] = cfg->DMin[s][t];
      n->sp_DMax[s][t] = cfg->DMax[s][t];
    }
  }
  {
    double dmin = 1e36, dmax = 0;
    for (uint32_t s = 0; s < n->nsub; s++)
      for (uint32_t t = 0; t < n->nsub; t++) {
        if (n->sp_DMax[s][t] > dmax) dmax = n->sp_DMax[s][t];
        if (n->sp_DMin[s][t] < dmin) dmin = n->sp_DMin[s][t];
      }
    n->delay_min = (uint32_t)dmin;
    n->delay_max = (uint32_t)dmax;
  }
  n->max_mod = (int32_t)cfg->stencil_dim - 1;
  n->stencil = 2 * cfg->stencil_dim - 1;
  n->prob = calloc((size_t)DPO_MAX_SUB * DPO_MAX_SUB * n->stencil * n->stencil, sizeof(float));
  for (uint32_t s = 0; s < n->nsub; s++)
    for (uint32_t t = 0; t < n->nsub; t++)
      for (uint32_t x = 0; x <= (uint32_t)n->max_mod; x++)
        for (uint32_t y = 0; y <= (uint32_t)n->max_mod; y++) {
          float p = cfg->spec[s][t][x][y];
          *prob_at(n, s, t, n->max_mod + x, n->max_mod + y) = p;
          *prob_at(n, s, t, n->max_mod - x, n->max_mod + y) = p;
          *prob_at(n, s, t, n->max_mod - x, n->max_mod - y) = p;
          *prob_at(n, s, t, n->max_mod + x, n->max_mod - y) = p;
        }
  for (uint32_t s = 0; s < n->nsub; s++) {  /* initLUT (ModuleGen.cpp:347-356) */
    float J = (float)(double)cfg->JExt[s], DJ = (float)(double)cfg->DJExt[s];
    dpo_gaussian_lut(J, J * DJ, 0.0, 2.0 * J, n->lut[s]);
  }
  /* STDP tables (DPSNN_neuron_sim.c:74-91), float arithmetic */
  n->causal_tab[0] = cfg->stdp_causalMax * cfg->stdp_multiplier;
  n->causal_tab[1] = n->causal_tab[0];
  n->anti_tab[0] = cfg->stdp_antiCausalCoeff * cfg->stdp_antiCausalMax * cfg->stdp_multiplier;
  for (int i = 1; i < 128; i++) n->causal_tab[i] = (1 - 1 / cfg->stdp_tau_ms) * n->causal_tab[i - 1];
  for (int i = 1; i < 128; i++) n->anti_tab[i] = (1 - 1 / cfg->stdp_tau_ms) * n->anti_tab[i - 1];
  return 0;
}

/* Per-neuron arrays that generation writes (state initialisation, bath
 * parameters) and the per-rank RNG holders. */
static int net_neuron_arrays(dpo_net *n) {
  size_t N = n->glob_n;
  n->v = calloc(N, sizeof(double));
  n->c = calloc(N, sizeof(double));
  n->tr = calloc(N, sizeof(double));
  n->te = calloc(N, sizeof(double));
  n->nb = calloc(N, sizeof(double));
  n->inv_nu = calloc(N, sizeof(double));
  n->max_ext = calloc(N, sizeof(uint32_t));
  n->sub = calloc(N, 1);
  n->fired = calloc(N, 1);
  n->rank = calloc(n->glob_h, sizeof(o_rank));
  if (!n->v || !n->c || !n->tr || !n->te || !n->nb || !n->inv_nu || !n->max_ext || !n->sub || !n->fired ||
      !n->rank) {
    set_err("out of memory");
    return -1;
  }
  return 0;
}

int dpo_outdegree_by_delay(const dpo_config *cfg, int libm_mode, uint16_t *out) {
  /* Synapses per (presynaptic neuron, delay slot), out[pre * D + delay],
   * from the generation alone (no synapse lists, no delay rings). */
  g_libm_mode = libm_mode;
  dpo_net *n = calloc(1, sizeof *n);
  if (!n) return -1;
  int rc = net_params(n, cfg);
  if (rc == 0) rc = net_neuron_arrays(n);
  if (rc == 0) {
    memset(out, 0, (size_t)n->glob_n * n->D * sizeof(uint16_t));
    rc = generate(n, NULL, NULL, out);
  }
  dpo_destroy(n);
  return rc;
}

dpo_net *dpo_create(const dpo_config *cfg, int libm_mode) {
  g_libm_mode = libm_mode;
  dpo_net *n = calloc(1, sizeof *n);
  if (!n) return NULL;
  if (net_params(n, cfg) != 0 || net_neuron_arrays(n) != 0) {
    dpo_destroy(n);
    return NULL;
  }
  size_t N = n->glob_n;
  n->last_spike_ms = calloc(N, sizeof(int32_t));
  n->fwd_hosts = calloc(N * n->glob_h, sizeof(uint32_t));
  n->spk_ids = malloc(N * sizeof(uint32_t));
  n->spk_t = malloc(N * sizeof(double));
  n->rank_spk_start = calloc(n->glob_h + 1, sizeof(uint32_t));
  n->in_cap = 6000;   /* miniSimSpikes */
  n->in_w = malloc((size_t)n->loc_n * n->in_cap * sizeof(float));
  n->in_frac = malloc((size_t)n->loc_n * n->in_cap * sizeof(double));
  n->in_cnt = calloc(n->loc_n, sizeof(uint32_t));
  n->ev_cap = n->in_cap + 4096;
  n->ev_time = malloc(n->ev_cap * sizeof(double));
  n->ev_val = malloc(n->ev_cap * sizeof(double));
  for (size_t i = 0; i < N; i++) n->last_spike_ms[i] = -100000;
  o_syn *gen = NULL;
  uint64_t *rstart = NULL;
  if (generate(n, &gen, &rstart, NULL) != 0) { dpo_destroy(n); return NULL; }
  for (uint32_t h = 0; h < n->glob_h; h++)
    if (build_rank(n, h, gen, rstart) != 0) { free(gen); free(rstart); dpo_destroy(n); return NULL; }
  free(gen);
  free(rstart);
  /* dynamics stream: SetRandomSeed(loc_h) (DPSNN_localNet_init.c:283) */
  for (uint32_t h = 0; h < n->glob_h; h++) o_seed(&n->rank[h].rng, (int32_t)h);
  n->t = 0;
  return n;
}

void dpo_destroy(dpo_net *n) {
  if (!n) return;
  if (n->rank) {
    for (uint32_t h = 0; h < n->glob_h; h++) {
      o_rank *R = &n->rank[h];
      free(R->syn); free(R->grp_count); free(R->grp_offset); free(R->offset_by_delay);
      free(R->src_syn_count); free(R->in_ptr); free(R->in_idx);
      if (R->ring) {
        for (size_t s = 0; s < (size_t)n->glob_h * O_RING; s++) free(R->ring[s].list);
        free(R->ring);
      }
    }
  }
  free(n->rank); free(n->prob); free(n->v); free(n->c); free(n->tr); free(n->te); free(n->nb);
  free(n->inv_nu); free(n->max_ext); free(n->sub); free(n->fired); free(n->last_spike_ms);
  free(n->fwd_hosts); free(n->spk_ids); free(n->spk_t); free(n->rank_spk_start);
  free(n->in_w); free(n->in_frac); free(n->in_cnt); free(n->ev_time); free(n->ev_val);
  free(n);
}

uint64_t dpo_total_synapses(const dpo_net *n) {
  uint64_t s = 0;
  for (uint32_t h = 0; h < n->glob_h; h++) s += n->rank[h].nsyn;
  return s;
}
uint64_t dpo_rank_synapse_count(const dpo_net *n, uint32_t h) { return n->rank[h].nsyn; }
void dpo_rank_synapses(const dpo_net *n, uint32_t h, uint32_t *pre, uint32_t *post,
                       uint8_t *delay, uint8_t *kind, int16_t *weight) {
  const o_rank *R = &n->rank[h];
  for (uint64_t k = 0; k < R->nsyn; k++) {
    if (pre) pre[k] = R->syn[k].pre;
    if (post) post[k] = R->syn[k].post;
    if (delay) delay[k] = R->syn[k].delay;
    if (kind) kind[k] = R->syn[k].kind;
    if (weight) weight[k] = R->syn[k].weight;
  }
}
void dpo_rank_plasticity(const dpo_net *n, uint32_t h, float *tderiv, int32_t *last_act) {
  const o_rank *R = &n->rank[h];
  for (uint64_t k = 0; k < R->nsyn; k++) {
    if (tderiv) tderiv[k] = R->syn[k].tderiv;
    if (last_act) last_act[k] = R->syn[k].last_act;
  }
}
void dpo_bath_params(const dpo_net *n, double *inv_nu_ext, uint32_t *max_ext) {
  for (uint32_t i = 0; i < n->glob_n; i++) {
    if (inv_nu_ext) inv_nu_ext[i] = n->inv_nu[i];
    if (max_ext) max_ext[i] = n->max_ext[i];
  }
}
void dpo_bath_lut(const dpo_net *n, uint32_t s, double *lut) { memcpy(lut, n->lut[s], 256 * sizeof(double)); }

int dpo_write_backward_dump(const dpo_net *n, const char *path) {
  FILE *f = fopen(path, "w");
  if (!f) return -1;
  const o_rank *R = &n->rank[0];
  for (uint64_t k = 0; k < R->nsyn; k++) {
    const o_syn *s = &R->syn[k];
    float w = (float)(s->weight * n->w2f);
    fprintf(f, "%d %d %d %d %d %f ", s->pre, s->post, s->post / n->loc_n, s->delay, s->kind, w);
    fprintf(f, "%f", s->tderiv);
    fprintf(f, "\n");
  }
  fclose(f);
  return 0;
}

/* ---------------------------------------------------------------- dynamics */
static double o_poisson_lapse(o_rng *g, double inv) {
  double temp = (double)1.0 - o_random(g);   /* getUniformLapse (:853-865) */
  if (temp < 0) temp = 0;
  return (-logf(temp) * inv);                   /* :844-851 */
}

/* LIFCADynamic, non-PerseoDyn branch (DPSNN_neuron_sim.c:664-824). */
static void o_lifca(dpo_net *n, uint32_t gn, double t, double I) {
  uint32_t s = n->sub[gn];
  double Tau = n->sp_Tau[s], Theta = n->sp_Theta[s], H = n->sp_H[s], Tarp = n->sp_Tarp[s];
  double AlphaC = n->sp_AlphaC[s], TauC = n->sp_TauC[s], gC = n->sp_gC[s];
  double v = n->v[gn], c = n->c[gn], Tr = n->tr[gn], Te = n->te[gn];
  double deltaT = t - Tr, TFLES = t - Te, rc, TrTe, dth, rmh;
  if (TFLES > Tarp) {
    TrTe = Tr - Te;
    if (TrTe < Tarp) {
      c *= o_exp(-(deltaT - TFLES + Tarp) / TauC);
      deltaT = TFLES - Tarp;
    }
    dth = deltaT / 2;
    rmh = dth / Tau;
    rc = deltaT / TauC;
    v = v - v * rmh - gC * c * dth;
    v = v - v * rmh - gC * c * dth;
    c = c * (1 - rc + rc * rc / 2);
    v += I;
    if (v >= Theta) {
      v = H;
      c += AlphaC;
      Te = t;
      n->fired[gn] = 1;
    }
  } else {
    rc = deltaT / TauC;
    c = c * (1 - rc + rc * rc / 2);
  }
  n->v[gn] = v;
  n->c[gn] = c;
  n->tr[gn] = t;
  n->te[gn] = Te;
}

/* stable insertion of (time,value) pairs: same order as the reference's
 * stable top-down merge sort (DPSNN_neuron_sim.c:391-434) */
static void o_stable_sort(double *tm, double *val, uint32_t k) {
  for (uint32_t i = 1; i < k; i++) {
    double a = tm[i], b = val[i];
    uint32_t j = i;
    while (j > 0 && tm[j - 1] > a) {
      tm[j] = tm[j - 1];
      val[j] = val[j - 1];
      j--;
    }
    tm[j] = a;
    val[j] = b;
  }
}

/* regularDynamicTimeStep, LIFCA (DPSNN_neuron_sim.c:522-662). */
static int o_neuron_step(dpo_net *n, o_rng *g, uint32_t li, uint32_t gn, uint32_t t) {
  double tF = (double)t, nextF = (double)(tF + 1.0);
  uint32_t k = n->in_cnt[li];
  if (k + n->max_ext[gn] > n->ev_cap) {
    set_err("event scratch too small");
    return -1;
  }
  for (uint32_t i = 0; i < k; i++) {
    n->ev_time[i] = tF + n->in_frac[(size_t)li * n->in_cap + i];
    n->ev_val[i] = n->in_w[(size_t)li * n->in_cap + i];
  }
  if (k) o_stable_sort(n->ev_time, n->ev_val, k);
  uint32_t nb_cnt = 0;
  double inv = n->inv_nu[gn];
  if (inv > 0) {
    double *lut = n->lut[n->sub[gn]];
    if (n->nb[gn] < nextF) {
      do {
        n->ev_time[k + nb_cnt] = n->nb[gn];
        n->ev_val[k + nb_cnt] = lut[(uint32_t)(o_random(g) * 256)];
        nb_cnt++;
        n->nb[gn] += o_poisson_lapse(g, inv);
      } while ((n->nb[gn] < nextF) && (nb_cnt < n->max_ext[gn]));
      if (nb_cnt >= n->max_ext[gn])
        if (n->nb[gn] < nextF) {
          do { n->nb[gn] += o_poisson_lapse(g, inv); } while (n->nb[gn] < nextF);
        }
    }
  }
  uint32_t tot = k + nb_cnt;
  if (k && nb_cnt) o_stable_sort(n->ev_time, n->ev_val, tot);  /* synaptic first on ties */
  n->last_bath += nb_cnt;
  for (uint32_t i = 0; i < tot; i++) {
    double ct = n->ev_time[i];
    if (((ct - (double)t) >= 1.0) || ((ct - (double)t) < 0)) {
      set_err("input currentTime in wrong ms on neuron %u", gn);
      return -1;
    }
    o_lifca(n, gn, ct, n->ev_val[i]);
  }
  return 0;
}

/* addInputSpike (DPSNN_neuron_sim.c:289-300). */
static void o_add_input(dpo_net *n, uint32_t li, float w, double t_emit) {
  uint32_t k = n->in_cnt[li];
  if (k < n->in_cap) {
    double ip;
    n->in_w[(size_t)li * n->in_cap + k] = w;
    n->in_frac[(size_t)li * n->in_cap + k] = modf(t_emit, &ip);
  }
  n->in_cnt[li] = k + 1;
}

int64_t dpo_step(dpo_net *n) {
  uint32_t t = n->t;
  int in_window = (t >= n->cfg.start_plasticity_ms) && (t <= n->cfg.stop_plasticity_ms);
  n->last_events = 0;
  n->last_bath = 0;
  /* detect + compress per rank (DPSNN_localNet_sim.c:103-132, :620-664) */
  n->spk_n = 0;
  for (uint32_t h = 0; h < n->glob_h; h++) {
    n->rank_spk_start[h] = n->spk_n;
    o_rank *R = &n->rank[h];
    for (uint32_t i = 0; i < n->loc_n; i++) {
      uint32_t gn = i + h * n->loc_n;
      if (n->fired[gn]) {
        n->fired[gn] = 0;
        n->last_spike_ms[gn] = (int32_t)t;
        if (in_window) {
          for (uint32_t q = R->in_ptr[i]; q < R->in_ptr[i + 1]; q++) {
            o_syn *s = &R->syn[R->in_idx[q]];
            int32_t la = s->last_act;
            float fc;
            if ((int32_t)t <= la) { set_err("causal STDP time order"); return -1; }
            int td = (int)t - 1 - la;
            fc = (la != 0 && td < 128) ? n->causal_tab[td] : 0.0f;
            s->tderiv = s->tderiv + fc;
          }
        }
        n->spk_ids[n->spk_n] = gn;
        n->spk_t[n->spk_n] = n->te[gn];
        n->spk_n++;
      }
    }
  }
  n->rank_spk_start[n->glob_h] = n->spk_n;
  for (uint32_t s = 0; s < n->spk_n; s++) {
    int any = 0;
    for (uint32_t h = 0; h < n->glob_h; h++) any |= n->fwd_hosts[(size_t)n->spk_ids[s] * n->glob_h + h] != 0;
    if (!any) { set_err("spiking neuron %u has no target host", n->spk_ids[s]); return -1; }
  }
  for (uint32_t hp = 0; hp < n->glob_h; hp++) {
    o_rank *R = &n->rank[hp];
    /* exchange + insertAxSpike (DPSNN_spike.c:209-239): slot receives the
     * spikes of source rank h that have a target on hp, ascending index */
    for (uint32_t h = 0; h < n->glob_h; h++) {
      o_slot *sl = &R->ring[(size_t)h * O_RING + R->next_free];
      sl->count = 0;
      for (uint32_t s = n->rank_spk_start[h]; s < n->rank_spk_start[h + 1]; s++)
        if (n->fwd_hosts[(size_t)n->spk_ids[s] * n->glob_h + hp] != 0) {
          sl->list[sl->count].pre = n->spk_ids[s];
          sl->list[sl->count].t = n->spk_t[s];
          sl->count++;
        }
    }
    R->read_index = R->next_free;
    R->next_free = (R->next_free + 1) % O_RING;
    for (uint32_t i = 0; i < n->loc_n; i++) n->in_cnt[i] = 0;
    /* delivery (DPSNN_localNet_sim.c:837-999, DPSNN_synapse.c:179-267) */
    for (int32_t d = (int32_t)n->D - 1; d >= 0; d--) {
      uint32_t idx = (uint32_t)((R->read_index - d + O_RING) % O_RING);
      for (uint32_t h = 0; h < n->glob_h; h++) {
        if (R->grp_count[(size_t)d * n->glob_h + h] == 0) continue;
        const o_slot *sl = &R->ring[(size_t)h * O_RING + idx];
        for (uint32_t q = 0; q < sl->count; q++) {
          uint32_t P = sl->list[q].pre;
          double te = sl->list[q].t;
          uint32_t j = R->offset_by_delay[(size_t)P * n->D + d];
          if (j == 0xFFFFFFFFu) continue;
          /* consecutive entries with pre == P, the scan ending at the list end */
          for (; j < R->nsyn && R->syn[j].pre == P; j++) {
            o_syn *s = &R->syn[j];
            uint32_t li = s->post % n->loc_n;
            float wf = ((float)(s->weight)) * n->w2f;
            o_add_input(n, li, wf, te);
            n->last_events++;
            if (in_window) {
              s->last_act = (int32_t)t;
              int32_t ls = n->last_spike_ms[s->post];
              if ((int32_t)t < ls) { set_err("anti-causal STDP time order"); return -1; }
              int td = (int)t - ls;
              float a = (td < 128) ? n->anti_tab[td] : 0.0f;
              s->tderiv = s->tderiv + a;
            }
          }
        }
      }
    }
    for (uint32_t i = 0; i < n->loc_n; i++)
      if (n->in_cnt[i] > n->in_cap) {
        set_err("more than %u synaptic inputs on neuron %u in one step", n->in_cap, i + hp * n->loc_n);
        return -1;
      }
    /* neuron dynamics in local index order with this rank's stream */
    for (uint32_t i = 0; i < n->loc_n; i++)
      if (o_neuron_step(n, &R->rng, i, i + hp * n->loc_n, t) != 0) return -1;
    /* long term plasticity at x999 ms (DPSNN_localNet_sim.c:312-414) */
    if ((t % 1000) == 999 && in_window) {
      if (n->cfg.stdp_tauDecay_s < 1.0f) { set_err("tauDerivativeDecay_s < 1.0"); return -1; }
      for (uint64_t k = 0; k < R->nsyn; k++) {
        o_syn *s = &R->syn[k];
        uint32_t sp = s->kind, tp = n->sub[s->post];
        float maxv = 2.0 * n->sp_J[sp][tp];
        float rmaxv = 2.0 * n->sp_J[tp][sp];
        float clamp = 0.0f;
        if (maxv > 0.0 && rmaxv > 0.0) {
          float wF = (float)(s->weight * n->w2f);
          float dF = s->tderiv;
          dF += n->cfg.stdp_drift;
          wF = wF + dF;
          if (wF > maxv) { clamp = (wF - maxv); dF = dF - clamp; wF = maxv; }
          if (wF < 0.0) { clamp = wF; dF = dF - clamp; wF = 0.0; }
          s->weight = (int16_t)(wF * n->f2w);
          s->tderiv = dF;
        }
        if (n->cfg.stdp_tauDecay_s == 1.0f)
          s->tderiv = 0.0;
        else
          s->tderiv = (s->tderiv - n->cfg.stdp_drift + clamp) * (1 - 1 / n->cfg.stdp_tauDecay_s);
      }
    }
  }
  n->t = t + 1;
  return n->spk_n;
}

void dpo_last_spikes(const dpo_net *n, uint32_t *ids, double *times) {
  for (uint32_t s = 0; s < n->spk_n; s++) {
    if (ids) ids[s] = n->spk_ids[s];
    if (times) times[s] = n->spk_t[s];
  }
}
uint64_t dpo_last_event_count(const dpo_net *n) { return n->last_events; }
uint64_t dpo_last_bath_count(const dpo_net *n) { return n->last_bath; }
void dpo_state(const dpo_net *n, double *v, double *c, double *tr, double *te, double *nb) {
  size_t N = n->glob_n;
  if (v) memcpy(v, n->v, N * sizeof(double));
  if (c) memcpy(c, n->c, N * sizeof(double));
  if (tr) memcpy(tr, n->tr, N * sizeof(double));
  if (te) memcpy(te, n->te, N * sizeof(double));
  if (nb) memcpy(nb, n->nb, N * sizeof(double));
}
