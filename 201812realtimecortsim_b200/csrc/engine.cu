// engine.cu -- the B200 engine: connectome build, bath producer, delivery,
// LIFCA update, spike compaction and STDP, behind the C ABI of
// include/dpsnn_b200.h.
//
// Arithmetic follows the reference operation by operation (compiled with
// --fmad=false so no multiply-add is contracted, like the reference's
// x86-64 SSE2 build); the comments cite the reference lines each kernel
// restates.  Data layout in HBM (N neurons, S synapses, D delays):
//   neuron state  SoA fp64 v, c, Tr, Te, nextBath (5*8 B/neuron)
//   connectome    CSR sorted by (pre, delay, generation order):
//                 row_ptr[N+1] u64, sub_off[N*(D+1)] u16 (per-delay offsets
//                 inside a row), post[S] u32, w16[S] i16 (6 B/synapse);
//                 with STDP also tderiv[S] f32, last_act[S] i32
//   spike ring    80 slots x N: ids u32, te f64 (one slot per step)
//   events        per target neuron `cap` slots of {u32 key, f32 weight};
//                 overflow list of {target, key, weight}
//   bath          per rank: 64-entry ran3 history, draw ring of LUT index
//                 (u8) and lapse (f32); per step per-neuron event lists
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <string>
#include <mutex>
#include <vector>

#include "dd_math.cuh"
#include "dpsnn_internal.h"

#define RING_SLOTS 80          // DSD__maxD: axonal delay ring length
#define MAX_SYN_PER_NEURON 7500  // DSD__maxM (Makefile miniM)
#define MAX_INPUTS_PER_STEP 6000 // DSD__maxSimultaneousSpikesOnSameTarget
#define MBIG 1000000000
#define MSEED 161803398
#define NEURON_BLOCK 256
#define LOCAL_EVENTS 16        // per-thread event buffer of the neuron kernel
#define NEURON_BATCH 8         // event loads in flight per thread
#define DEFAULT_EVENT_CAP 1024 // per-target event slots per step (capped by memory)

// ------------------------------------------------------------------ errors
static thread_local char g_err[1024];
int dpsnn_fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}
extern "C" const char *dpsnn_last_error(void) { return g_err; }

const char *dpsnn_library_dir(void) {
  // initialised once, thread-safely (engines may be created from several threads)
  static const std::string dir = [] {
    Dl_info info;
    if (dladdr((void *)&dpsnn_library_dir, &info) && info.dli_fname) {
      std::string d = info.dli_fname;
      size_t p = d.rfind('/');
      return (p == std::string::npos) ? std::string(".") : d.substr(0, p);
    }
    return std::string(".");
  }();
  return dir.c_str();
}

#define CK(x)                                                                       \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess)                                                          \
      return dpsnn_fail(DPSNN_E_CUDA, "%s: %s", #x, cudaGetErrorString(e_));        \
  } while (0)

// Error flags raised by kernels (bit set in Dev::flags[0]).
enum {
  F_TIME_WINDOW = 1,     // event time outside [t, t+1)  (DPSNN_neuron_sim.c:681-685)
  F_NO_TARGET = 2,       // spiking neuron without targets (DPSNN_localNet_sim.c:732-737)
  F_OVERFLOW = 4,        // overflow list full
  F_TOO_MANY_INPUTS = 8, // > miniSimSpikes inputs on one neuron in one step
  F_BATH_DRAWS = 16,     // bath draw ring exhausted
  F_GEN = 32,            // synapse generation error (see gen error code)
};

// ------------------------------------------------------------------ model
struct NetConst {
  uint32_t N, locN, P, D, nsub, npcm, cfx, cfy, nmod, mods_per_rank;
  uint32_t stencil, max_mod, stencil_dim, delay_min, delay_max;
  uint32_t offset[DPSNN_MAX_SUBPOP], count[DPSNN_MAX_SUBPOP];
  double Tau[DPSNN_MAX_SUBPOP], Theta[DPSNN_MAX_SUBPOP], H[DPSNN_MAX_SUBPOP];
  double Tarp[DPSNN_MAX_SUBPOP], AlphaC[DPSNN_MAX_SUBPOP], TauC[DPSNN_MAX_SUBPOP];
  double gC[DPSNN_MAX_SUBPOP], NuExt[DPSNN_MAX_SUBPOP];
  double J[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP], DJ[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP];
  double DMin[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP], DMax[DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP];
  float f2w, w2f, min_w;
  uint32_t global_seed, start_pl, stop_pl, stdp_on;
  float causal_tab[128], anti_tab[128];
  float stdp_drift, stdp_tauDecay;
  uint32_t ev_cap, ovf_cap;
  uint32_t light_max;   // neurons with more synaptic events take the heavy path
  uint32_t bath_need;  // largest maxExternCurrentCount
  uint32_t delay_exp;  // getRandomDelay_EXP instead of _UNI
  float inv_log_tn;    // (float)(1.0 / log(0.05)), the EXP tail constant
};

// ------------------------------------------------------------------ ran3
// Numerical Recipes ran3 with the reference's |mj| tweak and seeding rules
// (randdev.c:116-196, :477-502).  Same code on host and device.
struct Ran3 {
  int32_t ma[56];
  int32_t inext, inextp, iff, idum;
};

__host__ __device__ static inline double r3_rand(Ran3 &g) {
  int32_t mj, mk;
  if (g.idum < 0 || g.iff == 0) {
    g.iff = 1;
    mj = MSEED - (g.idum < 0 ? -g.idum : g.idum);
    mj = (mj < 0 ? -mj : mj);
    mj %= MBIG;
    g.ma[55] = mj;
    mk = 1;
    for (int i = 1; i <= 54; i++) {
      int ii = (21 * i) % 55;
      g.ma[ii] = mk;
      mk = mj - mk;
      if (mk < 0) mk += MBIG;
      mj = g.ma[ii];
    }
    for (int k = 1; k <= 4; k++)
      for (int i = 1; i <= 55; i++) {
        g.ma[i] -= g.ma[1 + (i + 30) % 55];
        if (g.ma[i] < 0) g.ma[i] += MBIG;
      }
    g.inext = 0;
    g.inextp = 31;
    g.idum = 1;
  }
  if (++g.inext == 56) g.inext = 1;
  if (++g.inextp == 56) g.inextp = 1;
  mj = g.ma[g.inext] - g.ma[g.inextp];
  if (mj < 0) mj += MBIG;
  g.ma[g.inext] = mj;
  return mj * (1.0 / (double)MBIG);
}
__host__ __device__ static inline void r3_seed(Ran3 &g, int32_t s) {
  g.idum = -s;
  (void)r3_rand(g);
}
// The last 55 outputs (oldest first): the whole state of the lagged
// Fibonacci recurrence x[n] = x[n-55] - x[n-24] (mod 1e9) that ran3 runs.
__host__ __device__ static inline void r3_history(const Ran3 &g, uint32_t *hist55) {
  int k = 0;
  for (int i = g.inext + 1; i <= 55; i++) hist55[k++] = (uint32_t)g.ma[i];
  for (int i = 1; i <= g.inext; i++) hist55[k++] = (uint32_t)g.ma[i];
}

struct NormState {
  int32_t set;
  double cache;
};
// NormDev: polar Box-Muller with a one-value cache (randdev.c:584-606).
__device__ static inline double normdev(Ran3 &g, NormState &ns) {
  if (ns.set == 0) {
    double v1, v2, r, fac;
    do {
      v1 = (double)(2.0 * r3_rand(g) - 1.0);
      v2 = (double)(2.0 * r3_rand(g) - 1.0);
      r = v1 * v1 + v2 * v2;
    } while (r >= 1.0 || r == 0.0);
    fac = (double)sqrt(-2.0 * log_cr(r) / r);
    ns.cache = v1 * fac;
    ns.set = 1;
    return v2 * fac;
  }
  ns.set = 0;
  return ns.cache;
}

// erflib.c:172-181.  The reference converts a possibly negative double to
// uint32_t; its x86-64 build truncates to 64 bits and keeps the low 32 bits
// (so -1.0 gives 0xFFFFFFFF), which the two casts state explicitly (a plain
// device cast would saturate to 0).
__host__ __device__ static inline uint32_t roundr2i(double r) {
  double i = floor(r);
  if (i + 0.5 > r) return (uint32_t)(int64_t)i;
  return (uint32_t)(int64_t)(i + 1.0);
}

__device__ static inline uint32_t subpop_of(const NetConst *net, uint32_t in_cm) {
  for (uint32_t s = 0; s < net->nsub; s++)
    if (in_cm >= net->offset[s] && in_cm < net->offset[s] + net->count[s]) return s;
  return 0xFFFFFFFFu;
}

// ------------------------------------------------------------------ generation
// One thread walks one cortical module's neurons in order, consuming that
// module's serial ran3 stream exactly as simpleCM_invokeIndivSynGenerators
// (DPSNN_LIFCAcorticalModuleGen.cpp:62-220) does.  Modules are independent
// streams (SetRandomSeed(module) at :96-107) except for NormDev's cached
// value, which carries from one module to the next inside a rank; pass A runs
// each module under both hypotheses for that cache (empty, or holding a value
// that the module's first weight accepts) and pass B regenerates the chosen
// one, writing synapses straight into their CSR slots.
struct GenRecord {
  uint32_t nsyn;
  int32_t used_normdev, set_out, err;
  double cache_out;
  float first_mean, first_sigma;
  uint32_t err_arg;
  uint32_t hist[55];
};

enum { GEN_ERR_TOO_MANY = 1, GEN_ERR_WEIGHT_RANGE = 2, GEN_ERR_PROB = 3, GEN_ERR_DELAY = 4,
       GEN_ERR_ZERO_MEAN = 5, GEN_ERR_DELAY_LEVEL = 6, GEN_ERR_DELAY_RANGE = 7 };

__device__ static inline uint32_t empty_random_synapses(Ran3 &g, float pf, uint32_t max_n) {
  // getEmptyRandomSynapses (DPSNN_LIFCAconnectome.cpp:1079-1133)
  double connectivity = (double)pf;
  double r = r3_rand(g);
  double P = connectivity, C = P;
  uint32_t n = 1;
  while ((C < r) && (n <= max_n)) {
    n++;
    P *= 1 - connectivity;
    C += P;
  }
  return n;
}

// Delay generators' error returns (the reference's exit(0) points).
#define DELAY_LEVEL_ERR 0xFFFFFFFFu   // level >= DSD__delayNum
#define DELAY_RANGE_ERR 0xFFFFFFFEu   // delay beyond the pair's DMax

__device__ static inline uint32_t random_delay_uni(const NetConst *net, Ran3 &g, uint32_t s, uint32_t t) {
  // getRandomDelay_UNI (DPSNN_LIFCAcorticalModuleGen.cpp:299-338)
  float outF, DMin, DMax, DelayMin, DelayMax, DelayStep, DelayNum;
  DMin = (float)net->DMin[s * DPSNN_MAX_SUBPOP + t];
  DMax = (float)net->DMax[s * DPSNN_MAX_SUBPOP + t];
  DelayMin = (float)net->delay_min;
  DelayMax = (float)net->delay_max;
  DelayNum = 80;
  DelayStep = (DelayMax - DelayMin) / DelayNum;
  DelayMax -= DelayStep / 2;
  DelayMin += DelayStep / 2;
  DMax = roundr2i((DMax - DelayMin) / DelayStep) * DelayStep + DelayMin;
  DMin = roundr2i((DMin - DelayMin) / DelayStep) * DelayStep + DelayMin;
  outF = (float)((r3_rand(g) * (DMax - DMin) + DMin - DelayMin) / DelayStep);
  (void)DelayMax;
  // the reference stops here: "delay level generated %f > %f max allowed
  // delay levels" (:322-326); the level goes back in the error argument
  if (outF >= DelayNum) return DELAY_LEVEL_ERR;
  const uint32_t outfunc = roundr2i(outF * DelayStep);
  if (outfunc > net->DMax[s * DPSNN_MAX_SUBPOP + t]) return DELAY_RANGE_ERR;   // :330-334
  return outfunc;
}

// getRandomDelay_EXP (DPSNN_LIFCAcorticalModuleGen.cpp:247-297), the
// reference Makefile's default: a truncated exponential over [DMin, DMax);
// DELAY_LEVEL_ERR / DELAY_RANGE_ERR where the reference stops with an error.
__device__ static inline uint32_t random_delay_exp(const NetConst *net, Ran3 &g, uint32_t s, uint32_t t) {
  float outfuncF, DMin, DMax, DelayMin, DelayMax, DelayStep, DelayNum;
  const float InvLogTN = net->inv_log_tn;
  DMin = (float)net->DMin[s * DPSNN_MAX_SUBPOP + t];
  DMax = (float)net->DMax[s * DPSNN_MAX_SUBPOP + t];
  DelayMin = (float)net->delay_min;
  DelayMax = (float)net->delay_max;
  DelayNum = 80;
  DelayStep = (DelayMax - DelayMin) / DelayNum;
  DelayMax -= DelayStep / 2;
  DelayMin += DelayStep / 2;
  DMax = roundr2i((DMax - DelayMin) / DelayStep) * DelayStep + DelayMin;
  DMin = roundr2i((DMin - DelayMin) / DelayStep) * DelayStep + DelayMin;
  outfuncF = (float)((((double)DMin + (double)(DMax - DMin - DelayStep) *
                       log_cr(1.0 - r3_rand(g) * (1.0 - 0.05)) * (double)InvLogTN) -
                      (double)DelayMin) / (double)DelayStep);
  if (outfuncF >= DelayNum) return DELAY_LEVEL_ERR;
  const uint32_t outfunc = roundr2i(outfuncF * DelayStep);
  if (outfunc >= net->DMax[s * DPSNN_MAX_SUBPOP + t]) return DELAY_RANGE_ERR;
  (void)DelayMax;
  return outfunc;
}

#define GEN_THREADS 16          // generation streams per block
#define GEN_TL_SMEM 2048        // targets of a neuron held in shared memory
#define GEN_TL_STRIDE (GEN_TL_SMEM + 1)   // odd stride: threads' lists in different banks
#define GEN_SMEM ((size_t)GEN_THREADS * (sizeof(Ran3) + 4 * GEN_TL_STRIDE + 2 * RING_SLOTS))

// A neuron's target list: the first GEN_TL_SMEM entries in shared memory,
// the rest (rare: in-degrees are ~1100) in the thread's global scratch.
struct GenTargets {
  uint32_t *sh, *gl;
  __device__ uint32_t &operator[](uint32_t j) const { return j < GEN_TL_SMEM ? sh[j] : gl[j]; }
};

__global__ void gen_kernel(const NetConst *__restrict__ net, const float *__restrict__ prob, int pass,
                           GenRecord *rec, const int32_t *__restrict__ chosen_hyp,
                           const double *__restrict__ chosen_cache, uint16_t *cnt_out,
                           const uint64_t *__restrict__ row_ptr, const uint16_t *__restrict__ sub_off,
                           uint32_t *post, int16_t *w16, uint32_t *scratch,
                           const uint32_t *__restrict__ bath_tmpl, double *inv_nu,
                           uint32_t *max_ext, uint8_t *sub) {
  // Each thread's serial stream keeps its ran3 table, the current neuron's
  // target list (its first GEN_TL_SMEM entries; more go to the global
  // scratch) and the per-delay counts in shared memory: the stream is a long
  // chain of dependent table reads.
  extern __shared__ __align__(16) unsigned char gen_smem_raw[];
  Ran3 *s_rng = reinterpret_cast<Ran3 *>(gen_smem_raw);
  uint32_t *s_tl = reinterpret_cast<uint32_t *>(s_rng + blockDim.x);
  uint16_t *s_cnt = reinterpret_cast<uint16_t *>(s_tl + (size_t)blockDim.x * GEN_TL_STRIDE);
  uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nthreads = (pass == 0) ? 2 * net->nmod : net->nmod;
  if (tid >= nthreads) return;
  uint32_t m = (pass == 0) ? (tid >> 1) : tid;
  int hyp = (pass == 0) ? (int)(tid & 1) : chosen_hyp[m];
  GenRecord *R = &rec[(pass == 0) ? tid : m];
  const uint32_t N = net->N, D = net->D, npcm = net->npcm, stencil = net->stencil;
  GenTargets tl{s_tl + (size_t)threadIdx.x * GEN_TL_STRIDE, scratch + (size_t)tid * MAX_SYN_PER_NEURON};
  uint16_t *cnt = s_cnt + (size_t)threadIdx.x * RING_SLOTS;

  Ran3 &g = s_rng[threadIdx.x];
  g.iff = 0;
  g.idum = 0;
  g.inext = g.inextp = 0;
  if (m % net->mods_per_rank == 0) r3_seed(g, (int32_t)net->global_seed);  // localNet_init.c:119
  r3_seed(g, (int32_t)m);  // module start (ModuleGen.cpp:96-107); m==0 does not re-initialise
  NormState ns;
  ns.set = hyp;
  ns.cache = (pass == 1 && hyp == 1) ? chosen_cache[m] : 0.0;
  int used = 0;
  uint32_t nsyn = 0;
  R->err = 0;
  for (uint32_t gi = m * npcm; gi < (m + 1) * npcm; gi++) {
    uint32_t mod = gi / npcm;
    uint32_t cfy = mod / net->cfx, cfx = mod % net->cfx;
    uint32_t ssub = subpop_of(net, gi % npcm);
    if (pass == 1) sub[gi] = (uint8_t)ssub;
    uint32_t tot = 0;
    for (uint32_t ts = 0; ts < net->nsub; ts++)
      for (uint32_t x = 0; x < stencil; x++)
        for (uint32_t y = 0; y < stencil; y++) {
          int32_t nx = (int32_t)cfx + (int32_t)x - (int32_t)net->max_mod;
          int32_t ny = (int32_t)cfy + (int32_t)y - (int32_t)net->max_mod;
          if (nx < 0 || nx >= (int32_t)net->cfx || ny < 0 || ny >= (int32_t)net->cfy) continue;
          float pf = prob[(((size_t)ssub * DPSNN_MAX_SUBPOP + ts) * stencil + x) * stencil + y];
          if (!(pf > 0)) continue;
          if (!(pf > 0.00001f)) { R->err = GEN_ERR_PROB; R->err_arg = gi; return; }
          uint32_t in_cm = net->offset[ts] - 1;
          uint32_t last = net->offset[ts] + net->count[ts];
          uint32_t avail = last - in_cm;
          while ((in_cm += empty_random_synapses(g, pf, avail)) < last) {
            if (tot >= MAX_SYN_PER_NEURON) { R->err = GEN_ERR_TOO_MANY; R->err_arg = gi; return; }
            tl[tot++] = in_cm + (uint32_t)nx * npcm + (uint32_t)ny * npcm * net->cfx;
          }
        }
    if (tot >= MAX_SYN_PER_NEURON) { R->err = GEN_ERR_TOO_MANY; R->err_arg = gi; return; }
    for (uint32_t d = 0; d < D; d++) cnt[d] = 0;
    for (uint32_t j = 0; j < tot; j++) {
      uint32_t tg = tl[j];
      uint32_t tsub = subpop_of(net, tg % npcm);
      uint32_t delay = net->delay_exp ? random_delay_exp(net, g, ssub, tsub) : random_delay_uni(net, g, ssub, tsub);
      if (delay == DELAY_LEVEL_ERR) { R->err = GEN_ERR_DELAY_LEVEL; R->err_arg = gi; return; }
      if (delay == DELAY_RANGE_ERR) { R->err = GEN_ERR_DELAY_RANGE; R->err_arg = gi; return; }
      if (delay >= D) { R->err = GEN_ERR_DELAY; R->err_arg = delay; return; }
      float mean = (float)net->J[ssub * DPSNN_MAX_SUBPOP + tsub];
      float sigma = (float)(net->DJ[ssub * DPSNN_MAX_SUBPOP + tsub] * (double)mean);
      if (!used) {
        used = 1;
        R->first_mean = mean;
        R->first_sigma = sigma;
      }
      float wf;
      if (mean > 0.0) {
        do { wf = (float)(mean + normdev(g, ns) * sigma); } while ((wf < 0.0) || (wf >= 2.0 * mean));
      } else {
        if (mean == 0.0f) { R->err = GEN_ERR_ZERO_MEAN; R->err_arg = gi; return; }
        do { wf = (float)(mean + normdev(g, ns) * sigma); } while ((wf <= 2.0 * mean) || (wf > 0));
      }
      if ((wf < net->min_w) || (wf > (-net->min_w))) { R->err = GEN_ERR_WEIGHT_RANGE; R->err_arg = gi; return; }
      int16_t w = (int16_t)(wf * net->f2w);
      if (pass == 0) {
        cnt[delay]++;
      } else {
        uint64_t pos = row_ptr[gi] + sub_off[(size_t)gi * (D + 1) + delay] + cnt[delay]++;
        post[pos] = tg;
        w16[pos] = w;
      }
      nsyn++;
    }
    if (pass == 0) {
      uint16_t *co = cnt_out + ((size_t)hyp * N + gi) * D;
      for (uint32_t d = 0; d < D; d++) co[d] = cnt[d];
    } else {
      // external bath rate (ModuleGen.cpp:201-211, LIFCAconnectome.cpp:871-887)
      float nu = (float)net->NuExt[ssub];
      uint32_t bx = cfx, by = cfy;
      if (bx >= net->cfx / 2) bx = 0u - (bx - net->cfx + 1u);   // unsigned, as the reference computes it
      if (by >= net->cfy / 2) by = 0u - (by - net->cfy + 1u);
      if (bx >= net->stencil_dim) bx = net->stencil_dim - 1;
      if (by >= net->stencil_dim) by = net->stencil_dim - 1;
      float cext = (float)bath_tmpl[bx * net->stencil_dim + by];
      if (cext != 0) {
        double inv = 1000.0 / (nu * cext);
        inv_nu[gi] = inv;
        max_ext[gi] = (uint32_t)ceil(20 / inv);
      } else {
        inv_nu[gi] = 0;
        max_ext[gi] = 0;
      }
    }
  }
  R->nsyn = nsyn;
  R->used_normdev = used;
  R->set_out = ns.set;
  R->cache_out = ns.cache;
  r3_history(g, R->hist);
}

// ------------------------------------------------------------------ step kernels
struct Dev {
  NetConst *net;
  double *lut;              // [nsub*256]
  // neurons
  double *v, *c, *tr, *te, *nb, *inv_nu;
  const double *nb_prev;    // nextBath before this step's bath (bath_kernel input)
  uint32_t *max_ext;
  uint8_t *sub, *fired;
  int32_t *last_spike_ms;
  uint32_t *block_fired;    // per NEURON_BLOCK block
  // connectome
  uint64_t *row_ptr;
  uint16_t *sub_off;
  uint32_t *post;
  int16_t *w16;
  float *tderiv;
  int32_t *last_act;
  // LTP probe (null unless enabled): weight and trace before the update,
  // and the trace after it before its decay
  int16_t *probe_w;
  float *probe_td, *probe_td_mid;
  // STDP event log of one step (null unless enabled): {synapse index lo/hi,
  // post | anti-causal << 31, contribution bits} of rank 0's synapses from
  // rank-0 neurons with a non-zero contribution
  uint4 *stdp_log;
  uint32_t *stdp_log_cnt;
  uint64_t *in_ptr;
  uint32_t *in_idx;
  // ring
  uint32_t *ring_ids, *ring_cnt;
  double *ring_te;
  // events
  uint32_t *ev_cnt;
  uint2 *ev;
  uint32_t *ovf_cnt;
  uint4 *ovf;
  double *huge_tau;                   // huge_kernel's scratch: HEAVY_MAX events per block
  uint32_t *huge_key;
  float *huge_val;
  uint32_t *heavy_list, *heavy_cnt;   // [4N]: neuron, event count of the warp path, then of
                                      // the block path; heavy_cnt[0..1]: their lengths
  // bath
  uint32_t *bath_hist;      // [P][64] ran3 history ring
  uint64_t *bath_produced, *bath_pos;  // [P]
  uint8_t *draw_idx;        // [P][BATH_RING] converted draws kept between steps
  float *draw_lapse;        // [P][BATH_RING]
  uint64_t *bath_rank_base; // [P+1]
  uint32_t *bath_off;       // [N]
  uint16_t *bath_cnt;       // [N]
  double *bath_time;
  uint8_t *bath_lut;
  logf_fixup_t fix;
  const uint32_t *fix_bitmap; // one bit per float in [0x30000000, 0x3F800000]: key has a fix-up
  const float *fix_near;      // [256] by the result's exponent: a fix-up input's exact log lies at most
                              // this many ulps from a rounding midpoint (-1: none in that binade)
  // control
  uint32_t *t;              // current step
  uint32_t *bath_t;         // step of the next bath launch (the bath runs one step ahead)
  uint32_t *flags;
  unsigned long long *events;  // synaptic events delivered
};

// Step 1: ordered spike compaction (compressNeuralSpikesInThisTimeStep,
// DPSNN_localNet_sim.c:103-132, :620-664): the neurons that fired during the
// previous step, ascending index, with their emission time Te, into ring slot
// t mod 80.  Also sets lastNeuralEmittedSpikeTime_ms = t.
__global__ void compact_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t N = net->N, t = *d.t, slot = t % RING_SLOTS;
  const uint32_t b = blockIdx.x, nb = gridDim.x;
  __shared__ uint32_t s_red[NEURON_BLOCK / 32];
  __shared__ uint32_t s_prefix;
  uint32_t part = 0;
  for (uint32_t k = threadIdx.x; k < b; k += blockDim.x) part += d.block_fired[k];
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int w = 0; w < NEURON_BLOCK / 32; w++) s += s_red[w];
    s_prefix = s;
  }
  __syncthreads();
  uint32_t i = b * NEURON_BLOCK + threadIdx.x;
  uint32_t f = (i < N) ? d.fired[i] : 0;
  uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t bal = __ballot_sync(0xffffffffu, f);
  __shared__ uint32_t s_wcnt[NEURON_BLOCK / 32];
  if (lane == 0) s_wcnt[warp] = __popc(bal);
  __syncthreads();
  uint32_t woff = 0;
  for (uint32_t w = 0; w < warp; w++) woff += s_wcnt[w];
  if (f) {
    uint32_t q = s_prefix + woff + __popc(bal & ((1u << lane) - 1));
    d.fired[i] = 0;
    d.ring_ids[(size_t)slot * N + q] = i;
    d.ring_te[(size_t)slot * N + q] = d.te[i];
    d.last_spike_ms[i] = (int32_t)t;
    if (d.row_ptr[i + 1] == d.row_ptr[i]) atomicOr(d.flags, F_NO_TARGET);
  }
  if (b == nb - 1 && threadIdx.x == 0) {
    uint32_t tot = s_prefix;
    for (int w = 0; w < NEURON_BLOCK / 32; w++) tot += s_wcnt[w];
    d.ring_cnt[slot] = tot;
  }
}

#define STDP_LOG_CAP DPSNN_STDP_LOG_CAP   // STDP event records per step

// One record of the STDP event log (the statSTDPevent.write calls of
// DPSNN_neuron_sim.c:152-166 and :230-246, which report rank 0's synapses
// whose both ends are rank-0 neurons); the host restores the reference's order.
__device__ static inline void stdp_log_append(const Dev &d, uint64_t k, uint32_t post, uint32_t anti, float c) {
  const uint32_t o = atomicAdd(d.stdp_log_cnt, 1u);
  if (o < STDP_LOG_CAP)
    d.stdp_log[o] = make_uint4((uint32_t)k, (uint32_t)(k >> 32), post | (anti << 31), __float_as_uint(c));
  else
    atomicOr(d.flags, F_OVERFLOW);
}

// The anti-causal records of the STDP event log, after delivery: a synapse
// delivered at step t carries last_act == t (one delivery per synapse and
// step, none at step 0), and its contribution is the one delivery added.
__global__ void stdp_anti_log_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t;
  if (t == 0 || !(t >= net->start_pl && t <= net->stop_pl)) return;
  const uint64_t end = d.row_ptr[net->locN];
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < end; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = d.post[k];
    if (j >= net->locN || d.last_act[k] != (int32_t)t) continue;
    const int td = (int)t - d.last_spike_ms[j];
    const float a = (td < 128) ? net->anti_tab[td] : 0.0f;
    if (a != 0.0f) stdp_log_append(d, k, j, 1u, a);
  }
}

// Causal STDP at detection (causalSTDP_ms_ofBackwardSynapses,
// DPSNN_neuron_sim.c:94-177): one warp per spiking neuron walks its incoming
// synapses.
__global__ void causal_stdp_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t;
  if (!(t >= net->start_pl && t <= net->stop_pl)) return;
  const uint32_t slot = t % RING_SLOTS, cnt = d.ring_cnt[slot], N = net->N;
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < cnt;
       w += (gridDim.x * blockDim.x) >> 5) {
    uint32_t i = d.ring_ids[(size_t)slot * N + w];
    for (uint64_t k = d.in_ptr[i] + lane; k < d.in_ptr[i + 1]; k += 32) {
      uint32_t s = d.in_idx[k];
      int32_t la = d.last_act[s];
      int td = (int)t - 1 - la;
      float fc = (la != 0 && td < 128) ? net->causal_tab[td] : 0.0f;
      // the reference adds the term even when it is zero
      // (DPSNN_neuron_sim.c:171); a time derivative is never -0.0 (it starts
      // at +0.0 and no step of the plasticity makes a -0.0 from other
      // values), so skipping the zero terms changes no bit
      if (fc != 0.0f) d.tderiv[s] = d.tderiv[s] + fc;
      if (d.stdp_log && fc != 0.0f && t != 0 && i < net->locN && s < d.row_ptr[net->locN])
        stdp_log_append(d, s, i, 0u, fc);
    }
  }
}

// Step 2: delivery (axonalSpikeSchedulersToSynapticSpikeSchedulers,
// DPSNN_localNet_sim.c:837-999, and findAndGetNextSyn, DPSNN_synapse.c:179-267).
// Work item = (delay d, spike q of the slot written d steps ago), i.e. the CSR
// segment (pre, d).  A warp takes 32 work items at a time: each lane fetches
// one item's segment bounds, then the warp walks the concatenation of the 32
// segments with every lane on a different synapse, appending {key, weight}
// to each target's event list: per lane a batch of DELIVER_UNROLL synapses
// takes its slots (atomics) while the next batch's synapse loads are in
// flight.
// key = (D-1-d) << 25 | q orders a target's events as the reference delivers
// them (delay descending, then source ascending), which breaks ties between
// equal arrival times.
#define DELIVER_THREADS 256
#define DELIVER_UNROLL 2

// Stores one event in slot s of target j's list (taken by the caller's
// atomicAdd on ev_cnt[j]), or in the overflow list past the bucket.
__device__ static inline void deliver_event(const Dev &d, const NetConst *net, uint64_t k, uint32_t key,
                                            uint32_t t, bool stdp, uint32_t cap, uint32_t j, float wf,
                                            uint32_t s) {
  if (s < cap) {
    d.ev[(size_t)j * cap + s] = make_uint2(key, __float_as_uint(wf));
  } else {
    const uint32_t o = atomicAdd(d.ovf_cnt, 1u);
    if (o < net->ovf_cap)
      d.ovf[o] = make_uint4(j, key, __float_as_uint(wf), 0u);
    else
      atomicOr(d.flags, F_OVERFLOW);
  }
  if (stdp) {  // synapseSetLastActiveTime_antiCausalSTDP (DPSNN_neuron_sim.c:179-277)
    d.last_act[k] = (int32_t)t;
    const int td = (int)t - d.last_spike_ms[j];
    const float a = (td < 128) ? net->anti_tab[td] : 0.0f;
    if (a != 0.0f) d.tderiv[k] = d.tderiv[k] + a;   // zero terms change no bit (causal_stdp_kernel)
  }
}

__global__ void __launch_bounds__(DELIVER_THREADS) deliver_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t, N = net->N, D = net->D, cap = net->ev_cap;
  __shared__ uint32_t s_pre[RING_SLOTS + 1];
  __shared__ uint32_t s_off[DELIVER_THREADS / 32][33];     // per warp: exclusive prefix of lengths
  __shared__ unsigned long long s_beg[DELIVER_THREADS / 32][32];
  __shared__ uint32_t s_key[DELIVER_THREADS / 32][32];
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t dd = 0; dd < D; dd++) {
      s_pre[dd] = acc;
      acc += d.ring_cnt[(t + RING_SLOTS - dd) % RING_SLOTS];
    }
    s_pre[D] = acc;
  }
  __syncthreads();
  const uint32_t total = s_pre[D];
  const uint32_t lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  const bool stdp = net->stdp_on && t >= net->start_pl && t <= net->stop_pl;
  const float w2f = net->w2f;
  uint32_t *off = s_off[wb];
  unsigned long long *bg = s_beg[wb];
  uint32_t *ky = s_key[wb];
  unsigned long long my_events = 0;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t w0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; w0 < total; w0 += nwarps * 32u) {
    const uint32_t w = w0 + lane;
    uint64_t beg = 0;
    uint32_t len = 0, key = 0;
    // the delay level of item w: the first dl with s_pre[dl + 1] > w.  The
    // warp finds w0's by a binary search over the D levels (some of them
    // empty), the same for every lane; each lane steps on from there (its 32
    // items span few levels)
    uint32_t dl = 0, hi = D - 1;
    while (dl < hi) {
      const uint32_t mid = (dl + hi) >> 1;
      if (s_pre[mid + 1] <= w0) dl = mid + 1; else hi = mid;
    }
    if (w < total) {
      while (s_pre[dl + 1] <= w) dl++;
      const uint32_t q = w - s_pre[dl];
      const uint32_t slot = (t + RING_SLOTS - dl) % RING_SLOTS;
      const uint32_t P = d.ring_ids[(size_t)slot * N + q];
      const uint16_t *so = d.sub_off + (size_t)P * (D + 1);
      const uint32_t a = so[dl], b = so[dl + 1];
      beg = d.row_ptr[P] + a;
      len = b - a;
      key = ((D - 1 - dl) << 25) | q;
    }
    uint32_t incl = len;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    off[lane] = incl - len;
    if (lane == 31) off[32] = tot;
    bg[lane] = beg;
    ky[lane] = key;
    my_events += len;
    __syncwarp();
    // the concatenated segments, element e = lane + 32 * i, in batches of
    // DELIVER_UNROLL per lane: the next batch's synapse loads are issued
    // while this batch's slot atomics are in flight
    uint32_t sg = 0;
    uint64_t k[DELIVER_UNROLL];
    uint32_t kk[DELIVER_UNROLL], jj[DELIVER_UNROLL];
    float wf[DELIVER_UNROLL];
#define DELIVER_FETCH(E0, K, KK, JJ, WF)                       \
  _Pragma("unroll") for (int u = 0; u < DELIVER_UNROLL; u++) { \
    const uint32_t e = (E0) + 32u * u + lane;                 \
    KK[u] = 0xFFFFFFFFu;                                      \
    if (e < tot) {                                            \
      while (off[sg + 1] <= e) sg++;                          \
      K[u] = bg[sg] + (e - off[sg]);                          \
      KK[u] = ky[sg];                                         \
      JJ[u] = __ldg(&d.post[K[u]]);                           \
      WF[u] = ((float)__ldg(&d.w16[K[u]])) * w2f;             \
    }                                                         \
  }
    DELIVER_FETCH(0u, k, kk, jj, wf);
    for (uint32_t e0 = 0; e0 < tot; e0 += 32u * DELIVER_UNROLL) {
      uint32_t sl[DELIVER_UNROLL];
#pragma unroll
      for (int u = 0; u < DELIVER_UNROLL; u++)
        if (kk[u] != 0xFFFFFFFFu) sl[u] = atomicAdd(&d.ev_cnt[jj[u]], 1u);
      uint64_t nk[DELIVER_UNROLL];
      uint32_t nkk[DELIVER_UNROLL], njj[DELIVER_UNROLL];
      float nwf[DELIVER_UNROLL];
      DELIVER_FETCH(e0 + 32u * DELIVER_UNROLL, nk, nkk, njj, nwf);
#pragma unroll
      for (int u = 0; u < DELIVER_UNROLL; u++)
        if (kk[u] != 0xFFFFFFFFu) deliver_event(d, net, k[u], kk[u], t, stdp, cap, jj[u], wf[u], sl[u]);
#pragma unroll
      for (int u = 0; u < DELIVER_UNROLL; u++) {
        k[u] = nk[u];
        kk[u] = nkk[u];
        jj[u] = njj[u];
        wf[u] = nwf[u];
      }
    }
#undef DELIVER_FETCH
    __syncwarp();
  }
  for (int o = 16; o > 0; o >>= 1) my_events += __shfl_down_sync(0xffffffffu, my_events, o);
  if (lane == 0 && my_events) atomicAdd(d.events, my_events);
}

// Step 3: the Poisson bath (regularDynamicTimeStep, DPSNN_neuron_sim.c:604-640,
// getPoissonLapse :844-865).  Each rank owns one serial ran3 stream that its
// neurons consume in index order: a neuron whose next bath time is before
// t+1 takes one pair of draws (LUT index, lapse) per event.  One block per
// rank runs a shared-memory pipeline:
//   warp 1     extends the lagged Fibonacci sequence 24 values per round
//              (x[n] = x[n-55] - x[n-24] mod 1e9) into a ring of raw draws;
//   warps 2, 3 convert groups of four rounds into the LUT index (uint32)(u*256)
//              and the lapse factor -logf((float)(1-u)), and extend q[], the
//              running sum over draws of one parity of the lapses in 2^-20
//              units (q[n] = q[n-2] + round(lap[n] * 2^20), integers mod 2^32);
//   warps 5-7, 9-15 (builders) tabulate the event counts of the chunk of 32
//              neurons two chunks ahead of the walk.  The number of events c
//              of a neuron is the first c at which nextBath + sum of c lapses
//              * invNuExt reaches t+1; it depends on where in the stream the
//              neuron starts, which is known only once every earlier neuron
//              of the rank is decided.  Each neuron's budget (t+1 -
//              nextBath)/invNuExt becomes two integer bounds that enclose
//              every rounding of the reference's sequential sum; its start is
//              predicted from the latest known chunk start and the expected
//              counts (1 + budget each); for the BATH_NC candidate starts
//              around the prediction (a warp per neuron, two candidates per
//              lane) a binary search of q[] finds c (c - 1 sums below the
//              lower bound, the c-th at or above the upper one); a candidate
//              the bounds do not decide is marked undecided.  A builder
//              takes whole quads of neurons (the rank's quads in turn) and
//              composes their tables itself: for every candidate start of
//              neuron 2p the events of neurons 2p and 2p+1 together, then of
//              4k .. 4k+3 together;
//   warp 0     (walk) follows the chain: one lookup per four neurons, at the
//              quad's actual start, gives the next quad's start.  A quad the
//              tables do not decide goes neuron by neuron, and an undecided
//              neuron (or one at the maxExternCurrentCount cap) runs the
//              reference's sequential loop.  The lanes then recover every
//              neuron's start and count from the pair and single tables in
//              parallel and hand the chunk to
//   warp 4     (emitter), whose lanes write the chunk's events, each
//              replaying its neuron in the reference's exact arithmetic;
//   warp 8     stays idle: warps go to the SM's four schedulers by index, so
//              the walk shares its scheduler with the emitter only.
// Rounds are published in order with a flag; every wait is bounded and
// raises F_BATH_DRAWS when its limit is reached.
#define BATH_THREADS 512       // 16 warps: roles in bath_kernel
#define BATH_RING 8192         // draws resident in shared memory
#define BATH_ROUNDS 512        // round flags tracked (BATH_ROUNDS*24 > BATH_RING)
#define BATH_MAX_EXT 2048      // largest maxExternCurrentCount supported
#define BATH_SPIN_LIMIT (1u << 26)
#define BATH_FAST_LANES 32     // events decided by one count table entry
#define BATH_WINDOW (2 * BATH_FAST_LANES + 2)   // draws a count decision reads past its start
#define BATH_NC 64             // candidate start positions tabulated per neuron
#define BATH_BUILDERS 10       // table-building warps: 5, 6, 7, 9 .. 15
#define BATH_AHEAD 2           // chunks the count tables are built ahead of the consumer (the code below
                               // predicts from chunk c-2's start)
#define BATH_TABS (BATH_AHEAD + 1)
#define BATH_CG 4              // generator rounds a converter takes at once: 96 draws, 3 per lane
#define BATH_TROW (BATH_NC + 4)  // bytes per neuron in a count table: BATH_NC candidates, then the sentinel

static_assert(BATH_NC == 64, "a builder lane takes two candidate starts");
static_assert(24 * BATH_CG == 96 && BATH_ROUNDS % BATH_CG == 0, "a converter group is 3 draws per lane");

// q[] keeps the two parities apart: draws n, n+2, n+4, .. sit in consecutive
// words, so the 32 lanes of a builder, each on its own candidate start two
// draws from the next, read 32 different banks.
__device__ __forceinline__ uint32_t bath_qi(unsigned long long n) {
  return (((uint32_t)n & 1u) * (BATH_RING / 2)) | (((uint32_t)n & (BATH_RING - 1)) >> 1);
}

struct BathSmem {
  uint32_t lap[BATH_RING];          // raw draw until converted, then the lapse (float bits)
  uint32_t q[BATH_RING];            // per-parity prefix of the lapses, 2^-20 units, at bath_qi(n)
  uint8_t idx[BATH_RING];
  // count tables of chunk c in buffer c % BATH_TABS.  Neuron j: its events
  // when it starts at bp_base[j] + 2o, 0xFF = undecided; entries BATH_NC..
  // answer a start outside the window (0xFF; 0 for a neuron with no event
  // this step, whose every entry is 0).  Pair p, quad k: the events of
  // neurons 2p, 2p+1 (4k .. 4k+3) when 2p (4k) starts at bp_base[2p] + 2o.
  uint8_t tab[BATH_TABS][32][BATH_TROW];
  uint8_t tab2[BATH_TABS][16][BATH_TROW];
  uint8_t tab4[BATH_TABS][8][BATH_TROW];
  uint32_t bp_base[BATH_TABS][32];  // position (low 32 bits) of candidate 0 of neuron j
  uint32_t tab_cnt[BATH_TABS];      // quads whose tables of this buffer are complete
  uint32_t c_start[32], c_cnt[32];  // the walk's record: quad starts, and neurons walked one by one
  uint32_t e_start[2][32], e_cnt[2][32];  // chunk c, handed to the emitter in buffer c & 1
  unsigned long long e_end[2];      // its end position
  uint32_t e_out[2];                // its first event slot
  uint32_t e_seq, emit_done;        // chunks handed over, chunks emitted
  unsigned long long emit_pos;      // ring slots before this position may be reused
  unsigned long long chunk_start[BATH_TABS];  // exact start of chunk c (walk, as it begins chunk c)
  uint32_t chunk_seq;               // chunks whose start is published
  uint32_t flag[BATH_ROUNDS];       // round r converted <=> flag[r % BATH_ROUNDS] == r + 1
  float near[256];                  // the logf fix-up filter's distances (Dev::fix_near)
  uint32_t hist[64];
  unsigned long long pos;           // walk position (draws)
  unsigned long long raw_end;       // draws generated
  unsigned long long conv_base;     // first draw of round 0 of this launch
  uint32_t next_round;              // next group of BATH_CG rounds a converter claims
  uint32_t published;               // rounds 0 .. published-1 are converted (raised after their flags)
  uint32_t done, err;
};

// The table entry for a start dl draws after candidate 0: dl / 2 for an
// even dl inside the window, else BATH_NC (an odd dl rotates into the top
// bit).
__device__ __forceinline__ uint32_t bath_row(uint32_t dl) {
  return min(__funnelshift_r(dl, dl, 1), (uint32_t)BATH_NC);
}

// The fix-up value of input key (when it has one), else f: a binary search of
// the keys of its block of 4096 floats.
__device__ static inline float logf_fixup_search(const logf_fixup_t &fx, uint32_t key, float f) {
  const uint32_t bk = (key >> 12) - LOGF_FIX_BASE;
  uint32_t lo = __ldg(&fx.bucket[bk]), hi = __ldg(&fx.bucket[bk + 1]);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(&fx.keys[mid]) < key) lo = mid + 1; else hi = mid;
  }
  return (lo < fx.n && __ldg(&fx.keys[lo]) == key) ? __ldg(&fx.vals[lo]) : f;
}

// logf of the host C library on (0,1].  The inputs where it differs from
// the correctly rounded float all have an exact logarithm close to a
// rounding midpoint; an input whose logarithm lies farther from one than any
// fix-up input of the same result binade returns the correctly rounded value
// at once.  Otherwise a one-bit-per-float filter, then a binary search of
// the fix-up keys of its block of 4096 floats.
__device__ static inline float logf_ref_dev(const logf_fixup_t &fx, const uint32_t *__restrict__ bitmap,
                                            const float *__restrict__ near, float x) {
  const double y = log((double)x);
  const float f = logf_cr_from(x, y);
  union { float f; uint32_t u; } b;
  b.f = x;
  const uint32_t key = b.u;
  if (key < 0x30000000u || key > 0x3F800000u) return f;
  const uint32_t fb = __float_as_uint(f), E = (fb >> 23) & 0xFFu;
  if ((fb & 0x7FFFFFu) != 0 && E > 24) {   // not a power of two: one ulp on either side
    const double inv_ulp = __longlong_as_double((long long)(150 - E + 1023) << 52);   // 2^(150-E)
    const double dist = 0.5 - fabs(y - (double)f) * inv_ulp;
    if (dist > (double)__ldg(&near[E])) return f;
  }
  const uint32_t bit = key - 0x30000000u;
  if (!((__ldg(&bitmap[bit >> 5]) >> (bit & 31)) & 1u)) return f;
  return logf_fixup_search(fx, key, f);
}

// Converts raw draw mj into (LUT index, lapse) (getPoissonLapse, :844-865,
// and the LUT index draw at :617-619).
__device__ static inline float bath_lapse(const Dev &d, uint32_t mj, uint8_t &idx) {
  const double u = mj * (1.0 / (double)MBIG);
  idx = (uint8_t)(uint32_t)(u * 256);
  double temp = (double)1.0 - u;
  if (temp < 0) temp = 0;
  return -logf_ref_dev(d.fix, d.fix_bitmap, d.fix_near, (float)temp);
}

// bath_lapse for three draws at once, each step for all three before the
// next: their filter-table loads are in flight together.  near is the
// per-binade distance table (logf_ref_dev), here from shared memory.
__device__ static inline void bath_lapse3(const Dev &d, const float *near, const uint32_t (&mj)[3], float (&lap)[3],
                                          uint8_t (&idx)[3]) {
  float f[3];
  uint32_t key[3], bw[3];
  bool chk[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const double u = mj[i] * (1.0 / (double)MBIG);
    idx[i] = (uint8_t)(uint32_t)(u * 256);
    double temp = (double)1.0 - u;
    if (temp < 0) temp = 0;
    const float x = (float)temp;
    const double y = log((double)x);
    f[i] = logf_cr_from(x, y);
    key[i] = __float_as_uint(x);
    chk[i] = key[i] >= 0x30000000u && key[i] <= 0x3F800000u;
    const uint32_t fb = __float_as_uint(f[i]), E = (fb >> 23) & 0xFFu;
    if (chk[i] && (fb & 0x7FFFFFu) != 0 && E > 24) {
      const double inv_ulp = __longlong_as_double((long long)(150 - E + 1023) << 52);   // 2^(150-E)
      chk[i] = 0.5 - fabs(y - (double)f[i]) * inv_ulp <= (double)near[E];
    }
  }
#pragma unroll
  for (int i = 0; i < 3; i++) bw[i] = chk[i] ? __ldg(&d.fix_bitmap[(key[i] - 0x30000000u) >> 5]) : 0u;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if ((bw[i] >> ((key[i] - 0x30000000u) & 31)) & 1u) f[i] = logf_fixup_search(d.fix, key[i], f[i]);
    lap[i] = -f[i];
  }
}

__device__ static inline uint32_t lap_fixed(float lap) {
  return __double2uint_rn((double)lap * 0x1p20);   // lap < 2^11: no overflow
}

// Integer bounds on the lapse sum, in 2^-20 units, for one neuron: a
// fixed-point sum F of c lapses below lo means the reference's sequential
// nextBath after c events is certainly < t+1, at or above hi1 certainly
// >= t+1.  E1 bounds the rounding of that sequential sum (c <= 32
// additions, |values| < |T1| + 42 invNuExt, and t+1 - nextBath); 2^-16
// bounds the rounding of F (32 terms of at most 2^-21); the 2^-30 relative
// margin covers the bound's own arithmetic.  Both are clamped to 32 bits
// (F < 2^30).  misc: 0 = no bath event this step; else 0x100 |
// min(32, maxExternCurrentCount).
__device__ static inline void bath_bounds(double T1, double nb, double inv, uint32_t mx, uint32_t &lo,
                                          uint32_t &hi1, uint32_t &misc) {
  lo = hi1 = misc = 0;
  if (inv > 0 && nb < T1) {
    const double E1 = 0x1p-44 * (fabs(T1) + fabs(nb) + 1.0 + 32.0 * inv);
    double blo = ((T1 - nb) - E1) / inv - 0x1p-16;
    double bhi = ((T1 - nb) + E1) / inv + 0x1p-16;
    const double mg = 0x1p-30 * (fabs(bhi) + 1.0);
    blo = fmin(fmax(floor((blo - mg) * 0x1p20), 0.0), 4294967295.0);
    bhi = fmin(fmax(ceil((bhi + mg) * 0x1p20) + 1.0, 0.0), 4294967295.0);
    lo = (uint32_t)blo;
    hi1 = (uint32_t)bhi;
    misc = 0x100u | min(32u, mx);
  }
}

// The reference's loop for one neuron from stream position pos
// (regularDynamicTimeStep, DPSNN_neuron_sim.c:604-640): the events go to c,
// the position after the neuron's draws is returned.  Waits (bounded) until
// the draws it reads are converted; sets fail when a wait gives up.
__device__ static inline unsigned long long bath_exact(BathSmem &s, double nbv, double inv, uint32_t mx, double T1,
                                                       unsigned long long pos, unsigned long long &lim, uint32_t &rr,
                                                       uint32_t &spins, bool &fail, uint32_t &c) {
  volatile BathSmem &vs = s;
  const uint32_t M = BATH_RING - 1;
  c = 0;
  while (lim < pos + 2ull * mx + 4) {
    const uint32_t pb = vs.published;
    if (pb > rr) {
      rr = pb;
      lim = s.conv_base + (unsigned long long)rr * 24;
      __threadfence_block();
    } else if (++spins > BATH_SPIN_LIMIT) {
      fail = true;
      return pos;
    }
  }
  float ln = __uint_as_float(s.lap[(pos + 1) & M]);
  do {
    c++;
    const double step = (double)ln * inv;
    pos += 2;
    ln = __uint_as_float(s.lap[(pos + 1) & M]);
    nbv += step;
  } while ((nbv < T1) && (c < mx));
  if (c >= mx && nbv < T1) {
    do {   // single draws past the cap (rare)
      while (lim <= pos) {
        const uint32_t pb = vs.published;
        if (pb > rr) {
          rr = pb;
          lim = s.conv_base + (unsigned long long)rr * 24;
          __threadfence_block();
        } else if (++spins > BATH_SPIN_LIMIT) {
          fail = true;
          return pos;
        }
      }
      nbv += (double)__uint_as_float(s.lap[pos & M]) * inv;
      pos += 1;
    } while (nbv < T1);
  }
  return pos;
}

__device__ static inline int bath_builder_index(uint32_t warp) {
  return (warp >= 5 && warp <= 7) ? (int)warp - 5 : (warp >= 9 && warp <= 15) ? (int)warp - 6 : -1;
}

__global__ void __launch_bounds__(BATH_THREADS, 2) bath_kernel(Dev d) {
  const uint32_t t = *d.bath_t;
  extern __shared__ __align__(16) unsigned char bath_smem_raw[];
  BathSmem &s = *reinterpret_cast<BathSmem *>(bath_smem_raw);
  volatile BathSmem &vs = s;
  const NetConst *net = d.net;
  const uint32_t h = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t M = BATH_RING - 1;
  // restore: generator history, consumer position, draws converted last launch
  const unsigned long long p0 = d.bath_pos[h], q0 = d.bath_produced[h];
  if (tid < 64) s.hist[tid] = d.bath_hist[h * 64 + tid];
  for (unsigned long long n = p0 + tid; n < q0; n += blockDim.x) {
    const uint32_t k = (uint32_t)n & M;
    s.lap[k] = __float_as_uint(d.draw_lapse[(size_t)h * BATH_RING + k]);
    s.idx[k] = d.draw_idx[(size_t)h * BATH_RING + k];
  }
  for (uint32_t r = tid; r < BATH_ROUNDS; r += blockDim.x) s.flag[r] = 0;
  for (uint32_t r = tid; r < 256; r += blockDim.x) s.near[r] = d.fix_near[r];
  if (tid == 0) {
    s.pos = p0;
    s.raw_end = q0;
    s.conv_base = q0;
    s.next_round = 0;
    s.published = 0;
    s.done = 0;
    s.err = 0;
    s.chunk_seq = 0;
    s.e_seq = 0;
    s.emit_done = 0;
    s.emit_pos = p0;
    for (int b = 0; b < BATH_TABS; b++) s.tab_cnt[b] = 0;
    s.q[bath_qi(p0 - 2)] = 0;   // the prefix starts at p0 in each launch
    s.q[bath_qi(p0 - 1)] = 0;
  }
  __syncthreads();
  if (warp == 0) {   // prefix of the restored draws [p0, q0)
    for (unsigned long long n0 = p0; n0 < q0; n0 += 32) {
      const unsigned long long n = n0 + lane;
      uint32_t v = (n < q0) ? lap_fixed(__uint_as_float(s.lap[n & M])) : 0u;
      for (int o = 2; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (uint32_t)o) v += y;
      }
      v += s.q[bath_qi(n0 - 2 + (lane & 1))];
      __syncwarp();
      if (n < q0) s.q[bath_qi(n)] = v;
      __syncwarp();
    }
  }
  __syncthreads();
  const double T1 = (double)((double)t + 1.0);
  const uint32_t locN = net->locN, i0 = h * locN;
  const uint64_t ev_base = d.bath_rank_base[h];

  if (warp == 1) {
    // ---- generator
    uint32_t r = 0;
    while (true) {
      const unsigned long long n0 = s.conv_base + (unsigned long long)r * 24;
      uint32_t spins = 0;
      while (!vs.done && n0 + 24 > vs.emit_pos + BATH_RING - 64) {
        if (++spins > BATH_SPIN_LIMIT) { vs.err = 1; vs.done = 1; break; }
        __nanosleep(64);   // leave the issue slots to the consumer
      }
      if (vs.done) break;
      const uint32_t nn = (uint32_t)(n0 + lane);
      int32_t x = 0;
      if (lane < 24) {
        x = (int32_t)s.hist[(nn - 55) & 63] - (int32_t)s.hist[(nn - 24) & 63];
        if (x < 0) x += MBIG;
      }
      __syncwarp();
      if (lane < 24) {
        s.hist[nn & 63] = (uint32_t)x;
        s.lap[nn & M] = (uint32_t)x;
      }
      __syncwarp();
      __threadfence_block();
      if (lane == 0) vs.raw_end = n0 + 24;
      r++;
    }
  } else if (bath_builder_index(warp) >= 0) {
    // ---- count tables, two chunks ahead of the walk
    const uint32_t bw = (uint32_t)bath_builder_index(warp);
    unsigned long long pred = p0;   // predicted start of chunk c
    uint32_t exp1 = 0, exp2 = 0;    // expected events of chunks c-1 and c-2
    unsigned long long lim = s.raw_end;
    uint32_t rr = 0, spins = 0;
    bool fail = false;
    // What does not depend on where a chunk starts -- each lane's neuron,
    // its bounds and expected events, their prefix over the chunk -- is
    // prepared a chunk early: the next chunk's loads are in flight while
    // this chunk's candidates are evaluated.
    uint32_t n_lo = 0, n_hi1 = 0, n_misc = 0, n_ec = 0, n_incl = 0;
    double x_nb = 0, x_inv = 0;
    uint32_t x_mx = 0;
    auto prepare = [&](uint32_t cc0) {
      const uint32_t ccn = min(32u, locN - cc0);
      n_lo = n_hi1 = n_misc = n_ec = 0;
      if (lane < ccn) {
        bath_bounds(T1, x_nb, x_inv, x_mx, n_lo, n_hi1, n_misc);
        if (n_misc) n_ec = 1u + (uint32_t)fmin(rint((T1 - x_nb) / x_inv), 64.0);   // expected events: 1 + budget
      }
      n_incl = n_ec;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, n_incl, o);
        if (lane >= (uint32_t)o) n_incl += y;
      }
    };
    if (lane < min(32u, locN)) {
      x_nb = d.nb_prev[i0 + lane];
      x_inv = d.inv_nu[i0 + lane];
      x_mx = d.max_ext[i0 + lane];
    }
    prepare(0);
    for (uint32_t c = 0, c0 = 0; c0 < locN; c++, c0 += 32) {
      const uint32_t cn = min(32u, locN - c0), b = c % BATH_TABS;
      const uint32_t lo = n_lo, hi1 = n_hi1, misc = n_misc, ec = n_ec, incl = n_incl;
      if (c0 + 32 < locN && lane < min(32u, locN - c0 - 32)) {   // the next chunk's neurons
        x_nb = d.nb_prev[i0 + c0 + 32 + lane];
        x_inv = d.inv_nu[i0 + c0 + 32 + lane];
        x_mx = d.max_ext[i0 + c0 + 32 + lane];
      }
      // the prediction starts from the latest chunk start known for sure,
      // chunk c-2's (BATH_AHEAD = 2), published by the consumer as it begins
      // that chunk (so it is also done with this buffer's previous tables),
      // plus the expected events of chunks c-2 and c-1; chunk 0 starts at p0
      unsigned long long floor_pos = p0;
      if (c >= 3) {
        while (vs.chunk_seq < c - 1) {
          if (vs.done) { fail = true; break; }
          if (++spins > BATH_SPIN_LIMIT) { vs.err = 1; vs.done = 1; fail = true; break; }
          __nanosleep(32);
        }
        if (fail) break;
        __threadfence_block();
        floor_pos = vs.chunk_start[(c - 2) % BATH_TABS];
      }
      pred = floor_pos + 2ull * ((c >= 2 ? exp2 : 0u) + (c >= 1 ? exp1 : 0u));
      exp2 = exp1;
      exp1 = __shfl_sync(0xffffffffu, incl, 31);
      // candidate o of this lane's neuron starts at base + 2o, the
      // prediction in the middle of the window
      const unsigned long long base = pred + 2ull * (incl - ec) - BATH_NC;
      // the draws every candidate of the chunk reads are converted; never
      // beyond what the generator may produce ahead of the walk (once the
      // emitter is done with the chunks before c-2, at least floor_pos +
      // BATH_RING - 64): candidates past that stay undecided
      const unsigned long long reach = floor_pos + BATH_RING - 512;
      const unsigned long long need =
          min(__shfl_sync(0xffffffffu, base, 31) + 2ull * BATH_NC + BATH_WINDOW, reach);
      while (lim < need) {
        const uint32_t pb = vs.published;
        if (pb > rr) {
          rr = pb;
          lim = s.conv_base + (unsigned long long)rr * 24;
          __threadfence_block();
        } else if (vs.done) {
          fail = true;
          break;
        } else if (++spins > BATH_SPIN_LIMIT) {
          vs.err = 1;
          vs.done = 1;
          fail = true;
          break;
        } else {
          __nanosleep(32);
        }
      }
      if (fail) break;
      const uint32_t b32 = (uint32_t)base, f32 = (uint32_t)floor_pos;
      const uint32_t r32 = (uint32_t)reach - BATH_WINDOW;
      // this warp's quads of the chunk: the rank's quads go to the builders
      // in turn (quad 8c + k to builder (8c + k) mod BATH_BUILDERS), so the
      // builders share the quads evenly and need no other warp
      for (uint32_t k = (bw + BATH_BUILDERS - (8 * c) % BATH_BUILDERS) % BATH_BUILDERS; k < 8; k += BATH_BUILDERS) {
        // stage 1: the quad's neurons j = 4k .. 4k+3, two at a time (a half
        // warp each); for neuron j the half's lanes take the candidates
        // o = hl, hl + 16, hl + 32, hl + 48.  For a start P the count is
        // m + 1, m the number of i < 32 whose sum of the i+1 lapses at P+1,
        // P+3, .., P+1+2i is below lo (the sums grow with i), when the
        // (m+1)-th sum reaches hi1.  Positions are taken modulo 2^32 (a step
        // reads far fewer draws); the four candidates' binary searches run
        // in lockstep.
        for (uint32_t jp = 4 * k; jp < 4 * k + 4; jp += 2) {
          const uint32_t hl = lane & 15u, j = jp + (lane >> 4);
          const uint32_t mj = __shfl_sync(0xffffffffu, misc, j);
          const uint32_t loj = __shfl_sync(0xffffffffu, lo, j), hij = __shfl_sync(0xffffffffu, hi1, j);
          const uint32_t bj = __shfl_sync(0xffffffffu, b32, j);
          uint8_t *row = s.tab[b][j];
          if (!mj) {   // no bath event this step (or past the rank's last neuron): 0 from any start
#pragma unroll
            for (int v = 0; v < 4; v++) row[hl + 16 * v] = 0;
          } else {
            const uint32_t cap = mj & 0xFFu;
            // draw P+1+2i of a candidate sits at word hv | ((w0 + i) mod 4096) of q[]
            const uint32_t hv = ((bj + 1) & 1u) * (BATH_RING / 2);
            uint32_t w0[4], qb[4], m[4];
            bool ok[4];
#pragma unroll
            for (int v = 0; v < 4; v++) {
              const uint32_t P = bj + 2u * (hl + 16u * v);
              ok[v] = (int32_t)(P - f32) >= 0 && (int32_t)(r32 - P) >= 0;
              w0[v] = (P + 1) >> 1;
              qb[v] = s.q[hv | ((w0[v] - 1) & (BATH_RING / 2 - 1))];
              m[v] = 0;
            }
#pragma unroll
            for (uint32_t st = 16; st > 0; st >>= 1) {
              uint32_t f[4];
#pragma unroll
              for (int v = 0; v < 4; v++) f[v] = s.q[hv | ((w0[v] + m[v] + st - 1) & (BATH_RING / 2 - 1))];
#pragma unroll
              for (int v = 0; v < 4; v++) m[v] += (f[v] - qb[v] < loj) ? st : 0u;
            }
#pragma unroll
            for (int v = 0; v < 4; v++) {
              const uint32_t F = s.q[hv | ((w0[v] + m[v]) & (BATH_RING / 2 - 1))] - qb[v];
              const uint32_t mm = (m[v] == 31 && F < loj) ? 32u : m[v];
              row[hl + 16 * v] = (ok[v] && mm < cap && F >= hij) ? (uint8_t)(mm + 1) : (uint8_t)0xFF;
            }
          }
        }
        // the quad's window bases, and each table's answer outside its
        // window: 0 when none of its neurons has an event, else undecided
        const uint32_t mq = __shfl_sync(0xffffffffu, misc, 4 * k + (lane & 3));
        const uint32_t bq = __shfl_sync(0xffffffffu, b32, 4 * k + (lane & 3));
        const uint32_t B0 = __shfl_sync(0xffffffffu, b32, 4 * k), B1 = __shfl_sync(0xffffffffu, b32, 4 * k + 1);
        const uint32_t B2 = __shfl_sync(0xffffffffu, b32, 4 * k + 2), B3 = __shfl_sync(0xffffffffu, b32, 4 * k + 3);
        const uint32_t m2a = __shfl_sync(0xffffffffu, mq, 0) | __shfl_sync(0xffffffffu, mq, 1);
        const uint32_t m2b = __shfl_sync(0xffffffffu, mq, 2) | __shfl_sync(0xffffffffu, mq, 3);
        if (lane < 4) {
          s.bp_base[b][4 * k + lane] = bq;
          *reinterpret_cast<uint32_t *>(&s.tab[b][4 * k + lane][BATH_NC]) = mq ? 0xFFFFFFFFu : 0u;
        }
        if (lane == 0) {
          *reinterpret_cast<uint32_t *>(&s.tab2[b][2 * k][BATH_NC]) = m2a ? 0xFFFFFFFFu : 0u;
          *reinterpret_cast<uint32_t *>(&s.tab2[b][2 * k + 1][BATH_NC]) = m2b ? 0xFFFFFFFFu : 0u;
          *reinterpret_cast<uint32_t *>(&s.tab4[b][k][BATH_NC]) = (m2a | m2b) ? 0xFFFFFFFFu : 0u;
        }
        __syncwarp();
        // stage 2: the two pairs, from each candidate start of neuron 2p through 2p+1
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const uint32_t pp = 2 * k + (v >> 1), o = lane + 32u * (v & 1), a = 2 * pp;
          const uint32_t ba = (v >> 1) ? B2 : B0, bn = (v >> 1) ? B3 : B1;
          const uint32_t ca = s.tab[b][a][o];
          uint32_t val = 0xFFu;
          if (ca != 0xFFu) {
            const uint32_t cb = s.tab[b][a + 1][bath_row(ba + 2 * (o + ca) - bn)];
            if (cb != 0xFFu) val = ca + cb;
          }
          s.tab2[b][pp][o] = (uint8_t)val;
        }
        __syncwarp();
        // stage 3: the quad, from each candidate start of neuron 4k through its two pairs
#pragma unroll
        for (int v = 0; v < 2; v++) {
          const uint32_t o = lane + 32u * v;
          const uint32_t va = s.tab2[b][2 * k][o];
          uint32_t val = 0xFFu;
          if (va != 0xFFu) {
            const uint32_t vb = s.tab2[b][2 * k + 1][bath_row(B0 + 2 * (o + va) - B2)];
            if (vb != 0xFFu) val = va + vb;   // at most 4 x 32
          }
          s.tab4[b][k][o] = (uint8_t)val;
        }
        __syncwarp();
        __threadfence_block();
        if (lane == 0) atomicAdd(&s.tab_cnt[b], 1u);
      }
      if (c0 + 32 < locN) prepare(c0 + 32);
    }
  } else if (warp == 2 || warp == 3) {
    // ---- converters: groups of BATH_CG rounds (3 draws per lane) are
    // claimed in order and published in order
    while (true) {
      uint32_t g = 0;
      if (lane == 0) g = atomicAdd(&s.next_round, 1u);
      g = __shfl_sync(0xffffffffu, g, 0);
      const uint32_t r0 = g * BATH_CG;
      const unsigned long long n0 = s.conv_base + (unsigned long long)r0 * 24;
      uint32_t spins = 0;
      bool quit = false;
      while (true) {
        if (vs.raw_end >= n0 + 24 * BATH_CG) break;
        if (vs.done) { quit = true; break; }
        if (++spins > BATH_SPIN_LIMIT) { vs.err = 1; vs.done = 1; quit = true; break; }
        __nanosleep(64);
      }
      if (quit) break;
      __threadfence_block();
      uint8_t ix[3];
      float lp[3];
      uint32_t v[3];
      {
        uint32_t raw[3];
#pragma unroll
        for (int i = 0; i < 3; i++) raw[i] = vs.lap[(n0 + lane + 32 * i) & M];
        bath_lapse3(d, s.near, raw, lp, ix);
      }
#pragma unroll
      for (int i = 0; i < 3; i++) v[i] = lap_fixed(lp[i]);
      // per-parity prefix over the 96 draws: within each 32, then the
      // totals of the earlier 32s (lanes 30, 31) carried
      for (int o = 2; o < 32; o <<= 1) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, v[i], o);
          if (lane >= (uint32_t)o) v[i] += y;
        }
      }
      const uint32_t c0 = __shfl_sync(0xffffffffu, v[0], 30 + (lane & 1));
      const uint32_t c1 = __shfl_sync(0xffffffffu, v[1], 30 + (lane & 1));
      v[1] += c0;
      v[2] += c0 + c1;
      // the previous group's prefix is final once its last flag is set
      if (r0 > 0) {
        spins = 0;
        while (true) {
          if (vs.flag[(r0 - 1) % BATH_ROUNDS] == r0) break;
          if (vs.done) { quit = true; break; }
          if (++spins > BATH_SPIN_LIMIT) { vs.err = 1; vs.done = 1; quit = true; break; }
          __nanosleep(32);
        }
        if (quit) break;   // nothing of this group was written
        __threadfence_block();
      }
      const uint32_t qb = vs.q[bath_qi(n0 - 2 + (lane & 1))];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const unsigned long long n = n0 + lane + 32 * i;
        s.lap[n & M] = __float_as_uint(lp[i]);
        s.idx[n & M] = ix[i];
        s.q[bath_qi(n)] = v[i] + qb;
      }
      __syncwarp();
      __threadfence_block();
      if (lane < BATH_CG) vs.flag[(r0 + lane) % BATH_ROUNDS] = r0 + lane + 1;
      if (lane == 0) atomicMax(&s.published, r0 + BATH_CG);   // groups finish in order, their stores need not
    }
  } else if (warp == 0) {
    // ---- walk (warp 0)
    unsigned long long pos = s.pos;
    unsigned long long lim = s.raw_end;   // converted draws available (prefix)
    uint32_t rr = 0;                      // rounds known converted
    uint32_t out = 0, spins = 0;
    bool fail = false;
    double nx_nb = 0, nx_inv = 0;
    uint32_t nx_mx = 0;
    if (lane < min(32u, locN)) {
      nx_nb = d.nb_prev[i0 + lane];
      nx_inv = d.inv_nu[i0 + lane];
      nx_mx = d.max_ext[i0 + lane];
    }
    for (uint32_t c0 = 0, ck = 0; c0 < locN && !fail; c0 += 32, ck++) {
      const uint32_t cn = min(32u, locN - c0), tb = ck % BATH_TABS, eb = ck & 1u;
      const double my_nb = nx_nb, my_inv = nx_inv;
      const uint32_t my_mx = nx_mx;
      // this chunk's count tables, then its start for the builders
      {
        uint32_t sp = 0;
        while (vs.tab_cnt[tb] < 8u * (ck / BATH_TABS + 1)) {
          if (vs.done || ++sp > BATH_SPIN_LIMIT) { fail = true; break; }
          __nanosleep(20);   // leave the shared-memory pipe to the builders
        }
        if (fail) break;
        __threadfence_block();
        if (lane == 0) {
          vs.chunk_start[ck % BATH_TABS] = pos;
          __threadfence_block();
          vs.chunk_seq = ck + 1;
        }
      }
      if (c0 + 32 < locN && lane < min(32u, locN - c0 - 32)) {   // prefetch the next chunk
        nx_nb = d.nb_prev[i0 + c0 + 32 + lane];
        nx_inv = d.inv_nu[i0 + c0 + 32 + lane];
        nx_mx = d.max_ext[i0 + c0 + 32 + lane];
      }
      // the serial chain: one lookup per quad at its actual start; a run
      // has no branch on the chain (an out-of-window start reads the
      // sentinel); the first undecided quad is walked neuron by neuron
      // below and the run goes on after it
      const unsigned long long base = pos;
      const uint32_t *bb = s.bp_base[tb];
      const uint8_t *t1 = &s.tab[tb][0][0], *t2 = &s.tab2[tb][0][0], *t4 = &s.tab4[tb][0][0];
      uint32_t P = (uint32_t)base, slow = 0;
      for (uint32_t k0 = 0; k0 < 8;) {
        uint32_t bad = 8;
#pragma unroll 4
        for (uint32_t k = k0; k < 8; k++) {
          const uint32_t v = t4[k * BATH_TROW + bath_row(P - bb[4 * k])];
          bad = (bad == 8 && v == 0xFFu) ? k : bad;
          if (lane == 0) s.c_start[4 * k] = P;
          P += 2 * v;
        }
        if (bad == 8) break;
        __syncwarp();
        P = s.c_start[4 * bad];
        for (uint32_t j = 4 * bad; j < 4 * bad + 4; j++) {
          uint32_t cx = t1[j * BATH_TROW + bath_row(P - bb[j])];
          uint32_t Pn = P + 2 * cx;
          if (cx == 0xFFu) {
            // the reference's loop from the actual start; the emitter
            // first finishes the earlier chunks, so that the ring holds
            // every draw the loop may read
            uint32_t sp = 0;
            while (vs.emit_done < ck) {
              if (vs.err || ++sp > BATH_SPIN_LIMIT) { fail = true; break; }
              __nanosleep(32);
            }
            if (fail) break;
            const unsigned long long pj = base + (uint32_t)(P - (uint32_t)base);
            const unsigned long long pe = bath_exact(s, __shfl_sync(0xffffffffu, my_nb, j),
                                                     __shfl_sync(0xffffffffu, my_inv, j),
                                                     __shfl_sync(0xffffffffu, my_mx, j), T1, pj, lim, rr, spins, fail, cx);
            if (fail) break;
            Pn = (uint32_t)pe;
          }
          if (lane == 0) {
            s.c_start[j] = P;
            s.c_cnt[j] = cx;
          }
          P = Pn;
        }
        if (fail) break;
        slow |= 1u << bad;
        k0 = bad + 1;
      }
      if (fail) break;
      __syncwarp();
      // every neuron's start and events: from its quad's start through the
      // pair and single tables (entries the quad's own entry was made of),
      // or as the neuron-by-neuron walk recorded them
      uint32_t my_start, my_cnt;
      if ((slow >> (lane >> 2)) & 1u) {
        my_start = s.c_start[lane];
        my_cnt = s.c_cnt[lane];
      } else {
        uint32_t pq = s.c_start[lane & ~3u];
        if (lane & 2u) pq += 2 * t2[((lane >> 1) & ~1u) * BATH_TROW + bath_row(pq - bb[lane & ~3u])];
        if (lane & 1u) pq += 2 * t1[(lane & ~1u) * BATH_TROW + bath_row(pq - bb[lane & ~1u])];
        my_start = pq;
        my_cnt = t1[lane * BATH_TROW + bath_row(pq - bb[lane])];
      }
      if (lane >= cn) my_cnt = 0;
      uint32_t tot = my_cnt;
      for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      pos = base + (uint32_t)(P - (uint32_t)base);
      // hand the chunk to the emitter: buffer eb is free once chunk ck-2 is emitted
      if (ck >= 2) {
        uint32_t sp = 0;
        while (vs.emit_done < ck - 1) {
          if (vs.err || ++sp > BATH_SPIN_LIMIT) { fail = true; break; }
          __nanosleep(32);
        }
        if (fail) break;
      }
      s.e_start[eb][lane] = my_start;
      s.e_cnt[eb][lane] = my_cnt;
      if (lane == 0) {
        s.e_out[eb] = out;
        s.e_end[eb] = pos;
      }
      out += tot;
      __syncwarp();
      __threadfence_block();
      if (lane == 0) vs.e_seq = ck + 1;
    }
    if (lane == 0) {
      if (fail) vs.err = 1;
      vs.pos = pos;
      __threadfence_block();
      vs.done = 1;
    }
  } else if (warp == 4) {
    // ---- emitter (warp 4): a chunk's events, each lane replaying its
    // neuron in the reference's arithmetic
    double nx_nb = 0, nx_inv = 0;
    uint32_t nx_mx = 0;
    if (lane < min(32u, locN)) {
      nx_nb = d.nb_prev[i0 + lane];
      nx_inv = d.inv_nu[i0 + lane];
      nx_mx = d.max_ext[i0 + lane];
    }
    for (uint32_t c0 = 0, ck = 0; c0 < locN; c0 += 32, ck++) {
      const uint32_t cn = min(32u, locN - c0), eb = ck & 1u;
      const double my_nb = nx_nb, my_inv = nx_inv;
      const uint32_t my_mx = nx_mx;
      if (c0 + 32 < locN && lane < min(32u, locN - c0 - 32)) {
        nx_nb = d.nb_prev[i0 + c0 + 32 + lane];
        nx_inv = d.inv_nu[i0 + c0 + 32 + lane];
        nx_mx = d.max_ext[i0 + c0 + 32 + lane];
      }
      bool quit = false;
      uint32_t sp = 0;
      while (vs.e_seq < ck + 1) {
        if (vs.err) { quit = true; break; }
        if (++sp > BATH_SPIN_LIMIT) { vs.err = 1; vs.done = 1; quit = true; break; }
        __nanosleep(32);
      }
      if (__any_sync(0xffffffffu, quit)) break;
      __threadfence_block();
      const uint32_t my_start = s.e_start[eb][lane], my_cnt = s.e_cnt[eb][lane];
      const uint32_t out = s.e_out[eb];
      const unsigned long long end = s.e_end[eb];
      if (__any_sync(0xffffffffu, lane < cn && my_cnt > my_mx)) {   // beyond the rank's event slots
        if (lane == 0) { vs.err = 1; vs.done = 1; }
        break;
      }
      uint32_t incl = my_cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const uint32_t my_off = out + incl - my_cnt;
      if (lane < cn) {
        double v = my_nb;
        uint32_t p = my_start;
        double *bt = d.bath_time + ev_base + my_off;
        uint8_t *bl = d.bath_lut + ev_base + my_off;
        for (uint32_t c = 0; c < my_cnt; c++) {
          bt[c] = v;
          bl[c] = s.idx[p & M];
          v += (double)__uint_as_float(s.lap[(p + 1) & M]) * my_inv;
          p += 2;
        }
        if (my_cnt >= my_mx && my_cnt > 0 && v < T1) {
          do {   // single draws past the cap
            v += (double)__uint_as_float(s.lap[p & M]) * my_inv;
            p += 1;
          } while (v < T1);
        }
        d.nb[i0 + c0 + lane] = v;
        d.bath_off[i0 + c0 + lane] = my_off;
        d.bath_cnt[i0 + c0 + lane] = (uint16_t)my_cnt;
      }
      __syncwarp();
      __threadfence_block();
      if (lane == 0) {
        vs.emit_pos = end;
        __threadfence_block();
        vs.emit_done = ck + 1;
      }
    }
  }
  __syncthreads();
  if (s.err) {
    if (tid == 0) atomicOr(d.flags, F_BATH_DRAWS);
    return;
  }
  // convert the generated rounds no converter published (they follow the
  // published ones, and still hold raw draws), then save the state
  const unsigned long long re = s.raw_end;
  for (unsigned long long n = s.conv_base + 24ull * s.published + tid; n < re; n += blockDim.x) {
    uint8_t ix = 0;
    const float lp = bath_lapse(d, s.lap[n & M], ix);
    s.lap[n & M] = __float_as_uint(lp);
    s.idx[n & M] = ix;
  }
  __syncthreads();
  for (unsigned long long n = s.pos + tid; n < re; n += blockDim.x) {
    const uint32_t k = (uint32_t)n & M;
    d.draw_lapse[(size_t)h * BATH_RING + k] = __uint_as_float(s.lap[k]);
    d.draw_idx[(size_t)h * BATH_RING + k] = s.idx[k];
  }
  if (tid < 64) d.bath_hist[h * 64 + tid] = s.hist[tid];
  if (tid == 0) {
    d.bath_pos[h] = s.pos;
    d.bath_produced[h] = re;
  }
}

// LIFCADynamic, non-PerseoDyn branch (DPSNN_neuron_sim.c:664-824): lifca_pre
// below.
struct NeuronRegs {
  double v, c, tr, te;
  int fired;
};
// The coefficients of one update: deltaT = t - Tr.  They depend on event
// times only (Tr is the previous event's time), so the neuron run computes
// them one event ahead, off the dependent chain of v and c.
__device__ static inline void lifca_coeff(double Tau, double TauC, double deltaT, double &dth, double &rmh,
                                          double &poly) {
  dth = deltaT / 2;
  rmh = dth / Tau;
  const double rc = deltaT / TauC;
  poly = 1 - rc + rc * rc / 2;
}

// LIFCADynamic with the coefficients of this event computed ahead; the branch
// that leaves the refractory period moves deltaT, and recomputes them.
__device__ static inline void lifca_pre(const NetConst *net, uint32_t s, NeuronRegs &n, double t, double I,
                                        double dth, double rmh, double poly) {
  const double Tau = net->Tau[s], Theta = net->Theta[s], H = net->H[s], Tarp = net->Tarp[s];
  const double AlphaC = net->AlphaC[s], TauC = net->TauC[s], gC = net->gC[s];
  double v = n.v, c = n.c, Te = n.te;
  const double Tr = n.tr, TFLES = t - Te;
  if (TFLES > Tarp) {
    const double TrTe = Tr - Te;
    if (TrTe < Tarp) {
      const double deltaT0 = t - Tr;
      c *= exp_cr(-(deltaT0 - TFLES + Tarp) / TauC);
      lifca_coeff(Tau, TauC, TFLES - Tarp, dth, rmh, poly);
    }
    v = v - v * rmh - gC * c * dth;
    v = v - v * rmh - gC * c * dth;
    c = c * poly;
    v += I;
    if (v >= Theta) {
      v = H;
      c += AlphaC;
      Te = t;
      n.fired = 1;
    }
  } else {
    c = c * poly;
  }
  n.v = v;
  n.c = c;
  n.tr = t;
  n.te = Te;
}

__device__ static inline double event_time(const Dev &d, uint32_t key, uint32_t t, uint32_t D, uint32_t N) {
  uint32_t dl = (D - 1) - (key >> 25), q = key & ((1u << 25) - 1);
  double te = d.ring_te[(size_t)((t + RING_SLOTS - dl) % RING_SLOTS) * N + q];
  return (double)t + (te - floor(te));   // thisTimeStepF + modf(originalEmissionTime)
}

// Runs the merged event sequence of one neuron: synaptic events (sorted by
// (time, key)) merged with the bath events (time-ordered), synaptic first on
// equal times (mergeFunction, DPSNN_neuron_sim.c:391-421, called at :644-646).
// One event of a light neuron's insertion sort (thread-local): one 16-byte
// load or store per move.  The warp sorts keep separate arrays, whose 8- and
// 4-byte shared accesses conflict less at the network's short strides.
struct __align__(16) SortEv {
  double tau;
  uint32_t key;
  float val;
};

__device__ static inline bool sortev_gt(const SortEv &a, const SortEv &b) {
  return (a.tau > b.tau) || (a.tau == b.tau && a.key > b.key);
}


template <typename Events>
__device__ static inline int run_neuron_ev(const Dev &d, uint32_t i, uint32_t t, const Events &evs, uint32_t ns) {
  const NetConst *net = d.net;
  const uint32_t s = d.sub[i];
  NeuronRegs n;
  n.v = d.v[i];
  n.c = d.c[i];
  n.tr = d.tr[i];
  n.te = d.te[i];
  n.fired = 0;
  const double T0 = (double)t;
  const uint32_t boff = d.bath_off[i], bc = d.bath_cnt[i];
  const uint64_t bbase = d.bath_rank_base[i / net->locN] + boff;
  const double *lut = d.lut + (size_t)s * 256;
  const double Tau = net->Tau[s], TauC = net->TauC[s];
  uint32_t a = 0, b = 0;
  double bt = (b < bc) ? d.bath_time[bbase] : 0.0;
  // the merge's next event (time, input)
  auto next = [&](double &ct, double &I) -> bool {
    if (a < ns && (b >= bc || evs.time(a) <= bt)) {
      ct = evs.time(a);
      I = (double)evs.weight(a);
      a++;
      return true;
    }
    if (b < bc) {
      ct = bt;
      I = lut[d.bath_lut[bbase + b]];
      b++;
      if (b < bc) bt = d.bath_time[bbase + b];
      return true;
    }
    return false;
  };
  double ct = 0, I = 0, dth = 0, rmh = 0, poly = 0;
  bool have = next(ct, I);
  if (have) lifca_coeff(Tau, TauC, ct - n.tr, dth, rmh, poly);
  while (have) {
    double ct1 = 0, I1 = 0, dth1 = 0, rmh1 = 0, poly1 = 0;
    const bool have1 = next(ct1, I1);
    if (have1) lifca_coeff(Tau, TauC, ct1 - ct, dth1, rmh1, poly1);   // after this event Tr = ct
    if (((ct - T0) >= 1.0) || ((ct - T0) < 0)) atomicOr(d.flags, F_TIME_WINDOW);
    lifca_pre(net, s, n, ct, I, dth, rmh, poly);
    ct = ct1;
    I = I1;
    dth = dth1;
    rmh = rmh1;
    poly = poly1;
    have = have1;
  }
  d.v[i] = n.v;
  d.c[i] = n.c;
  d.tr[i] = n.tr;
  d.te[i] = n.te;
  if (n.fired) d.fired[i] = 1;
  return n.fired;
}

struct EvArrays {   // sorted times and weights in two arrays
  const double *tau;
  const float *val;
  __device__ double time(uint32_t a) const { return tau[a]; }
  __device__ float weight(uint32_t a) const { return val[a]; }
};
struct EvRecords {  // sorted 16-byte records
  const SortEv *se;
  __device__ double time(uint32_t a) const { return se[a].tau; }
  __device__ float weight(uint32_t a) const { return se[a].val; }
};

__device__ static inline int run_neuron(const Dev &d, uint32_t i, uint32_t t, const double *tau,
                                        const float *val, uint32_t ns) {
  return run_neuron_ev(d, i, t, EvArrays{tau, val}, ns);
}
__device__ static inline int run_neuron_se(const Dev &d, uint32_t i, uint32_t t, const SortEv *se, uint32_t ns) {
  return run_neuron_ev(d, i, t, EvRecords{se}, ns);
}

// Step 4: neuron update (regularDynamicTimeStep, DPSNN_neuron_sim.c:522-662).
// Light neurons (at most LOCAL_EVENTS synaptic events this step): one thread
// each, insertion sort by (arrival time, key) in registers/local memory.
// Heavier neurons are queued for the heavy path below.
__device__ static inline uint32_t warp_path_max(const NetConst *net);

__global__ void __launch_bounds__(NEURON_BLOCK, 4) neuron_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t, N = net->N, D = net->D, cap = net->ev_cap;
  const uint32_t i = blockIdx.x * NEURON_BLOCK + threadIdx.x;
  int fired = 0;
  if (i < N) {
    const uint32_t cnt = d.ev_cnt[i];
    d.ev_cnt[i] = 0;
    if (cnt > net->light_max) {
      const uint32_t path = (cnt <= warp_path_max(net)) ? 0u : 1u;
      const uint32_t k = atomicAdd(&d.heavy_cnt[path], 1u);
      if (k < N) {
        d.heavy_list[2ull * N * path + k] = i;
        d.heavy_list[2ull * N * path + N + k] = cnt;
      }
    } else {
      SortEv se[LOCAL_EVENTS];
      const uint2 *ev = d.ev + (size_t)i * cap;
      // events in groups of NEURON_BATCH: the loads, then the arrival-time
      // gathers, are all in flight together; then insertion by (time, key)
      for (uint32_t e0 = 0; e0 < cnt; e0 += NEURON_BATCH) {
        uint2 x[NEURON_BATCH];
        double tm[NEURON_BATCH];
#pragma unroll
        for (int u = 0; u < NEURON_BATCH; u++)
          if (e0 + u < cnt) x[u] = ev[e0 + u];
#pragma unroll
        for (int u = 0; u < NEURON_BATCH; u++)
          if (e0 + u < cnt) tm[u] = event_time(d, x[u].x, t, D, N);
#pragma unroll
        for (int u = 0; u < NEURON_BATCH; u++) {
          if (e0 + u < cnt) {
            SortEv y;
            y.tau = tm[u];
            y.key = x[u].x;
            y.val = __uint_as_float(x[u].y);
            uint32_t p = e0 + u;
            while (p > 0 && sortev_gt(se[p - 1], y)) {
              se[p] = se[p - 1];
              p--;
            }
            se[p] = y;
          }
        }
      }
      fired = run_neuron_se(d, i, t, se, cnt);
    }
  }
  const uint32_t bc = __syncthreads_count(fired);
  if (threadIdx.x == 0) d.block_fired[blockIdx.x] = bc;
}

// Heavy neurons, more than LOCAL_EVENTS synaptic events in one step.
// heavy_sort_kernel: one warp per neuron with at most HEAVY_WARP_MAX events
// loads its bucket into registers, computes the arrival times, sorts by
// (time, key) and writes the sorted events back into the bucket;
// heavy_run_kernel then runs those neurons one thread each.  Neurons with
// more events (including any beyond the bucket, in the overflow list) are
// sorted by huge_kernel, one block each; those with at most half a bucket of
// events go back to the bucket and run in heavy_run_kernel, the others run
// in their block.
#define HEAVY_WARP_MAX 256     // events a warp sorts (8 per lane)
#define HEAVY_MAX 8192
#define HEAVY_THREADS 256
#define HUGE_SMEM_EVENTS 2048   // a huge neuron sorted in shared memory (32 KB); more in global scratch

__device__ static inline void bitonic_sort_shared(double *tau, uint32_t *key, float *val, uint32_t n2,
                                                  uint32_t tid, uint32_t nthr, bool warp_only) {
  for (uint32_t k = 2; k <= n2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      // pair p compares a = p with bit j inserted as 0, and b = a | j
      for (uint32_t p = tid; p < (n2 >> 1); p += nthr) {
        const uint32_t a = ((p & ~(j - 1)) << 1) | (p & (j - 1)), b = a | j;
        const bool up = (a & k) == 0;
        const double ta = tau[a], tb = tau[b];
        const uint32_t ka = key[a], kb = key[b];
        const bool gt = (ta > tb) || (ta == tb && ka > kb);
        if (gt == up) {
          tau[a] = tb;
          tau[b] = ta;
          key[a] = kb;
          key[b] = ka;
          const float va = val[a];
          val[a] = val[b];
          val[b] = va;
        }
      }
      if (warp_only) __syncwarp(); else __syncthreads();
    }
  }
}

// Events per neuron handled by the warp path: at most the bucket size.
// (the sorted times and weights are written back into the first half and
// the second half of the bucket)
__device__ static inline uint32_t warp_path_max(const NetConst *net) {
  return min(net->ev_cap / 2, (uint32_t)HEAVY_WARP_MAX);
}

// A warp's sort of one heavy neuron's events: a bucket sort on the arrival
// time.  Arrival times lie in [t, t+1); bucket (time - t) * 256 is monotone
// in the time, so buckets order the events, and inside a bucket each event's
// place is the number of the bucket's events before it in (time, key) order
// (keys are unique per target).  Buckets are small unless many events share
// one arrival time, as a cascade's do; then the count is quadratic in the
// bucket's size, spread over the lanes.
#define HS_BUCKETS 256

#define HS_BATH_MAX 128         // bath events a warp merges into the sorted stream

struct HeavySortWarp {
  uint32_t start[HS_BUCKETS + 1];   // counts, then the buckets' first positions
  double tau[HEAVY_WARP_MAX + HS_BATH_MAX];   // events staged by bucket for the counts
  uint32_t key[HEAVY_WARP_MAX + HS_BATH_MAX];
};

// A heavy neuron's merged event stream in its bucket: {time, input} per
// event, synaptic and bath events in the order the reference merges them
// (mergeFunction, DPSNN_neuron_sim.c:391-421: a synaptic event first on
// equal times).  The list's count entry carries this flag when the sort
// left the stream merged.
#define HEAVY_MERGED 0x80000000u

// One heavy neuron's n <= 32*E events (element e = lane + 32r in register r):
// loaded with their arrival times and sorted by (time, key).  When the
// merged stream fits half the bucket, the neuron's bath events join the sort
// with keys above every synaptic key (so a synaptic event comes first on
// equal times, and bath events keep their order) and the bucket receives the
// merged stream {time, input}; otherwise it receives the sorted times in its
// first half and the weights in its second half.  Returns whether merged.
#define HS_BATH_KEY 0xFFFFFF80u   // + j for bath event j; synaptic keys are below 80 << 25
static_assert(RING_SLOTS <= 127, "synaptic keys (D-1-d) << 25 | q stay below the bath keys");

template <int E>
__device__ static inline bool heavy_sort_one(const Dev &d, uint32_t i, uint2 *ev, uint32_t n, uint32_t t, uint32_t D,
                                             uint32_t N, uint32_t cap, uint32_t lane, HeavySortWarp &w) {
  const double T0 = (double)t;
  const uint32_t bcnt = d.bath_cnt[i];
  const uint64_t bbase = d.bath_rank_base[i / d.net->locN] + d.bath_off[i];
  const bool merged = n + bcnt <= cap / 2 && bcnt <= HS_BATH_MAX;
  const uint32_t bc = merged ? bcnt : 0u;
  for (uint32_t b = lane; b <= HS_BUCKETS; b += 32) w.start[b] = 0;
  uint2 x[E];
#pragma unroll
  for (int r = 0; r < E; r++) {
    const uint32_t e = lane + 32u * r;
    if (e < n) x[r] = ev[e];
  }
  __syncwarp();
  double tau[E];
  uint32_t bs[E], bb[HS_BATH_MAX / 32];   // bucket << 16 | place among the bucket's elements in arrival order
#pragma unroll
  for (int r = 0; r < E; r++) {
    const uint32_t e = lane + 32u * r;
    if (e < n) {
      tau[r] = event_time(d, x[r].x, t, D, N);
      const uint32_t b = min((uint32_t)((tau[r] - T0) * (double)HS_BUCKETS), (uint32_t)HS_BUCKETS - 1);
      bs[r] = (b << 16) | atomicAdd(&w.start[b], 1u);
    }
  }
#pragma unroll
  for (int r = 0; r < HS_BATH_MAX / 32; r++) {
    const uint32_t j = lane + 32u * r;
    if (j < bc) {
      const double btj = d.bath_time[bbase + j];
      const uint32_t b = min((uint32_t)((btj - T0) * (double)HS_BUCKETS), (uint32_t)HS_BUCKETS - 1);
      bb[r] = (b << 16) | atomicAdd(&w.start[b], 1u);
    }
  }
  __syncwarp();
  // exclusive prefix of the counts, 8 consecutive buckets per lane
  {
    uint32_t c[HS_BUCKETS / 32], tot = 0;
#pragma unroll
    for (int q = 0; q < HS_BUCKETS / 32; q++) {
      c[q] = w.start[lane * (HS_BUCKETS / 32) + q];
      const uint32_t v = c[q];
      c[q] = tot;
      tot += v;
    }
    uint32_t incl = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
#pragma unroll
    for (int q = 0; q < HS_BUCKETS / 32; q++) w.start[lane * (HS_BUCKETS / 32) + q] = incl - tot + c[q];
    if (lane == 31) w.start[HS_BUCKETS] = incl;
  }
  __syncwarp();
  // staged by bucket; bs/bb become bucket << 16 | staged position
#pragma unroll
  for (int r = 0; r < E; r++) {
    const uint32_t e = lane + 32u * r;
    if (e < n) {
      const uint32_t b = bs[r] >> 16, p = w.start[b] + (bs[r] & 0xFFFFu);
      w.tau[p] = tau[r];
      w.key[p] = x[r].x;
      bs[r] = (b << 16) | p;
    }
  }
#pragma unroll
  for (int r = 0; r < HS_BATH_MAX / 32; r++) {
    const uint32_t j = lane + 32u * r;
    if (j < bc) {
      const uint32_t b = bb[r] >> 16, p = w.start[b] + (bb[r] & 0xFFFFu);
      w.tau[p] = d.bath_time[bbase + j];
      w.key[p] = HS_BATH_KEY + j;
      bb[r] = (b << 16) | p;
    }
  }
  __syncwarp();
  // each element's place: its bucket's start plus the bucket's elements
  // before it in (time, key) order
  auto place = [&](uint32_t v) -> uint32_t {
    const uint32_t b = v >> 16, p = v & 0xFFFFu;
    const uint32_t b0 = w.start[b], b1 = w.start[b + 1], k = w.key[p];
    const double tm = w.tau[p];
    uint32_t rank = 0;
    for (uint32_t j = b0; j < b1; j++) {
      const double tj = w.tau[j];
      rank += (tj < tm) || (tj == tm && w.key[j] < k);
    }
    return b0 + rank;
  };
  double2 *ms = reinterpret_cast<double2 *>(ev);
  double *st = reinterpret_cast<double *>(ev);
  float *sv = reinterpret_cast<float *>(ev + cap / 2);
#pragma unroll
  for (int r = 0; r < E; r++) {
    const uint32_t e = lane + 32u * r;
    if (e < n) {
      const uint32_t pos = place(bs[r]);
      const double tm = w.tau[bs[r] & 0xFFFFu];
      if (merged) {
        ms[pos] = make_double2(tm, (double)__uint_as_float(x[r].y));
      } else {
        st[pos] = tm;
        sv[pos] = __uint_as_float(x[r].y);
      }
    }
  }
  if (merged) {
    const double *lut = d.lut + (size_t)d.sub[i] * 256;
#pragma unroll
    for (int r = 0; r < HS_BATH_MAX / 32; r++) {
      const uint32_t j = lane + 32u * r;
      if (j < bc) ms[place(bb[r])] = make_double2(w.tau[bb[r] & 0xFFFFu], lut[d.bath_lut[bbase + j]]);
    }
  }
  __syncwarp();   // the warp's next neuron reuses the staging arrays
  return merged;
}

#define HEAVY_SORT_THREADS 256

// A warp per neuron of the warp path (LOCAL_EVENTS < n <= HEAVY_WARP_MAX),
// each warp with its own bucket-sort arrays in shared memory.  Two kernels
// over the same list: up to 64 events (one or two per lane, the common case
// outside bursts) at four blocks per SM, more events (four or eight per lane,
// more registers) at two.
#define HEAVY_SORT_SMALL 64

template <bool SMALL>
__device__ static inline void heavy_sort_list(const Dev &d) {
  __shared__ HeavySortWarp s_ws[HEAVY_SORT_THREADS / 32];
  const NetConst *net = d.net;
  const uint32_t t = *d.t, N = net->N, D = net->D, cap = net->ev_cap, wmax = warp_path_max(net);
  const uint32_t lane = threadIdx.x & 31;
  HeavySortWarp &ws = s_ws[threadIdx.x >> 5];
  const uint32_t nh = min(d.heavy_cnt[0], N);
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  // a neuron not listed here was sorted already by the other kernel, which
  // flags the count
  auto mine = [&](uint32_t n) { return n <= wmax && (SMALL ? n <= HEAVY_SORT_SMALL : n > HEAVY_SORT_SMALL); };
  // the warp's list entries are read two neurons ahead, and the next
  // neuron's events are prefetched into L2 while this one is sorted
  uint32_t hh = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t i = 0, n = 0, i1 = 0, n1 = 0;
  if (hh < nh) {
    i = d.heavy_list[hh];
    n = d.heavy_list[N + hh];
  }
  if (hh + nwarps < nh) {
    i1 = d.heavy_list[hh + nwarps];
    n1 = d.heavy_list[N + hh + nwarps];
  }
  for (; hh < nh; hh += nwarps) {
    const uint32_t h2 = hh + 2u * nwarps;
    uint32_t i2 = 0, n2 = 0;
    if (h2 < nh) {
      i2 = d.heavy_list[h2];
      n2 = d.heavy_list[N + h2];
    }
    // 16 events (128 bytes) per lane's line, inside neuron i1's bucket
    if (hh + nwarps < nh && mine(n1) && lane * 16u < n1)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(d.ev + (size_t)i1 * cap + lane * 16u));
    if (mine(n)) {
      uint2 *ev = d.ev + (size_t)i * cap;
      bool merged;
      if (SMALL) {
        if (n <= 32)
          merged = heavy_sort_one<1>(d, i, ev, n, t, D, N, cap, lane, ws);
        else
          merged = heavy_sort_one<2>(d, i, ev, n, t, D, N, cap, lane, ws);
      } else {
        if (n <= 128)
          merged = heavy_sort_one<4>(d, i, ev, n, t, D, N, cap, lane, ws);
        else
          merged = heavy_sort_one<8>(d, i, ev, n, t, D, N, cap, lane, ws);
      }
      if (merged && lane == 0) d.heavy_list[N + hh] = n | HEAVY_MERGED;
    }
    i = i1;
    n = n1;
    i1 = i2;
    n1 = n2;
  }
}

__global__ void __launch_bounds__(HEAVY_SORT_THREADS, 4) heavy_sort_kernel(Dev d) { heavy_sort_list<true>(d); }
__global__ void __launch_bounds__(HEAVY_SORT_THREADS, 2) heavy_sort_big_kernel(Dev d) { heavy_sort_list<false>(d); }

// Runs a neuron whose events were left sorted in its bucket (arrival times,
// then weights): the warp path's neurons, and the block path's neurons with
// at most half a bucket of events, which huge_kernel sorts and leaves there.
// Same merge and arithmetic as run_neuron.
__device__ static inline bool huge_runs_here(const NetConst *net, uint32_t cnt) {
  return cnt <= net->ev_cap / 2 && cnt <= MAX_INPUTS_PER_STEP;
}

// A neuron's merged stream of ne events ({time, input}, in the order they
// apply): LIFCADynamic over it, four events' loads in flight ahead of the
// four being applied, each update's coefficients computed off the v/c chain.
__device__ static inline int run_neuron_merged(const Dev &d, uint32_t i, uint32_t t, const double2 *ms,
                                               uint32_t ne) {
  const NetConst *net = d.net;
  const uint32_t s = d.sub[i];
  NeuronRegs n;
  n.v = d.v[i];
  n.c = d.c[i];
  n.tr = d.tr[i];
  n.te = d.te[i];
  n.fired = 0;
  const double T0 = (double)t;
  const double Tau = net->Tau[s], TauC = net->TauC[s];
  double2 cur[4], nxt[4];
#pragma unroll
  for (int u = 0; u < 4; u++) cur[u] = (u < (int)ne) ? ms[u] : make_double2(0.0, 0.0);
  bool bad = false;
  for (uint32_t e0 = 0; e0 < ne; e0 += 4) {
#pragma unroll
    for (int u = 0; u < 4; u++) nxt[u] = (e0 + 4 + u < ne) ? ms[e0 + 4 + u] : make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (e0 + u < ne) {
        const double ct = cur[u].x;
        double dth, rmh, poly;
        lifca_coeff(Tau, TauC, ct - n.tr, dth, rmh, poly);
        bad |= ((ct - T0) >= 1.0) || ((ct - T0) < 0);
        lifca_pre(net, s, n, ct, cur[u].y, dth, rmh, poly);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) cur[u] = nxt[u];
  }
  if (bad) atomicOr(d.flags, F_TIME_WINDOW);
  d.v[i] = n.v;
  d.c[i] = n.c;
  d.tr[i] = n.tr;
  d.te[i] = n.te;
  if (n.fired) d.fired[i] = 1;
  return n.fired;
}

// The warp path's neurons whose sort left a merged stream, a thread each.
__global__ void __launch_bounds__(128, 6) heavy_run_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t, N = net->N, cap = net->ev_cap;
  const uint32_t nh = min(d.heavy_cnt[0], N);
  for (uint32_t hh = blockIdx.x * blockDim.x + threadIdx.x; hh < nh; hh += gridDim.x * blockDim.x) {
    const uint32_t i = d.heavy_list[hh], ns = d.heavy_list[N + hh];
    if (!(ns & HEAVY_MERGED)) continue;
    const uint32_t ne = (ns & ~HEAVY_MERGED) + d.bath_cnt[i];
    if (run_neuron_merged(d, i, t, reinterpret_cast<const double2 *>(d.ev + (size_t)i * cap), ne))
      atomicAdd(&d.block_fired[i / NEURON_BLOCK], 1u);
  }
}

// The other neurons left sorted in their bucket (times and weights in its
// halves, merged with the bath events here): the warp path's neurons whose
// merged stream would not fit half the bucket, and the block path's with at
// most half a bucket of events.  A thread each.
__global__ void heavy_rest_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t, N = net->N, cap = net->ev_cap, wmax = warp_path_max(net);
  const uint32_t nh0 = min(d.heavy_cnt[0], N), nh = nh0 + min(d.heavy_cnt[1], N);
  for (uint32_t hh = blockIdx.x * blockDim.x + threadIdx.x; hh < nh; hh += gridDim.x * blockDim.x) {
    uint32_t i, ns;
    if (hh < nh0) {
      i = d.heavy_list[hh];
      ns = d.heavy_list[N + hh];
      if ((ns & HEAVY_MERGED) || ns > wmax) continue;
    } else {
      i = d.heavy_list[2ull * N + (hh - nh0)];
      ns = d.heavy_list[3ull * N + (hh - nh0)];
      if (ns <= wmax || !huge_runs_here(net, ns)) continue;
    }
    const uint2 *ev = d.ev + (size_t)i * cap;
    const double *st = reinterpret_cast<const double *>(ev);
    const float *sv = reinterpret_cast<const float *>(ev + cap / 2);
    if (run_neuron_ev(d, i, t, EvArrays{st, sv}, ns)) atomicAdd(&d.block_fired[i / NEURON_BLOCK], 1u);
  }
}

// Gather a neuron's events (bucket, then overflow list) into shared arrays.
__device__ static inline uint32_t gather_events(const Dev &d, uint32_t i, uint32_t cnt, uint32_t *key, float *val,
                                                uint32_t capacity, uint32_t tid, uint32_t nthr, uint32_t *counter) {
  const NetConst *net = d.net;
  const uint32_t cap = net->ev_cap, nb = min(cnt, cap);
  for (uint32_t e = tid; e < nb; e += nthr) {
    const uint2 x = d.ev[(size_t)i * cap + e];
    key[e] = x.x;
    val[e] = __uint_as_float(x.y);
  }
  if (tid == 0) *counter = nb;
  __syncthreads();
  if (cnt > cap) {
    const uint32_t novf = min(*d.ovf_cnt, net->ovf_cap);
    for (uint32_t o = tid; o < novf; o += nthr) {
      const uint4 x = d.ovf[o];
      if (x.x == i) {
        uint32_t k = atomicAdd(counter, 1u);
        if (k < capacity) {
          key[k] = x.y;
          val[k] = __uint_as_float(x.z);
        }
      }
    }
    __syncthreads();
  }
  return min(*counter, capacity);
}

__global__ void __launch_bounds__(HEAVY_THREADS) huge_kernel(Dev d) {
  // 32 KB of shared memory, so that a block fits on an SM beside the bath's
  // blocks; the rare neuron with more events sorts in its block's global
  // scratch (HEAVY_MAX events)
  __shared__ double sh_tau[HUGE_SMEM_EVENTS];
  __shared__ uint32_t sh_key[HUGE_SMEM_EVENTS];
  __shared__ float sh_val[HUGE_SMEM_EVENTS];
  __shared__ uint32_t s_n;
  const NetConst *net = d.net;
  const uint32_t t = *d.t, N = net->N, D = net->D, tid = threadIdx.x;
  const uint32_t nh = min(d.heavy_cnt[1], N);
  const uint32_t *hl = d.heavy_list + 2ull * N;
  for (uint32_t hh = blockIdx.x; hh < nh; hh += gridDim.x) {
    const uint32_t i = hl[hh], cnt = hl[N + hh];
    if (cnt <= warp_path_max(net)) continue;   // not listed here
    if (cnt > MAX_INPUTS_PER_STEP) {
      if (tid == 0) atomicOr(d.flags, F_TOO_MANY_INPUTS);
      continue;
    }
    const bool in_smem = cnt <= HUGE_SMEM_EVENTS;
    double *s_tau = in_smem ? sh_tau : d.huge_tau + (size_t)blockIdx.x * HEAVY_MAX;
    uint32_t *s_key = in_smem ? sh_key : d.huge_key + (size_t)blockIdx.x * HEAVY_MAX;
    float *s_val = in_smem ? sh_val : d.huge_val + (size_t)blockIdx.x * HEAVY_MAX;
    const uint32_t n = gather_events(d, i, cnt, s_key, s_val, in_smem ? HUGE_SMEM_EVENTS : HEAVY_MAX, tid,
                                     blockDim.x, &s_n);
    uint32_t n2 = 1;
    while (n2 < n) n2 <<= 1;
    for (uint32_t e = tid; e < n2; e += blockDim.x) {
      if (e < n) {
        s_tau[e] = event_time(d, s_key[e], t, D, N);
      } else {
        s_tau[e] = INFINITY;
        s_key[e] = 0xFFFFFFFFu;
      }
    }
    __syncthreads();
    bitonic_sort_shared(s_tau, s_key, s_val, n2, tid, blockDim.x, false);
    if (huge_runs_here(net, cnt)) {
      // sorted back into the bucket's halves; heavy_run_kernel runs the
      // neuron, beside the others, one thread each
      uint2 *ev = d.ev + (size_t)i * net->ev_cap;
      double *st = reinterpret_cast<double *>(ev);
      float *sv = reinterpret_cast<float *>(ev + net->ev_cap / 2);
      for (uint32_t e = tid; e < n; e += blockDim.x) {
        st[e] = s_tau[e];
        sv[e] = s_val[e];
      }
    } else if (tid == 0) {
      if (run_neuron(d, i, t, s_tau, s_val, n)) atomicAdd(&d.block_fired[i / NEURON_BLOCK], 1u);
    }
    __syncthreads();
  }
}

// Long term plasticity at x999 ms (longTermPlasticity, DPSNN_localNet_sim.c:312-414),
// one warp per presynaptic neuron.
__global__ void ltp_kernel(Dev d) {
  const NetConst *net = d.net;
  const uint32_t t = *d.t;
  if (!((t % 1000) == 999 && t >= net->start_pl && t <= net->stop_pl)) return;
  const uint32_t N = net->N, lane = threadIdx.x & 31;
  for (uint32_t P = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; P < N;
       P += (gridDim.x * blockDim.x) >> 5) {
    uint32_t sp = d.sub[P];
    for (uint64_t k = d.row_ptr[P] + lane; k < d.row_ptr[P + 1]; k += 32) {
      uint32_t tp = d.sub[d.post[k]];
      float maxv = (float)(2.0 * net->J[sp * DPSNN_MAX_SUBPOP + tp]);
      float rmaxv = (float)(2.0 * net->J[tp * DPSNN_MAX_SUBPOP + sp]);
      float clamp = 0.0f;
      float td = d.tderiv[k];
      const int16_t w0 = d.w16[k];
      if (d.probe_w) {
        d.probe_w[k] = w0;
        d.probe_td[k] = td;
      }
      if (maxv > 0.0 && rmaxv > 0.0) {
        float wF = (float)(w0 * net->w2f);
        float dF = td;
        dF += net->stdp_drift;
        wF = wF + dF;
        if (wF > maxv) { clamp = (wF - maxv); dF = dF - clamp; wF = maxv; }
        if (wF < 0.0) { clamp = wF; dF = dF - clamp; wF = 0.0f; }
        d.w16[k] = (int16_t)(wF * net->f2w);
        td = dF;
      }
      if (d.probe_w) d.probe_td_mid[k] = td;
      if (net->stdp_tauDecay == 1.0f)
        td = 0.0f;
      else
        td = (td - net->stdp_drift + clamp) * (1 - 1 / net->stdp_tauDecay);
      d.tderiv[k] = td;
    }
  }
}

// After each bath launch, on the bath stream: the next bath's step.
__global__ void bath_tick_kernel(Dev d) { *d.bath_t = *d.bath_t + 1; }

__global__ void end_step_kernel(Dev d) {
  *d.ovf_cnt = 0;
  d.heavy_cnt[0] = 0;
  d.heavy_cnt[1] = 0;
  *d.t = *d.t + 1;
}

// Per-(neuron, delay) counts of the chosen hypothesis -> per-row totals and
// the in-row per-delay offsets.
__global__ void counts_to_csr_kernel(const NetConst *net, const uint16_t *cnt_out,
                                     const int32_t *hyp, uint16_t *sub_off, uint32_t *row_len) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= net->N) return;
  uint32_t D = net->D;
  int h = hyp[i / net->npcm];
  const uint16_t *c = cnt_out + ((size_t)h * net->N + i) * D;
  uint32_t acc = 0;
  for (uint32_t dl = 0; dl < D; dl++) {
    sub_off[(size_t)i * (D + 1) + dl] = (uint16_t)acc;
    acc += c[dl];
  }
  sub_off[(size_t)i * (D + 1) + D] = (uint16_t)acc;
  row_len[i] = acc;
}

__global__ void init_neurons_kernel(Dev d) {
  const NetConst *net = d.net;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= net->N) return;
  // initNeuralKind (DPSNN_neuron_init.c:99-115); Tr is zero (static storage)
  d.v[i] = net->H[d.sub[i]];
  d.c[i] = 0.0;
  d.te[i] = -1000;
  d.nb[i] = 0.0;
  d.tr[i] = 0.0;
  d.fired[i] = 0;
  d.last_spike_ms[i] = -100000;  // DPSNN_localNet_init.c:217
  d.ev_cnt[i] = 0;
}

// incoming-synapse lists (causal STDP), per post neuron
__global__ void in_count_kernel(const NetConst *net, const uint32_t *post, uint64_t S, uint64_t *in_ptr) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < S; k += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd((unsigned long long *)&in_ptr[post[k] + 1], 1ull);
}
__global__ void in_fill_kernel(const NetConst *net, const uint32_t *post, uint64_t S, const uint64_t *in_ptr,
                               unsigned long long *fill, uint32_t *in_idx) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < S; k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t j = post[k];
    unsigned long long p = atomicAdd(&fill[j], 1ull);
    in_idx[in_ptr[j] + p] = (uint32_t)k;
  }
}

// per (rank, delay): max and min presynaptic index among synapses aimed at
// that rank -- used to detect the reference's run-over-group-end search case
__global__ void group_extrema_kernel(const NetConst *net, const uint64_t *row_ptr, const uint16_t *sub_off,
                                     const uint32_t *post, uint32_t *gmax, uint32_t *gmin) {
  const uint32_t N = net->N, D = net->D, lane = threadIdx.x & 31;
  for (uint32_t P = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; P < N; P += (gridDim.x * blockDim.x) >> 5) {
    for (uint32_t dl = 0; dl < D; dl++) {
      uint64_t b = row_ptr[P] + sub_off[(size_t)P * (D + 1) + dl], e = row_ptr[P] + sub_off[(size_t)P * (D + 1) + dl + 1];
      for (uint64_t k = b + lane; k < e; k += 32) {
        uint32_t h = post[k] / net->locN;
        atomicMax(&gmax[h * D + dl], P);
        atomicMin(&gmin[h * D + dl], P);
      }
    }
  }
}

// ------------------------------------------------------------------ host engine
struct dpsnn_engine {
  NetConst hnet;
  Dev d;
  cudaStream_t stream = nullptr;
  // The bath of step t+1 runs on bath_stream while step t runs on stream:
  // its outputs and nextBath are double-buffered by step parity.
  cudaStream_t bath_stream = nullptr;
  cudaEvent_t ev_bath[2] = {nullptr, nullptr}, ev_neuron[2] = {nullptr, nullptr}, ev_start = nullptr;
  bool bath_primed = false;
  double *nb2[2] = {nullptr, nullptr}, *bath_time2[2] = {nullptr, nullptr};
  uint8_t *bath_lut2[2] = {nullptr, nullptr};
  uint32_t *bath_off2[2] = {nullptr, nullptr};
  uint16_t *bath_cnt2[2] = {nullptr, nullptr};
  int device = 0;
  uint64_t S = 0;
  uint32_t t_host = 0;   // steps enqueued
  uint32_t probe_t = UINT32_MAX;   // step of the last LTP probe taken
  uint32_t stdp_log_t = UINT32_MAX;   // step the STDP event log holds
  std::vector<uint64_t> h_row;     // host copies of the CSR row and delay offsets
  std::vector<uint16_t> h_so;      // (for the STDP event log's order)
  std::vector<void *> allocs;
  std::vector<void *> temps;       // build scratch, released when the build ends
  uint64_t bytes = 0;              // device memory held (allocs)
  uint32_t grid_neuron = 0, grid_deliver = 0, grid_heavy = 0, grid_heavy_run = 0, grid_huge = 0;
  int sms = 148;                   // the device's SMs (default grids)
  int timing = 0;
  bool capturing = false;          // steps are being recorded into a graph
  struct TimedLaunch { int family; cudaEvent_t a, b; cudaStream_t st; };
  std::vector<TimedLaunch> pending;   // recorded, not yet read
  std::vector<cudaEvent_t> event_pool;
  double ktime[DPSNN_TIMING_SLOTS] = {};
  uint64_t klaunch[DPSNN_TIMING_SLOTS] = {};
  uint64_t launches = 0;               // kernels enqueued by dpsnn_step
  std::vector<float> fix_vals;
  std::vector<uint32_t> fix_keys, fix_bucket;
  uint32_t *h_pin = nullptr;          // pinned {flags, spike count} for per-step reads
  // spike lists are read on their own stream as soon as the compaction of
  // their step is done, while the rest of that step (and later ones) run
  cudaStream_t read_stream = nullptr;
  cudaEvent_t ev_slot[RING_SLOTS] = {};
};

static void collect_timings(dpsnn_engine *e);

// Device allocations are stream-ordered on the engine stream (the
// device's memory pool): unlike cudaMalloc/cudaFree they do not synchronise
// the device, so engines built from several host threads, or while other
// engines step, do not wait for each other.  `temp` allocations (the
// connectome build's scratch) are released at the end of the build.
template <typename T>
static int dalloc(dpsnn_engine *e, T **p, size_t n, bool temp = false) {
  void *q = nullptr;
  size_t bytes = std::max<size_t>(n * sizeof(T), 16);
  cudaError_t err = cudaMallocAsync(&q, bytes, e->stream);
  if (err != cudaSuccess)
    return dpsnn_fail(DPSNN_E_NOMEM, "cudaMallocAsync(%zu bytes): %s", bytes, cudaGetErrorString(err));
  (temp ? e->temps : e->allocs).push_back(q);
  if (!temp) e->bytes += bytes;
  err = cudaMemsetAsync(q, 0, bytes, e->stream);
  if (err != cudaSuccess) return dpsnn_fail(DPSNN_E_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(err));
  *p = (T *)q;
  return 0;
}
#define DALLOC(ptr, n)                          \
  do {                                          \
    int rc_ = dalloc(e, &(ptr), (size_t)(n));   \
    if (rc_) return rc_;                        \
  } while (0)
#define TALLOC(ptr, n)                                \
  do {                                                \
    int rc_ = dalloc(e, &(ptr), (size_t)(n), true);   \
    if (rc_) return rc_;                              \
  } while (0)

static void free_temps(dpsnn_engine *e) {
  for (void *q : e->temps) cudaFreeAsync(q, e->stream);
  e->temps.clear();
}

static int load_logf_fixup(dpsnn_engine *e) {
  std::string path = std::string(dpsnn_library_dir()) + "/logf_fixup.bin";
  const char *envp = getenv("DPSNN_LOGF_FIXUP");
  if (envp) path = envp;
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return dpsnn_fail(DPSNN_E_PARAM, "cannot open %s (built with the engine)", path.c_str());
  uint32_t n = 0;
  bool ok = fread(&n, 4, 1, f) == 1;
  e->fix_keys.resize(n);
  e->fix_vals.resize(n);
  e->fix_bucket.resize(LOGF_FIX_NBUCKET);
  ok = ok && fread(e->fix_keys.data(), 4, n, f) == n;
  ok = ok && fread(e->fix_vals.data(), 4, n, f) == n;
  ok = ok && fread(e->fix_bucket.data(), 4, LOGF_FIX_NBUCKET, f) == LOGF_FIX_NBUCKET;
  fclose(f);
  if (!ok) return dpsnn_fail(DPSNN_E_PARAM, "truncated %s", path.c_str());
  uint32_t *k; float *v; uint32_t *b;
  DALLOC(k, n);
  DALLOC(v, n);
  DALLOC(b, LOGF_FIX_NBUCKET);
  CK(cudaMemcpyAsync(k, e->fix_keys.data(), 4ull * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(v, e->fix_vals.data(), 4ull * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(b, e->fix_bucket.data(), 4ull * LOGF_FIX_NBUCKET, cudaMemcpyHostToDevice, e->stream));
  e->d.fix.keys = k;
  e->d.fix.vals = v;
  e->d.fix.bucket = b;
  e->d.fix.n = n;
  {
    const size_t words = ((size_t)(0x3F800000u - 0x30000000u) + 1 + 31) / 32;
    std::vector<uint32_t> bm(words, 0u);
    for (uint32_t key : e->fix_keys)
      if (key >= 0x30000000u && key <= 0x3F800000u) bm[(key - 0x30000000u) >> 5] |= 1u << ((key - 0x30000000u) & 31);
    uint32_t *dbm;
    DALLOC(dbm, words);
    CK(cudaMemcpyAsync(dbm, bm.data(), 4 * words, cudaMemcpyHostToDevice, e->stream));
    e->d.fix_bitmap = dbm;
    // per result binade, the fix-up inputs' largest distance (ulps) from a
    // rounding midpoint, with a margin for the device log's last bit
    std::vector<float> near(256, -1.0f);
    for (uint32_t key : e->fix_keys) {
      if (key < 0x30000000u || key > 0x3F800000u) continue;
      float xf;
      memcpy(&xf, &key, 4);
      const double y = log((double)xf);
      const float f = logf_cr_from(xf, y);
      uint32_t fb;
      memcpy(&fb, &f, 4);
      const uint32_t E = (fb >> 23) & 0xFFu;
      if ((fb & 0x7FFFFFu) == 0 || E <= 24) continue;   // always checked on the device
      const double dist = 0.5 - fabs(y - (double)f) * ldexp(1.0, 150 - (int)E);
      near[E] = std::max(near[E], (float)(dist + 1e-3));
    }
    float *dnear;
    DALLOC(dnear, 256);
    CK(cudaMemcpyAsync(dnear, near.data(), 4 * 256, cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    e->d.fix_near = dnear;
  }
  return 0;
}

// ---- erflib Gaussian LUT on the host (erflib.c:41-169), C library exp
static double h_erfcc(double x) {
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
                                              t * (1.48851587 + t * (-0.82215223 + t * 0.17087277)))))))));
  return x >= 0.0 ? ans : 2.0 - ans;
}
static double h_normcum(double x, double mu, double sigma) {
  return 1 - 0.5 * h_erfcc((x - mu) / (sqrt(2.0) * sigma));
}
static double h_cutnormcum(double x, double mu, double sigma, double a, double b) {
  double n0 = h_normcum(a, mu, sigma);
  return (h_normcum(x, mu, sigma) - n0) / (h_normcum(b, mu, sigma) - n0);
}
static double h_findprob(double p, double mu, double sigma, double a, double b) {
  double err = 1e-6, x, xmin = a, xmax = b;
  int maxit = 256, i = 0;
  if (p <= 0.0) return a;
  if (p >= 1.0) return b;
  while ((xmax - xmin) > err && i < maxit) {
    x = (xmax + xmin) * 0.5;
    if (h_cutnormcum(x, mu, sigma, a, b) < p)
      xmin = x;
    else
      xmax = x;
    i++;
  }
  return (xmax + xmin) * 0.5;
}
static void h_gaussian_lut(double mu, double sigma, double xmin, double xmax, double *table) {
  if (sigma > 0.0) {
    double dp = 1.0 / 256.0, x0, x1 = xmin, p;
    int i;
    for (p = dp, i = 0; p <= 1.0; p += dp, i++) {
      x0 = x1;
      x1 = h_findprob(p, mu, sigma, xmin, xmax);
      table[i] = (x1 + x0) * 0.5;
    }
  } else {
    for (int i = 0; i < 256; i++) table[i] = mu;
  }
}

// The kernels' shared-memory attributes, set once per device and process,
// before the device's first build: setting an attribute waits for the
// kernel's running instances, which would serialise the builds of engines
// built concurrently, and builds with other engines' steps.
static int set_kernel_attributes(int device) {
  static std::mutex mu;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (done[device]) return 0;
  CK(cudaFuncSetAttribute(gen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEN_SMEM));
  CK(cudaFuncSetAttribute(bath_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BathSmem)));
  // the bath's blocks stay resident for most of a step: with the largest
  // shared-memory carveout, the SMs that hold two of them still have room for
  // a block of the main stream's kernels that use shared memory
  CK(cudaFuncSetAttribute(bath_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                          (int)cudaSharedmemCarveoutMaxShared));
  done[device] = 1;
  return 0;
}

static int engine_build(dpsnn_engine *e, const dpsnn_params *p, const dpsnn_options *o) {
  NetConst &n = e->hnet;
  memset(&n, 0, sizeof n);
  if (p->nsub == 0 || p->nsub > DPSNN_MAX_SUBPOP)
    return dpsnn_fail(DPSNN_E_PARAM, "number of sub-populations %u out of range", p->nsub);
  if (p->stencil_dim == 0 || !p->spec || !p->bath) return dpsnn_fail(DPSNN_E_PARAM, "missing stencil description");
  if (p->D == 0 || p->D > RING_SLOTS) return dpsnn_fail(DPSNN_E_PARAM, "env_D=%u out of range [1,%d]", p->D, RING_SLOTS);
  if (p->glob_h == 0) return dpsnn_fail(DPSNN_E_PARAM, "env_globH must be >= 1");
  n.nsub = p->nsub;
  n.npcm = 0;
  for (uint32_t s = 0; s < n.nsub; s++) {
    n.offset[s] = n.npcm;
    n.count[s] = p->count[s];
    n.npcm += p->count[s];
  }
  if (n.npcm == 0) return dpsnn_fail(DPSNN_E_PARAM, "neuronsPerCM <= 0");
  n.cfx = p->cfx;
  n.cfy = p->cfy;
  n.nmod = p->cfx * p->cfy;
  if (n.nmod == 0) return dpsnn_fail(DPSNN_E_PARAM, "empty grid");
  if ((n.nmod % p->glob_h) != 0 || p->glob_h > n.nmod)
    return dpsnn_fail(DPSNN_E_PARAM, "#processes and #cort. columns must be multiple OR equal");
  n.P = p->glob_h;
  n.mods_per_rank = n.nmod / n.P;
  n.locN = n.npcm * n.mods_per_rank;
  n.N = n.locN * n.P;
  if ((uint64_t)n.npcm * n.nmod >= (1ull << 25))
    return dpsnn_fail(DPSNN_E_PARAM, "network of %llu neurons exceeds the engine limit of 2^25",
                      (unsigned long long)n.npcm * n.nmod);
  n.D = p->D;
  n.stencil_dim = p->stencil_dim;
  n.max_mod = p->stencil_dim - 1;
  n.stencil = 2 * p->stencil_dim - 1;
  for (uint32_t s = 0; s < n.nsub; s++) {
    n.Tau[s] = p->Tau[s];
    n.Theta[s] = p->Theta[s];
    n.H[s] = p->H[s];
    n.Tarp[s] = p->Tarp[s];
    n.AlphaC[s] = p->AlphaC[s];
    n.TauC[s] = p->TauC[s];
    n.gC[s] = p->gC[s];
    n.NuExt[s] = p->NuExt[s];
    for (uint32_t t = 0; t < n.nsub; t++) {
      n.J[s * DPSNN_MAX_SUBPOP + t] = p->J[s * p->nsub + t];
      n.DJ[s * DPSNN_MAX_SUBPOP + t] = p->DJ[s * p->nsub + t];
      n.DMin[s * DPSNN_MAX_SUBPOP + t] = p->DMin[s * p->nsub + t];
      n.DMax[s * DPSNN_MAX_SUBPOP + t] = p->DMax[s * p->nsub + t];
    }
  }
  {
    double dmin = 1e36, dmax = 0;
    for (uint32_t s = 0; s < n.nsub; s++)
      for (uint32_t t = 0; t < n.nsub; t++) {
        if (n.DMax[s * DPSNN_MAX_SUBPOP + t] > dmax) dmax = n.DMax[s * DPSNN_MAX_SUBPOP + t];
        if (n.DMin[s * DPSNN_MAX_SUBPOP + t] < dmin) dmin = n.DMin[s * DPSNN_MAX_SUBPOP + t];
      }
    n.delay_min = (uint32_t)dmin;
    n.delay_max = (uint32_t)dmax;
    n.delay_exp = p->delay_exponential ? 1u : 0u;
    n.inv_log_tn = (float)(1.0 / log_cr(0.05));
  }
  if (!(p->min_syn_weight_f < 0) || p->min_syn_weight_f < -6.0f)
    return dpsnn_fail(DPSNN_E_PARAM, "env_minSynWeigth out of range -6.000000 - 0.0");
  n.f2w = -32767 / p->min_syn_weight_f;
  n.w2f = p->min_syn_weight_f / -32767;
  n.min_w = p->min_syn_weight_f;
  n.global_seed = p->global_seed;
  n.start_pl = p->start_plasticity_ms;
  n.stop_pl = p->stop_plasticity_ms;
  n.stdp_on = (p->start_plasticity_ms <= p->stop_plasticity_ms &&
               p->start_plasticity_ms < (p->total_sim_time_ms ? p->total_sim_time_ms : 0xFFFFFFFFu)) ? 1 : 0;
  n.causal_tab[0] = p->stdp_causalMax * p->stdp_multiplier;
  n.causal_tab[1] = n.causal_tab[0];
  n.anti_tab[0] = p->stdp_antiCausalCoeff * p->stdp_antiCausalMax * p->stdp_multiplier;
  for (int i = 1; i < 128; i++) n.causal_tab[i] = (1 - 1 / p->stdp_tau_ms) * n.causal_tab[i - 1];
  for (int i = 1; i < 128; i++) n.anti_tab[i] = (1 - 1 / p->stdp_tau_ms) * n.anti_tab[i - 1];
  n.stdp_drift = p->stdp_drift;
  n.stdp_tauDecay = p->stdp_tauDecay_s;
  n.ev_cap = (o && o->events_per_neuron) ? o->events_per_neuron : DEFAULT_EVENT_CAP;
  {  // tuning knob: the largest event count of the thread-per-neuron path
    const char *lm = getenv("DPSNN_LIGHT_EVENTS");
    n.light_max = lm ? (uint32_t)atoi(lm) : LOCAL_EVENTS;
    if (n.light_max < 1 || n.light_max > LOCAL_EVENTS) n.light_max = LOCAL_EVENTS;
  }
  if (n.ev_cap > 4096) n.ev_cap = 4096;
  if (!(o && o->events_per_neuron)) {   // default: at most 16 GiB of event slots
    while (n.ev_cap > 64 && 8ull * n.ev_cap * n.N > (16ull << 30)) n.ev_cap >>= 1;
  }
  n.ovf_cap = (o && o->overflow_events) ? o->overflow_events : (1u << 22);

  Dev &d = e->d;
  const uint32_t N = n.N, D = n.D, P = n.P;
  DALLOC(d.net, 1);
  CK(cudaMemcpyAsync(d.net, &n, sizeof n, cudaMemcpyHostToDevice, e->stream));
  // bath LUTs (initLUT, DPSNN_LIFCAcorticalModuleGen.cpp:347-356)
  {
    std::vector<double> lut((size_t)n.nsub * 256);
    for (uint32_t s = 0; s < n.nsub; s++) {
      float J = p->JExt[s], DJ = p->DJExt[s];
      h_gaussian_lut(J, J * DJ, 0.0, 2.0 * J, &lut[(size_t)s * 256]);
    }
    DALLOC(d.lut, lut.size());
    CK(cudaMemcpyAsync(d.lut, lut.data(), lut.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
  }
  // mirrored stencil probabilities (initProbConnectMatrix, LIFCAconnectome.cpp:136-198)
  float *dprob;
  {
    const uint32_t st = n.stencil, M = n.max_mod, S = p->stencil_dim;
    std::vector<float> prob((size_t)DPSNN_MAX_SUBPOP * DPSNN_MAX_SUBPOP * st * st, 0.0f);
    for (uint32_t s = 0; s < n.nsub; s++)
      for (uint32_t t = 0; t < n.nsub; t++)
        for (uint32_t x = 0; x <= M; x++)
          for (uint32_t y = 0; y <= M; y++) {
            float v = p->spec[((size_t)(s * n.nsub + t) * S + x) * S + y];
            auto at = [&](uint32_t X, uint32_t Y) -> float & {
              return prob[(((size_t)s * DPSNN_MAX_SUBPOP + t) * st + X) * st + Y];
            };
            at(M + x, M + y) = v;
            at(M - x, M + y) = v;
            at(M - x, M - y) = v;
            at(M + x, M - y) = v;
          }
    TALLOC(dprob, prob.size());
    CK(cudaMemcpyAsync(dprob, prob.data(), prob.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
  }
  // neuron arrays
  DALLOC(d.v, N); DALLOC(d.c, N); DALLOC(d.tr, N); DALLOC(d.te, N);
  DALLOC(e->nb2[0], N); DALLOC(e->nb2[1], N);
  d.nb = e->nb2[0];
  d.nb_prev = e->nb2[1];
  DALLOC(d.inv_nu, N); DALLOC(d.max_ext, N); DALLOC(d.sub, N); DALLOC(d.fired, N);
  DALLOC(d.last_spike_ms, N);
  e->grid_neuron = (N + NEURON_BLOCK - 1) / NEURON_BLOCK;
  DALLOC(d.block_fired, e->grid_neuron);

  // ---- synapse generation, pass A (both NormDev-cache hypotheses)
  const uint32_t nmod = n.nmod;
  GenRecord *drec;
  uint16_t *cnt_out;
  uint32_t *scratch;
  TALLOC(drec, 2 * nmod);
  TALLOC(cnt_out, 2ull * N * D);
  const uint32_t SD = p->stencil_dim;
  uint32_t *bath_tmpl;
  {
    TALLOC(scratch, (size_t)2 * nmod * MAX_SYN_PER_NEURON);
    TALLOC(bath_tmpl, SD * SD);
    std::vector<uint32_t> bath(p->bath, p->bath + SD * SD);
    CK(cudaMemcpyAsync(bath_tmpl, bath.data(), 4ull * SD * SD, cudaMemcpyHostToDevice, e->stream));
  }
  int32_t *dhyp;
  double *dcache;
  TALLOC(dhyp, nmod);
  TALLOC(dcache, nmod);
  {
    int rc = set_kernel_attributes(e->device);
    if (rc) return rc;
  }
  gen_kernel<<<(2 * nmod + GEN_THREADS - 1) / GEN_THREADS, GEN_THREADS, GEN_SMEM, e->stream>>>(
      d.net, dprob, 0, drec, dhyp, dcache, cnt_out,
                                                          nullptr, nullptr, nullptr, nullptr, scratch,
                                                          bath_tmpl, nullptr, nullptr, nullptr);
  CK(cudaGetLastError());
  std::vector<GenRecord> rec(2 * nmod);
  CK(cudaMemcpyAsync(rec.data(), drec, sizeof(GenRecord) * 2 * nmod, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  for (uint32_t k = 0; k < 2 * nmod; k++)
    if (rec[k].err && !((k & 1) && (k / 2) % n.mods_per_rank == 0)) {
      const char *what[] = {"", "too many synapses generated for neuron", "synaptic weight out of minSynWeight_f range",
                            "connection probability in (0,1e-5] is not supported", "delay >= env_D",
                            "zero mean synaptic efficacy",
                            "ERROR: delay level generated beyond the 80 max allowed delay levels, source neuron",
                            "ERROR: delay generated beyond the pair's DMax, source neuron"};
      return dpsnn_fail(DPSNN_E_MODEL, "synapse generation: %s (%u)", what[rec[k].err], rec[k].err_arg);
    }
  // resolve the NormDev cache hand-off rank by rank, module by module
  std::vector<int32_t> hyp(nmod);
  std::vector<double> cache(nmod, 0.0);
  for (uint32_t h = 0; h < P; h++) {
    int32_t set = 0;
    double cval = 0.0;
    for (uint32_t mm = 0; mm < n.mods_per_rank; mm++) {
      uint32_t m = h * n.mods_per_rank + mm;
      int choose = 0;
      if (mm > 0 && set == 1) {
        const GenRecord &r1 = rec[2 * m + 1];
        if (!r1.used_normdev) {
          choose = 1;
        } else {
          float mean = r1.first_mean, sigma = r1.first_sigma;
          float wf = (float)(mean + cval * sigma);
          bool acc = (mean > 0.0) ? !((wf < 0.0) || (wf >= 2.0 * mean)) : !((wf <= 2.0 * mean) || (wf > 0));
          choose = acc ? 1 : 0;
        }
      }
      hyp[m] = choose;
      cache[m] = cval;
      const GenRecord &rc = rec[2 * m + choose];
      if (rc.used_normdev) {
        set = rc.set_out;
        cval = rc.cache_out;
      }
    }
  }
  CK(cudaMemcpyAsync(dhyp, hyp.data(), 4ull * nmod, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(dcache, cache.data(), 8ull * nmod, cudaMemcpyHostToDevice, e->stream));
  // ---- CSR offsets from the chosen counts
  uint32_t *row_len;
  DALLOC(d.sub_off, (size_t)N * (D + 1));
  TALLOC(row_len, N);
  counts_to_csr_kernel<<<(N + 255) / 256, 256, 0, e->stream>>>(d.net, cnt_out, dhyp, d.sub_off, row_len);
  CK(cudaGetLastError());
  std::vector<uint32_t> hlen(N);
  std::vector<uint64_t> hrow(N + 1);
  CK(cudaMemcpyAsync(hlen.data(), row_len, 4ull * N, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  hrow[0] = 0;
  for (uint32_t i = 0; i < N; i++) hrow[i + 1] = hrow[i] + hlen[i];
  e->S = hrow[N];
  DALLOC(d.row_ptr, N + 1);
  CK(cudaMemcpyAsync(d.row_ptr, hrow.data(), 8ull * (N + 1), cudaMemcpyHostToDevice, e->stream));
  DALLOC(d.post, e->S);
  DALLOC(d.w16, e->S);
  // ---- pass B: regenerate the chosen hypothesis straight into the CSR
  gen_kernel<<<(nmod + GEN_THREADS - 1) / GEN_THREADS, GEN_THREADS, GEN_SMEM, e->stream>>>(
      d.net, dprob, 1, drec, dhyp, dcache, cnt_out, d.row_ptr,
                                                      d.sub_off, d.post, d.w16, scratch, bath_tmpl, d.inv_nu,
                                                      d.max_ext, d.sub);
  CK(cudaGetLastError());
  std::vector<GenRecord> recB(nmod);
  CK(cudaMemcpyAsync(recB.data(), drec, sizeof(GenRecord) * nmod, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  for (uint32_t m = 0; m < nmod; m++)
    if (recB[m].err) return dpsnn_fail(DPSNN_E_MODEL, "synapse generation pass B error %d", recB[m].err);
  // ---- run-over-group-end check (see DPSNN_synapse.c:211-265): the reference's
  // search continues past a (delay, source rank) group while the next entry has
  // the same presynaptic index; this happens only when the last source of a
  // delay group is also the first source of the next non-empty group.
  {
    uint32_t *gmax, *gmin;
    TALLOC(gmax, (size_t)P * D);
    TALLOC(gmin, (size_t)P * D);
    CK(cudaMemsetAsync(gmin, 0xFF, 4ull * P * D, e->stream));
    group_extrema_kernel<<<std::min<uint32_t>(4096, (N + 7) / 8), 256, 0, e->stream>>>(d.net, d.row_ptr,
                                                                                     d.sub_off, d.post, gmax, gmin);
    CK(cudaGetLastError());
    std::vector<uint32_t> hmax((size_t)P * D), hmin((size_t)P * D);
    CK(cudaMemcpyAsync(hmax.data(), gmax, 4ull * P * D, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(hmin.data(), gmin, 4ull * P * D, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    for (uint32_t h = 0; h < P; h++)
      for (uint32_t dl = 0; dl < D; dl++) {
        if (hmin[h * D + dl] == 0xFFFFFFFFu) continue;
        uint32_t dn = dl + 1;
        while (dn < D && hmin[h * D + dn] == 0xFFFFFFFFu) dn++;
        if (dn < D && hmax[h * D + dl] == hmin[h * D + dn])
          return dpsnn_fail(DPSNN_E_MODEL,
                            "rank %u: neuron %u ends delay group %u and starts group %u; the reference's "
                            "search would run across the group boundary (not reproduced)",
                            h, hmax[h * D + dl], dl, dn);
      }
  }
  // ---- STDP arrays
  if (n.stdp_on && e->S > 0xFFFFFFFFull)   // in_idx holds 32-bit synapse indices
    return dpsnn_fail(DPSNN_E_CAPACITY, "plasticity supports at most 2^32-1 synapses (%llu generated)",
                      (unsigned long long)e->S);
  if (n.stdp_on) {
    DALLOC(d.tderiv, e->S);
    DALLOC(d.last_act, e->S);
    DALLOC(d.in_ptr, N + 1);
    DALLOC(d.in_idx, e->S);
    unsigned long long *fill;
    TALLOC(fill, N);
    in_count_kernel<<<2048, 256, 0, e->stream>>>(d.net, d.post, e->S, d.in_ptr);
    CK(cudaGetLastError());
    std::vector<uint64_t> ip(N + 1);
    CK(cudaMemcpyAsync(ip.data(), d.in_ptr, 8ull * (N + 1), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    for (uint32_t i = 0; i < N; i++) {
      if (ip[i + 1] >= 2 * MAX_SYN_PER_NEURON)
        return dpsnn_fail(DPSNN_E_MODEL, "ERROR too many syn incoming on neuron glob_n=%u", i);
      ip[i + 1] += ip[i];
    }
    CK(cudaMemcpyAsync(d.in_ptr, ip.data(), 8ull * (N + 1), cudaMemcpyHostToDevice, e->stream));
    in_fill_kernel<<<2048, 256, 0, e->stream>>>(d.net, d.post, e->S, d.in_ptr, fill, d.in_idx);
    CK(cudaGetLastError());
  }
  // ---- ring, events, bath
  DALLOC(d.ring_ids, (size_t)RING_SLOTS * N);
  DALLOC(d.ring_te, (size_t)RING_SLOTS * N);
  DALLOC(d.ring_cnt, RING_SLOTS);
  DALLOC(d.ev_cnt, N);
  DALLOC(d.ev, (size_t)N * n.ev_cap);
  DALLOC(d.ovf_cnt, 1);
  DALLOC(d.ovf, n.ovf_cap);
  DALLOC(d.heavy_list, 4ull * N);
  {   // huge_kernel's global scratch: one neuron of up to HEAVY_MAX events per block
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device);
    DALLOC(d.huge_tau, (size_t)nsm * HEAVY_MAX);
    DALLOC(d.huge_key, (size_t)nsm * HEAVY_MAX);
    DALLOC(d.huge_val, (size_t)nsm * HEAVY_MAX);
  }
  DALLOC(d.heavy_cnt, 2);
  DALLOC(d.t, 1);
  DALLOC(d.bath_t, 1);
  DALLOC(d.flags, 4);
  DALLOC(d.events, 1);
  init_neurons_kernel<<<(N + 255) / 256, 256, 0, e->stream>>>(d);
  CK(cudaGetLastError());
  {
    // per-rank bath event capacity = sum of maxExternCurrentCount
    std::vector<uint32_t> mx(N);
    CK(cudaMemcpyAsync(mx.data(), d.max_ext, 4ull * N, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    std::vector<uint64_t> base(P + 1, 0);
    for (uint32_t h = 0; h < P; h++) {
      uint64_t s = 0;
      for (uint32_t i = h * n.locN; i < (h + 1) * n.locN; i++) s += mx[i];
      base[h + 1] = base[h] + s;
    }
    uint32_t mx_max = 0;
    for (uint32_t i = 0; i < N; i++) mx_max = std::max(mx_max, mx[i]);
    // one 32-neuron chunk plus one neuron's look-ahead must fit in the draw ring
    if (mx_max > BATH_MAX_EXT || 66ull * mx_max + 200 > BATH_RING)
      return dpsnn_fail(DPSNN_E_CAPACITY, "maxExternCurrentCount %u exceeds what the bath ring holds (%d)", mx_max,
                        (BATH_RING - 200) / 66);
    n.bath_need = mx_max;
    CK(cudaMemcpyAsync(d.net, &n, sizeof n, cudaMemcpyHostToDevice, e->stream));
    DALLOC(d.bath_rank_base, P + 1);
    CK(cudaMemcpyAsync(d.bath_rank_base, base.data(), 8ull * (P + 1), cudaMemcpyHostToDevice, e->stream));
    for (int b = 0; b < 2; b++) {
      DALLOC(e->bath_time2[b], base[P]);
      DALLOC(e->bath_lut2[b], base[P]);
      DALLOC(e->bath_off2[b], N);
      DALLOC(e->bath_cnt2[b], N);
    }
    d.bath_time = e->bath_time2[0];
    d.bath_lut = e->bath_lut2[0];
    d.bath_off = e->bath_off2[0];
    d.bath_cnt = e->bath_cnt2[0];
    // dynamics streams: SetRandomSeed(loc_h) (DPSNN_localNet_init.c:283).
    // Rank 0 continues its generation stream; others re-initialise.
    std::vector<uint32_t> hist((size_t)P * 64, 0);
    std::vector<uint64_t> produced(P, 0), pos(P, 1);
    for (uint32_t h = 0; h < P; h++) {
      uint32_t h55[55];
      if (h == 0) {
        memcpy(h55, recB[n.mods_per_rank - 1].hist, sizeof h55);
      } else {
        Ran3 g;
        memset(&g, 0, sizeof g);
        g.idum = -(int32_t)h;
        // table initialisation only; the draw SetRandomSeed makes is x[0]
        int32_t mj = MSEED - (int32_t)h, mk;
        mj = (mj < 0 ? -mj : mj) % MBIG;
        g.ma[55] = mj;
        mk = 1;
        for (int i = 1; i <= 54; i++) {
          int ii = (21 * i) % 55;
          g.ma[ii] = mk;
          mk = mj - mk;
          if (mk < 0) mk += MBIG;
          mj = g.ma[ii];
        }
        for (int k = 1; k <= 4; k++)
          for (int i = 1; i <= 55; i++) {
            g.ma[i] -= g.ma[1 + (i + 30) % 55];
            if (g.ma[i] < 0) g.ma[i] += MBIG;
          }
        g.inext = 0;
        r3_history(g, h55);
      }
      // x[-55..-1] at ring positions (k-55) & 63
      for (int k = 0; k < 55; k++) hist[(size_t)h * 64 + ((k - 55) & 63)] = h55[k];
    }
    DALLOC(d.bath_hist, (size_t)P * 64);
    DALLOC(d.bath_produced, P);
    DALLOC(d.bath_pos, P);
    DALLOC(d.draw_idx, (size_t)P * BATH_RING);
    DALLOC(d.draw_lapse, (size_t)P * BATH_RING);
    CK(cudaMemcpyAsync(d.bath_hist, hist.data(), 4ull * P * 64, cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(d.bath_produced, produced.data(), 8ull * P, cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(d.bath_pos, pos.data(), 8ull * P, cudaMemcpyHostToDevice, e->stream));
  }
  int rc = load_logf_fixup(e);
  if (rc) return rc;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  e->sms = sms;
  e->grid_deliver = (uint32_t)sms * 8;
  e->grid_heavy = (uint32_t)sms * 8;
  e->grid_heavy_run = (uint32_t)sms * 16;
  e->grid_huge = (uint32_t)sms;
  free_temps(e);   // after their last use on this stream
  CK(cudaStreamSynchronize(e->stream));
  return 0;
}

extern "C" int dpsnn_create(const dpsnn_params *p, const dpsnn_options *opts, dpsnn_engine **out) {
  if (!p || !out) return dpsnn_fail(DPSNN_E_PARAM, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return dpsnn_fail(DPSNN_E_CUDA, "no CUDA device available");
  dpsnn_engine *e = new dpsnn_engine();
  if (opts && opts->device >= 0 && opts->device < ndev) {
    e->device = opts->device;
  } else {
    cudaGetDevice(&e->device);
  }
  // The bath of the next step runs beside this step's kernels and has a
  // step of slack; the main stream's blocks go first when both wait for room.
  int prio_least = 0, prio_greatest = 0;
  bool ok = cudaSetDevice(e->device) == cudaSuccess &&
            cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) == cudaSuccess &&
            cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, prio_greatest) == cudaSuccess &&
            cudaStreamCreateWithPriority(&e->bath_stream, cudaStreamNonBlocking, prio_least) == cudaSuccess;
  for (int b = 0; b < 2 && ok; b++)
    ok = cudaEventCreateWithFlags(&e->ev_bath[b], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&e->ev_neuron[b], cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&e->ev_start, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&e->read_stream, cudaStreamNonBlocking) == cudaSuccess;
  for (int k = 0; k < RING_SLOTS && ok; k++)
    ok = cudaEventCreateWithFlags(&e->ev_slot[k], cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaMallocHost((void **)&e->h_pin, 2 * sizeof(uint32_t)) == cudaSuccess;
  if (!ok) {
    const int dev = e->device;
    dpsnn_destroy(e);
    return dpsnn_fail(DPSNN_E_CUDA, "cannot set up device %d", dev);
  }
  int rc = engine_build(e, p, opts);
  if (rc) {
    dpsnn_destroy(e);
    return rc;
  }
  *out = e;
  return 0;
}

extern "C" void dpsnn_destroy(dpsnn_engine *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->bath_stream) cudaStreamSynchronize(e->bath_stream);
  if (e->read_stream) cudaStreamSynchronize(e->read_stream);
  if (e->stream) {
    free_temps(e);   // a build that stopped early
    for (void *q : e->allocs) cudaFreeAsync(q, e->stream);
    cudaStreamSynchronize(e->stream);
  }
  collect_timings(e);
  for (cudaEvent_t ev : e->event_pool) cudaEventDestroy(ev);
  for (int b = 0; b < 2; b++) {
    if (e->ev_bath[b]) cudaEventDestroy(e->ev_bath[b]);
    if (e->ev_neuron[b]) cudaEventDestroy(e->ev_neuron[b]);
  }
  if (e->ev_start) cudaEventDestroy(e->ev_start);
  for (int k = 0; k < RING_SLOTS; k++)
    if (e->ev_slot[k]) cudaEventDestroy(e->ev_slot[k]);
  if (e->read_stream) {
    cudaStreamSynchronize(e->read_stream);
    cudaStreamDestroy(e->read_stream);
  }
  if (e->h_pin) cudaFreeHost(e->h_pin);
  if (e->bath_stream) cudaStreamDestroy(e->bath_stream);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

static int flags_error(uint32_t f);
static int check_flags(dpsnn_engine *e) {
  uint32_t f = 0;
  CK(cudaMemcpyAsync(&f, e->d.flags, 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return flags_error(f);
}
static int flags_error(uint32_t f) {
  if (!f) return 0;
  if (f & F_TIME_WINDOW) return dpsnn_fail(DPSNN_E_MODEL, "ERROR in neu dynamic: input currentTime in wrong ms");
  if (f & F_NO_TARGET) return dpsnn_fail(DPSNN_E_MODEL, "ERROR neuSpikToAxSp: no forw host targ for a spiking neuron");
  if (f & F_TOO_MANY_INPUTS)
    return dpsnn_fail(DPSNN_E_CAPACITY, "more than %d synaptic inputs on one neuron in one step", MAX_INPUTS_PER_STEP);
  if (f & F_OVERFLOW) return dpsnn_fail(DPSNN_E_CAPACITY, "event overflow list full");
  if (f & F_BATH_DRAWS) return dpsnn_fail(DPSNN_E_CAPACITY, "bath draw buffer exhausted");
  return dpsnn_fail(DPSNN_E_MODEL, "device error flags 0x%x", f);
}

// Kernel timing records an event pair per kernel family and step on the
// engine stream without synchronising; dpsnn_kernel_times reads them.
static cudaEvent_t pool_event(dpsnn_engine *e) {
  if (e->event_pool.empty()) {
    cudaEvent_t ev;
    cudaEventCreate(&ev);
    return ev;
  }
  cudaEvent_t ev = e->event_pool.back();
  e->event_pool.pop_back();
  return ev;
}
static void timed_launch_begin(dpsnn_engine *e, int k, cudaStream_t st = nullptr) {
  if (!e->timing) return;
  dpsnn_engine::TimedLaunch tl;
  tl.family = k;
  tl.a = pool_event(e);
  tl.b = pool_event(e);
  tl.st = st ? st : e->stream;
  cudaEventRecord(tl.a, tl.st);
  e->pending.push_back(tl);
}
static void timed_launch_end(dpsnn_engine *e, int k) {
  if (!e->timing) return;
  (void)k;
  cudaEventRecord(e->pending.back().b, e->pending.back().st);
}
static void collect_timings(dpsnn_engine *e) {
  for (auto &tl : e->pending) {
    cudaEventSynchronize(tl.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, tl.a, tl.b);
    e->ktime[tl.family] += ms * 1e-3;
    e->klaunch[tl.family]++;
    e->event_pool.push_back(tl.a);
    e->event_pool.push_back(tl.b);
  }
  e->pending.clear();
}

// The bath of step t (bath_kernel) depends only on the ranks' RNG streams
// and nextBath, not on synaptic input, so it runs one step ahead on its own
// stream, overlapping the delivery and neuron update of the previous step.
// Its outputs (per-neuron bath events) and nextBath live in two buffers by
// step parity: bath(t) writes set t&1 once neuron(t-2), the last reader of
// that set, is done; neuron(t) reads set t&1 once bath(t) is done.
static void enqueue_bath(dpsnn_engine *e, uint32_t t) {
  Dev db = e->d;
  const int b = t & 1;
  db.nb_prev = e->nb2[b ^ 1];
  db.nb = e->nb2[b];
  db.bath_time = e->bath_time2[b];
  db.bath_lut = e->bath_lut2[b];
  db.bath_off = e->bath_off2[b];
  db.bath_cnt = e->bath_cnt2[b];
  cudaStreamWaitEvent(e->bath_stream, e->ev_neuron[b], 0);
  timed_launch_begin(e, 2, e->bath_stream);
  // the kernel reads its step from d.bath_t (baths are launched in step order)
  bath_kernel<<<e->hnet.P, BATH_THREADS, sizeof(BathSmem), e->bath_stream>>>(db);
  bath_tick_kernel<<<1, 1, 0, e->bath_stream>>>(db);
  timed_launch_end(e, 2);
  cudaEventRecord(e->ev_bath[b], e->bath_stream);
}

static int enqueue_step(dpsnn_engine *e) {
  const uint32_t t = e->t_host;
  const int b = t & 1;
  if (!e->bath_primed) {   // the first bath waits for the network build
    cudaEventRecord(e->ev_start, e->stream);
    cudaStreamWaitEvent(e->bath_stream, e->ev_start, 0);
    enqueue_bath(e, t);
    e->bath_primed = true;
    e->launches += 2;
  }
  enqueue_bath(e, t + 1);
  if (e->d.stdp_log) {
    cudaMemsetAsync(e->d.stdp_log_cnt, 0, 4, e->stream);
    e->stdp_log_t = t;
  }
  Dev d = e->d;
  d.bath_time = e->bath_time2[b];
  d.bath_lut = e->bath_lut2[b];
  d.bath_off = e->bath_off2[b];
  d.bath_cnt = e->bath_cnt2[b];
  timed_launch_begin(e, 0);
  compact_kernel<<<e->grid_neuron, NEURON_BLOCK, 0, e->stream>>>(d);
  timed_launch_end(e, 0);
  // slot t is final (inside a graph: an event the graph records on every run)
  if (e->capturing)
    cudaEventRecordWithFlags(e->ev_slot[t % RING_SLOTS], e->stream, cudaEventRecordExternal);
  else
    cudaEventRecord(e->ev_slot[t % RING_SLOTS], e->stream);
  if (e->hnet.stdp_on) {
    timed_launch_begin(e, 4);
    causal_stdp_kernel<<<e->grid_deliver, 256, 0, e->stream>>>(d);
    timed_launch_end(e, 4);
  }
  timed_launch_begin(e, 1);
  deliver_kernel<<<e->grid_deliver, DELIVER_THREADS, 0, e->stream>>>(d);
  timed_launch_end(e, 1);
  if (d.stdp_log) {
    stdp_anti_log_kernel<<<e->grid_deliver, 256, 0, e->stream>>>(d);
    e->launches++;
  }
  cudaStreamWaitEvent(e->stream, e->ev_bath[b], 0);
  timed_launch_begin(e, 3);
  neuron_kernel<<<e->grid_neuron, NEURON_BLOCK, 0, e->stream>>>(d);
  timed_launch_end(e, 3);
  timed_launch_begin(e, 5);
  heavy_sort_kernel<<<e->grid_heavy, HEAVY_SORT_THREADS, 0, e->stream>>>(d);
  heavy_sort_big_kernel<<<e->grid_heavy, HEAVY_SORT_THREADS, 0, e->stream>>>(d);
  timed_launch_end(e, 5);
  timed_launch_begin(e, 7);
  huge_kernel<<<e->grid_huge, HEAVY_THREADS, 0, e->stream>>>(d);
  timed_launch_end(e, 7);
  timed_launch_begin(e, 6);
  heavy_run_kernel<<<e->grid_heavy_run, 128, 0, e->stream>>>(d);
  timed_launch_end(e, 6);
  timed_launch_begin(e, 7);
  heavy_rest_kernel<<<e->grid_huge, 128, 0, e->stream>>>(d);
  timed_launch_end(e, 7);
  cudaEventRecord(e->ev_neuron[b], e->stream);
  if (e->hnet.stdp_on) {
    if (d.probe_w && t % 1000 == 999 && t >= e->hnet.start_pl && t <= e->hnet.stop_pl) e->probe_t = t;
    timed_launch_begin(e, 4);
    ltp_kernel<<<e->grid_deliver, 256, 0, e->stream>>>(d);
    timed_launch_end(e, 4);
  }
  end_step_kernel<<<1, 1, 0, e->stream>>>(d);
  e->launches += 11 + (e->hnet.stdp_on ? 2 : 0);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return dpsnn_fail(DPSNN_E_CUDA, "kernel launch: %s", cudaGetErrorString(err));
  e->t_host++;
  return 0;
}

extern "C" int dpsnn_step(dpsnn_engine *e, uint32_t nsteps) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  cudaSetDevice(e->device);
  for (uint32_t k = 0; k < nsteps; k++) {
    int rc = enqueue_step(e);
    if (rc) return rc;
  }
  return 0;
}

extern "C" int dpsnn_step_many(dpsnn_engine *const *engines, uint32_t n, uint32_t nsteps) {
  if (!engines && n) return dpsnn_fail(DPSNN_E_PARAM, "null engine array");
  for (uint32_t i = 0; i < n; i++)
    if (!engines[i]) return dpsnn_fail(DPSNN_E_PARAM, "null engine %u", i);
  // one step of every engine in turn: each engine's kernels queue on its own
  // streams, so the networks' steps overlap on the device
  for (uint32_t k = 0; k < nsteps; k++)
    for (uint32_t i = 0; i < n; i++) {
      dpsnn_engine *e = engines[i];
      cudaSetDevice(e->device);
      int rc = enqueue_step(e);
      if (rc) return rc;
    }
  return 0;
}

// ------------------------------------------------------------------ graphs of batched steps
// nsteps steps of n engines queued as dpsnn_step_many does, recorded once into
// a CUDA graph and run as one launch: the host cost of a step of many small
// networks (a dozen launches and event operations per network) is paid once.
// A graph encodes the engines' ring slots and step parities, so it runs only
// when every engine is at the step (mod 80) it was recorded at; nsteps is a
// multiple of 80, so consecutive runs chain.
// The events that order an engine's two streams between steps, recorded at
// the streams' current ends: after a graph run (whose own copies of them are
// internal to the graph) later steps wait on everything before.
static void rearm_step_events(dpsnn_engine *e) {
  for (int b = 0; b < 2; b++) {
    cudaEventRecord(e->ev_neuron[b], e->stream);
    cudaEventRecord(e->ev_bath[b], e->bath_stream);
  }
}

struct dpsnn_graph {
  std::vector<dpsnn_engine *> engines;
  std::vector<uint32_t> t0;        // each engine's step (mod RING_SLOTS) at recording
  std::vector<cudaEvent_t> pre;    // per engine: its two streams' last work before a run
  uint32_t nsteps = 0;
  uint64_t launches_per_run = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
};

extern "C" void dpsnn_graph_destroy(dpsnn_graph *g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (cudaEvent_t ev : g->pre) cudaEventDestroy(ev);
  if (g->fork) cudaEventDestroy(g->fork);
  if (g->done) cudaEventDestroy(g->done);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

extern "C" int dpsnn_graph_create(dpsnn_engine *const *engines, uint32_t n, uint32_t nsteps, dpsnn_graph **out) {
  if (!out || (!engines && n)) return dpsnn_fail(DPSNN_E_PARAM, "null argument");
  *out = nullptr;
  if (n == 0 || nsteps == 0 || nsteps % RING_SLOTS)
    return dpsnn_fail(DPSNN_E_PARAM, "a graph holds a positive multiple of %d steps of at least one engine",
                      RING_SLOTS);
  for (uint32_t i = 0; i < n; i++) {
    const dpsnn_engine *e = engines[i];
    if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine %u", i);
    if (e->device != engines[0]->device) return dpsnn_fail(DPSNN_E_PARAM, "engines on different devices");
    if (!e->bath_primed) return dpsnn_fail(DPSNN_E_STATE, "engine %u has not run its first step", i);
    if (e->timing || e->d.stdp_log || e->d.probe_w)
      return dpsnn_fail(DPSNN_E_STATE, "engine %u has kernel timing, the STDP event log or the LTP probe on", i);
    for (uint32_t k = 0; k < i; k++)
      if (engines[k] == e) return dpsnn_fail(DPSNN_E_PARAM, "engine %u is listed twice", i);
  }
  dpsnn_graph *g = new dpsnn_graph();
  g->device = engines[0]->device;
  g->nsteps = nsteps;
  g->engines.assign(engines, engines + n);
  cudaSetDevice(g->device);
  auto fail = [&](int rc) {
    dpsnn_graph_destroy(g);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming) != cudaSuccess)
    return fail(dpsnn_fail(DPSNN_E_CUDA, "cannot create the graph's stream and events"));
  g->pre.resize(2 * n, nullptr);
  for (auto &ev : g->pre)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      return fail(dpsnn_fail(DPSNN_E_CUDA, "cannot create the graph's events"));
  std::vector<uint32_t> t_saved(n);
  std::vector<uint64_t> l_saved(n);
  cudaError_t err = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return fail(dpsnn_fail(DPSNN_E_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(err)));
  cudaEventRecord(g->fork, g->stream);
  int rc = 0;
  for (uint32_t i = 0; i < n; i++) {
    dpsnn_engine *e = engines[i];
    t_saved[i] = e->t_host;
    l_saved[i] = e->launches;
    g->t0.push_back(e->t_host % RING_SLOTS);
    // both streams join the recording; the events they wait on between
    // each other are recorded inside it from here on
    cudaStreamWaitEvent(e->stream, g->fork, 0);
    cudaStreamWaitEvent(e->bath_stream, g->fork, 0);
    for (int b = 0; b < 2; b++) {
      cudaEventRecord(e->ev_neuron[b], e->stream);
      cudaEventRecord(e->ev_bath[b], e->bath_stream);
    }
    e->capturing = true;
  }
  for (uint32_t k = 0; k < nsteps && !rc; k++)
    for (uint32_t i = 0; i < n && !rc; i++) rc = enqueue_step(engines[i]);
  for (uint32_t i = 0; i < n; i++) {
    dpsnn_engine *e = engines[i];
    e->capturing = false;
    cudaEventRecord(g->pre[2 * i], e->stream);
    cudaEventRecord(g->pre[2 * i + 1], e->bath_stream);
    cudaStreamWaitEvent(g->stream, g->pre[2 * i], 0);
    cudaStreamWaitEvent(g->stream, g->pre[2 * i + 1], 0);
    g->launches_per_run += e->launches - l_saved[i];
    e->t_host = t_saved[i];   // nothing ran
    e->launches = l_saved[i];
  }
  err = cudaStreamEndCapture(g->stream, &g->graph);
  // the streams' order events were last recorded inside the capture: record
  // them again outside it, so that plain steps can wait on them (no step ran)
  for (uint32_t i = 0; i < n; i++) rearm_step_events(engines[i]);
  if (rc) return fail(rc);
  if (err != cudaSuccess) return fail(dpsnn_fail(DPSNN_E_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(err)));
  err = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (err != cudaSuccess) return fail(dpsnn_fail(DPSNN_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(err)));
  *out = g;
  return 0;
}

extern "C" int dpsnn_graph_run(dpsnn_graph *g) {
  if (!g) return dpsnn_fail(DPSNN_E_PARAM, "null graph");
  cudaSetDevice(g->device);
  const uint32_t n = (uint32_t)g->engines.size();
  for (uint32_t i = 0; i < n; i++)
    if (g->engines[i]->t_host % RING_SLOTS != g->t0[i])
      return dpsnn_fail(DPSNN_E_STATE, "engine %u is at step %u; the graph was recorded at a step = %u (mod %d)", i,
                        g->engines[i]->t_host, g->t0[i], RING_SLOTS);
  for (uint32_t i = 0; i < n; i++) {   // after the engines' queued work
    dpsnn_engine *e = g->engines[i];
    CK(cudaEventRecord(g->pre[2 * i], e->stream));
    CK(cudaEventRecord(g->pre[2 * i + 1], e->bath_stream));
    CK(cudaStreamWaitEvent(g->stream, g->pre[2 * i], 0));
    CK(cudaStreamWaitEvent(g->stream, g->pre[2 * i + 1], 0));
  }
  CK(cudaGraphLaunch(g->exec, g->stream));
  CK(cudaEventRecord(g->done, g->stream));
  for (uint32_t i = 0; i < n; i++) {   // later work on the engines' streams follows the graph
    dpsnn_engine *e = g->engines[i];
    CK(cudaStreamWaitEvent(e->stream, g->done, 0));
    CK(cudaStreamWaitEvent(e->bath_stream, g->done, 0));
    rearm_step_events(e);
    e->t_host += g->nsteps;
  }
  g->engines[0]->launches += g->launches_per_run;   // counted on the first engine
  return 0;
}

extern "C" int dpsnn_set_launch_shape(dpsnn_engine *e, uint32_t deliver_blocks, uint32_t heavy_sort_blocks,
                                      uint32_t heavy_run_blocks) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  const uint32_t lim = 1u << 20;
  if (deliver_blocks > lim || heavy_sort_blocks > lim || heavy_run_blocks > lim)
    return dpsnn_fail(DPSNN_E_PARAM, "a grid of more than %u blocks", lim);
  e->grid_deliver = deliver_blocks ? deliver_blocks : (uint32_t)e->sms * 8;
  e->grid_heavy = heavy_sort_blocks ? heavy_sort_blocks : (uint32_t)e->sms * 8;
  e->grid_heavy_run = heavy_run_blocks ? heavy_run_blocks : (uint32_t)e->sms * 16;
  return 0;
}

extern "C" int dpsnn_sync(dpsnn_engine *e) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  cudaSetDevice(e->device);
  CK(cudaStreamSynchronize(e->stream));
  return check_flags(e);
}

extern "C" uint32_t dpsnn_glob_n(const dpsnn_engine *e) { return e ? e->hnet.N : 0; }
extern "C" uint32_t dpsnn_time_ms(const dpsnn_engine *e) { return e ? e->t_host : 0; }
extern "C" uint64_t dpsnn_synapse_count(const dpsnn_engine *e) { return e ? e->S : 0; }
extern "C" uint64_t dpsnn_events_delivered(const dpsnn_engine *e) {
  if (!e) return 0;
  unsigned long long v = 0;
  cudaSetDevice(e->device);
  cudaMemcpyAsync(&v, e->d.events, 8, cudaMemcpyDeviceToHost, e->stream);
  cudaStreamSynchronize(e->stream);
  return v;
}

extern "C" int dpsnn_spikes(dpsnn_engine *e, uint32_t t_ms, uint32_t *ids, double *te, uint32_t cap,
                            uint32_t *count) {
  if (!e || !count) return dpsnn_fail(DPSNN_E_PARAM, "null argument");
  if (t_ms >= e->t_host || t_ms + RING_SLOTS < e->t_host)
    return dpsnn_fail(DPSNN_E_STATE, "step %u is not among the last %d completed steps", t_ms, RING_SLOTS);
  cudaSetDevice(e->device);
  const uint32_t slot = t_ms % RING_SLOTS;
  // wait only for the compaction of step t_ms (the rest of that step and
  // later steps may still run): one round trip for the error flags and the
  // count, one for the list
  CK(cudaStreamWaitEvent(e->read_stream, e->ev_slot[slot], 0));
  CK(cudaMemcpyAsync(e->h_pin, e->d.flags, 4, cudaMemcpyDeviceToHost, e->read_stream));
  CK(cudaMemcpyAsync(e->h_pin + 1, e->d.ring_cnt + slot, 4, cudaMemcpyDeviceToHost, e->read_stream));
  CK(cudaStreamSynchronize(e->read_stream));
  int rc = flags_error(e->h_pin[0]);
  if (rc) return rc;
  const uint32_t cnt = e->h_pin[1];
  *count = cnt;
  const uint32_t k = std::min(cnt, cap);
  if (k && ids)
    CK(cudaMemcpyAsync(ids, e->d.ring_ids + (size_t)slot * e->hnet.N, 4ull * k, cudaMemcpyDeviceToHost,
                       e->read_stream));
  if (k && te)
    CK(cudaMemcpyAsync(te, e->d.ring_te + (size_t)slot * e->hnet.N, 8ull * k, cudaMemcpyDeviceToHost,
                       e->read_stream));
  if (k && (ids || te)) CK(cudaStreamSynchronize(e->read_stream));
  return 0;
}

extern "C" int dpsnn_spikes_range(dpsnn_engine *e, uint32_t t0, uint32_t n, uint32_t *ids, double *te,
                                  uint64_t cap, uint32_t *counts) {
  if (!e || !counts || (n && (!ids || !te))) return dpsnn_fail(DPSNN_E_PARAM, "null argument");
  if (n == 0) return 0;
  if (n > RING_SLOTS || t0 + n > e->t_host || t0 + RING_SLOTS < e->t_host)
    return dpsnn_fail(DPSNN_E_STATE, "steps %u..%u are not among the last %d completed steps", t0, t0 + n - 1,
                      RING_SLOTS);
  cudaSetDevice(e->device);
  // after the compaction of the last step of the run (steps complete in
  // order on the engine stream): the counts and the error flags, then the lists
  CK(cudaStreamWaitEvent(e->read_stream, e->ev_slot[(t0 + n - 1) % RING_SLOTS], 0));
  CK(cudaMemcpyAsync(e->h_pin, e->d.flags, 4, cudaMemcpyDeviceToHost, e->read_stream));
  for (uint32_t k = 0; k < n; k++)
    CK(cudaMemcpyAsync(counts + k, e->d.ring_cnt + (t0 + k) % RING_SLOTS, 4, cudaMemcpyDeviceToHost,
                       e->read_stream));
  CK(cudaStreamSynchronize(e->read_stream));
  int rc = flags_error(e->h_pin[0]);
  if (rc) return rc;
  uint64_t off = 0;
  for (uint32_t k = 0; k < n; k++) off += counts[k];
  if (off > cap) return dpsnn_fail(DPSNN_E_CAPACITY, "%llu spikes in steps %u..%u exceed the buffers (%llu)",
                                   (unsigned long long)off, t0, t0 + n - 1, (unsigned long long)cap);
  off = 0;
  for (uint32_t k = 0; k < n; k++) {
    const size_t slot = (t0 + k) % RING_SLOTS;
    if (counts[k]) {
      CK(cudaMemcpyAsync(ids + off, e->d.ring_ids + slot * e->hnet.N, 4ull * counts[k], cudaMemcpyDeviceToHost,
                         e->read_stream));
      CK(cudaMemcpyAsync(te + off, e->d.ring_te + slot * e->hnet.N, 8ull * counts[k], cudaMemcpyDeviceToHost,
                         e->read_stream));
    }
    off += counts[k];
  }
  CK(cudaStreamSynchronize(e->read_stream));
  return 0;
}

extern "C" uint64_t dpsnn_device_bytes(const dpsnn_engine *e) { return e ? e->bytes : 0; }

extern "C" int dpsnn_state(dpsnn_engine *e, double *v, double *c, double *tr, double *te, double *nb) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  int rc = dpsnn_sync(e);
  if (rc) return rc;
  size_t B = 8ull * e->hnet.N;
  if (v) CK(cudaMemcpy(v, e->d.v, B, cudaMemcpyDeviceToHost));
  if (c) CK(cudaMemcpy(c, e->d.c, B, cudaMemcpyDeviceToHost));
  if (tr) CK(cudaMemcpy(tr, e->d.tr, B, cudaMemcpyDeviceToHost));
  if (te) CK(cudaMemcpy(te, e->d.te, B, cudaMemcpyDeviceToHost));
  // nextBath after the last completed step (the bath of the next step may
  // already have run into the other buffer)
  if (nb) CK(cudaMemcpy(nb, e->nb2[e->t_host ? (e->t_host - 1) & 1 : 1], B, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int dpsnn_bath_params(dpsnn_engine *e, double *inv_nu_ext, uint32_t *max_ext) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  int rc = dpsnn_sync(e);
  if (rc) return rc;
  if (inv_nu_ext) CK(cudaMemcpy(inv_nu_ext, e->d.inv_nu, 8ull * e->hnet.N, cudaMemcpyDeviceToHost));
  if (max_ext) CK(cudaMemcpy(max_ext, e->d.max_ext, 4ull * e->hnet.N, cudaMemcpyDeviceToHost));
  return 0;
}

// Host-side view of the connectome for the reference-order backward list.
struct HostCsr {
  std::vector<uint64_t> row;
  std::vector<uint16_t> so;
  std::vector<uint32_t> post;
  std::vector<int16_t> w;
  std::vector<float> td;
  std::vector<uint8_t> sub;
};
static int fetch_csr(dpsnn_engine *e, HostCsr &h, bool with_td) {
  int rc = dpsnn_sync(e);
  if (rc) return rc;
  const uint32_t N = e->hnet.N, D = e->hnet.D;
  h.row.resize(N + 1);
  h.so.resize((size_t)N * (D + 1));
  h.post.resize(e->S);
  h.w.resize(e->S);
  h.sub.resize(N);
  CK(cudaMemcpy(h.row.data(), e->d.row_ptr, 8ull * (N + 1), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.so.data(), e->d.sub_off, 2ull * N * (D + 1), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.post.data(), e->d.post, 4ull * e->S, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.w.data(), e->d.w16, 2ull * e->S, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.sub.data(), e->d.sub, N, cudaMemcpyDeviceToHost));
  if (with_td && e->d.tderiv) {
    h.td.resize(e->S);
    CK(cudaMemcpy(h.td.data(), e->d.tderiv, 4ull * e->S, cudaMemcpyDeviceToHost));
  }
  return 0;
}

extern "C" uint64_t dpsnn_rank_synapse_count(dpsnn_engine *e, uint32_t h) {
  if (!e || h >= e->hnet.P) return 0;
  HostCsr c;
  if (fetch_csr(e, c, false)) return 0;
  uint64_t n = 0;
  for (uint64_t k = 0; k < e->S; k++) n += (c.post[k] / e->hnet.locN == h);
  return n;
}

extern "C" int dpsnn_backward_synapses(dpsnn_engine *e, uint32_t h, uint32_t *pre, uint32_t *post, uint8_t *delay,
                                       uint8_t *kind, int16_t *weight, float *tderiv) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  if (h >= e->hnet.P) return dpsnn_fail(DPSNN_E_PARAM, "rank %u out of range", h);
  HostCsr c;
  int rc = fetch_csr(e, c, tderiv != nullptr);
  if (rc) return rc;
  // reference order (inflateIntermToBackwardSynList): delay, then source
  // rank / presynaptic index, then generation order
  const uint32_t N = e->hnet.N, D = e->hnet.D, locN = e->hnet.locN;
  uint64_t o = 0;
  for (uint32_t dl = 0; dl < D; dl++)
    for (uint32_t P = 0; P < N; P++) {
      uint64_t b = c.row[P] + c.so[(size_t)P * (D + 1) + dl], en = c.row[P] + c.so[(size_t)P * (D + 1) + dl + 1];
      for (uint64_t k = b; k < en; k++) {
        if (c.post[k] / locN != h) continue;
        if (pre) pre[o] = P;
        if (post) post[o] = c.post[k];
        if (delay) delay[o] = (uint8_t)dl;
        if (kind) kind[o] = c.sub[P];
        if (weight) weight[o] = c.w[k];
        if (tderiv) tderiv[o] = c.td.empty() ? 0.0f : c.td[k];
        o++;
      }
    }
  return 0;
}

extern "C" int dpsnn_enable_ltp_probe(dpsnn_engine *e) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  if (!e->hnet.stdp_on) return dpsnn_fail(DPSNN_E_PARAM, "the LTP probe needs plasticity switched on");
  if (e->d.probe_w) return 0;
  if (e->t_host) return dpsnn_fail(DPSNN_E_PARAM, "the LTP probe is enabled before the first step");
  cudaSetDevice(e->device);
  DALLOC(e->d.probe_w, e->S);
  DALLOC(e->d.probe_td, e->S);
  DALLOC(e->d.probe_td_mid, e->S);
  return 0;
}

extern "C" int dpsnn_ltp_probe(dpsnn_engine *e, uint32_t h, uint32_t *t_ms, int16_t *w_before, float *td_before,
                               int16_t *w_after, float *td_after) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  if (h >= e->hnet.P) return dpsnn_fail(DPSNN_E_PARAM, "rank %u out of range", h);
  if (!e->d.probe_w) return dpsnn_fail(DPSNN_E_PARAM, "the LTP probe is not enabled");
  if (e->probe_t == UINT32_MAX) return dpsnn_fail(DPSNN_E_PARAM, "no plasticity update has run yet");
  HostCsr c;
  int rc = fetch_csr(e, c, false);   // synchronises: the probe and the weights are final
  if (rc) return rc;
  std::vector<int16_t> pw(e->S);
  std::vector<float> pt(e->S), pm(e->S);
  CK(cudaMemcpy(pw.data(), e->d.probe_w, 2ull * e->S, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(pt.data(), e->d.probe_td, 4ull * e->S, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(pm.data(), e->d.probe_td_mid, 4ull * e->S, cudaMemcpyDeviceToHost));
  if (t_ms) *t_ms = e->probe_t;
  // the order of dpsnn_backward_synapses; the weights change only at an LTP
  // update, so the live weights are those the last update wrote
  const uint32_t N = e->hnet.N, D = e->hnet.D, locN = e->hnet.locN;
  uint64_t o = 0;
  for (uint32_t dl = 0; dl < D; dl++)
    for (uint32_t P = 0; P < N; P++) {
      uint64_t b = c.row[P] + c.so[(size_t)P * (D + 1) + dl], en = c.row[P] + c.so[(size_t)P * (D + 1) + dl + 1];
      for (uint64_t k = b; k < en; k++) {
        if (c.post[k] / locN != h) continue;
        if (w_before) w_before[o] = pw[k];
        if (td_before) td_before[o] = pt[k];
        if (w_after) w_after[o] = c.w[k];
        if (td_after) td_after[o] = pm[k];
        o++;
      }
    }
  return 0;
}

extern "C" int dpsnn_enable_stdp_events(dpsnn_engine *e) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  if (!e->hnet.stdp_on) return dpsnn_fail(DPSNN_E_PARAM, "the STDP event log needs plasticity switched on");
  if (e->d.stdp_log) return 0;
  if (e->t_host) return dpsnn_fail(DPSNN_E_PARAM, "the STDP event log is enabled before the first step");
  cudaSetDevice(e->device);
  HostCsr c;
  int rc = fetch_csr(e, c, false);
  if (rc) return rc;
  e->h_row = std::move(c.row);
  e->h_so = std::move(c.so);
  DALLOC(e->d.stdp_log, STDP_LOG_CAP);
  DALLOC(e->d.stdp_log_cnt, 1);
  return 0;
}

extern "C" int dpsnn_stdp_events(dpsnn_engine *e, uint32_t *t_ms, uint32_t *pre, uint32_t *post, float *contribution,
                                 uint32_t cap, uint32_t *count) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  if (!e->d.stdp_log) return dpsnn_fail(DPSNN_E_PARAM, "the STDP event log is not enabled");
  if (e->stdp_log_t == UINT32_MAX) return dpsnn_fail(DPSNN_E_PARAM, "no step has run yet");
  int rc = dpsnn_sync(e);   // also reports a full log (DPSNN_E_CAPACITY)
  if (rc) return rc;
  uint32_t n = 0;
  CK(cudaMemcpy(&n, e->d.stdp_log_cnt, 4, cudaMemcpyDeviceToHost));
  if (n > STDP_LOG_CAP) return dpsnn_fail(DPSNN_E_CAPACITY, "more than %u STDP events in one step", STDP_LOG_CAP);
  std::vector<uint4> rec(n);
  if (n) CK(cudaMemcpy(rec.data(), e->d.stdp_log, 16ull * n, cudaMemcpyDeviceToHost));
  // presynaptic neuron and delay of each record's synapse from the CSR, then
  // the reference's order: causal events (detection, ascending post, each
  // post's synapses in backward-list order: delay, then presynaptic neuron,
  // then generation order), then anti-causal events (delivery: delay
  // descending, then presynaptic neuron, then generation order)
  const uint32_t D = e->hnet.D;
  struct Ev {
    uint64_t key0, key1;
    uint32_t pre, post;
    float c;
  };
  std::vector<Ev> ev(n);
  for (uint32_t i = 0; i < n; i++) {
    const uint64_t k = (uint64_t)rec[i].x | ((uint64_t)rec[i].y << 32);
    const uint32_t P = (uint32_t)(std::upper_bound(e->h_row.begin(), e->h_row.end(), k) - e->h_row.begin()) - 1;
    uint32_t dl = 0;
    while (dl + 1 < D && e->h_row[P] + e->h_so[(size_t)P * (D + 1) + dl + 1] <= k) dl++;
    const uint32_t j = rec[i].z & 0x7fffffffu, anti = rec[i].z >> 31;
    Ev &v = ev[i];
    v.pre = P;
    v.post = j;
    memcpy(&v.c, &rec[i].w, 4);
    if (anti) {
      v.key0 = (1ull << 63) | (uint64_t)(D - 1 - dl);
    } else {
      v.key0 = ((uint64_t)j << 8) | dl;
    }
    v.key1 = k;
  }
  std::sort(ev.begin(), ev.end(), [](const Ev &a, const Ev &b) {
    return a.key0 != b.key0 ? a.key0 < b.key0 : a.key1 < b.key1;
  });
  if (t_ms) *t_ms = e->stdp_log_t;
  if (count) *count = n;
  const uint32_t m = std::min(n, cap);
  for (uint32_t i = 0; i < m; i++) {
    if (pre) pre[i] = ev[i].pre;
    if (post) post[i] = ev[i].post;
    if (contribution) contribution[i] = ev[i].c;
  }
  return 0;
}

extern "C" int dpsnn_set_timing(dpsnn_engine *e, int enable) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  e->timing = enable;
  return 0;
}

extern "C" uint64_t dpsnn_kernel_launches(const dpsnn_engine *e) { return e ? e->launches : 0; }
extern "C" void *dpsnn_cuda_stream(const dpsnn_engine *e) { return e ? (void *)e->stream : nullptr; }

extern "C" int dpsnn_kernel_times(dpsnn_engine *e, double *seconds, uint64_t *launches) {
  if (!e) return dpsnn_fail(DPSNN_E_PARAM, "null engine");
  cudaSetDevice(e->device);
  collect_timings(e);
  for (int k = 0; k < DPSNN_TIMING_SLOTS; k++) {
    if (seconds) seconds[k] = e->ktime[k];
    if (launches) launches[k] = e->klaunch[k];
  }
  return 0;
}

// ------------------------------------------------------------------ no-allocation rank spike read
// dpsnn_rank_spikes_noalloc: the spike list of one emulated rank at one step,
// gathered on the device into a fixed scratch area that is part of the
// library image (no cudaMalloc/cudaFree on this path), then copied to the
// caller's host buffers.  The scratch holds DPSNN_NOALLOC_MAX_SPIKES spikes,
// the reference's largest rank (miniLocN = 32000 neurons) rounded up; ranks
// with more neurons are rejected.  One scratch per device and process: calls
// that overlap in time on the same device race on it.
struct NoAllocScratch {
  uint32_t count;                            // written by the kernel each call
  uint32_t pad[63];
  uint32_t ids[DPSNN_NOALLOC_MAX_SPIKES];
  double te[DPSNN_NOALLOC_MAX_SPIKES];
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// One block: binary search of the rank's neuron range [lo, hi) in the
// ascending spike list of the slot, then an ordered copy of that range.
// Nothing in the scratch has to start at zero: count and the copied entries
// are all written here before the host reads them.
__global__ void rank_select_kernel(const uint32_t *__restrict__ ids, const double *__restrict__ te,
                                   const uint32_t *__restrict__ cnt_ptr, uint32_t lo, uint32_t hi,
                                   NoAllocScratch *__restrict__ out) {
  __shared__ uint32_t s_a, s_b;
  const uint32_t cnt = *cnt_ptr;
  if (threadIdx.x == 0) {
    uint32_t a = 0, b = cnt;
    while (a < b) {
      const uint32_t m = (a + b) >> 1;
      if (ids[m] < lo) a = m + 1; else b = m;
    }
    uint32_t c = a, d = cnt;
    while (c < d) {
      const uint32_t m = (c + d) >> 1;
      if (ids[m] < hi) c = m + 1; else d = m;
    }
    s_a = a;
    s_b = c;
    out->count = c - a;
  }
  __syncthreads();
  const uint32_t a = s_a, n = min(s_b - s_a, (uint32_t)DPSNN_NOALLOC_MAX_SPIKES);
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    out->ids[k] = ids[a + k];
    out->te[k] = te[a + k];
  }
}

#define DPSNN_NOALLOC_MAX_DEVICES 64
static std::mutex g_noalloc_mu;
static NoAllocScratch *g_noalloc_addr[DPSNN_NOALLOC_MAX_DEVICES];

// Device address of the scratch, looked up once per device.
static int noalloc_scratch(int device, NoAllocScratch **out) {
  if (device < 0 || device >= DPSNN_NOALLOC_MAX_DEVICES)
    return dpsnn_fail(DPSNN_E_PARAM, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess)
      return dpsnn_fail(DPSNN_E_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(err));
    g_noalloc_addr[device] = (NoAllocScratch *)p;
  }
  *out = g_noalloc_addr[device];
  return 0;
}

extern "C" int dpsnn_rank_spikes_noalloc(dpsnn_engine *e, uint32_t t_ms, uint32_t h, uint32_t *ids, double *te,
                                         uint32_t cap, uint32_t *count) {
  if (!e || !count) return dpsnn_fail(DPSNN_E_PARAM, "null argument");
  if (h >= e->hnet.P) return dpsnn_fail(DPSNN_E_PARAM, "rank %u out of range (env_globH = %u)", h, e->hnet.P);
  if (e->hnet.locN > DPSNN_NOALLOC_MAX_SPIKES)
    return dpsnn_fail(DPSNN_E_CAPACITY, "rank of %u neurons exceeds the %d-spike scratch of dpsnn_rank_spikes_noalloc",
                      e->hnet.locN, DPSNN_NOALLOC_MAX_SPIKES);
  if (t_ms >= e->t_host || t_ms + RING_SLOTS < e->t_host)
    return dpsnn_fail(DPSNN_E_STATE, "step %u is not among the last %d completed steps", t_ms, RING_SLOTS);
  cudaSetDevice(e->device);
  NoAllocScratch *s = nullptr;
  int rc = noalloc_scratch(e->device, &s);
  if (rc) return rc;
  const uint32_t slot = t_ms % RING_SLOTS;
  const size_t off = (size_t)slot * e->hnet.N;
  // on the read stream, after the compaction of step t_ms only (as
  // dpsnn_spikes): later steps keep running on the engine stream
  CK(cudaStreamWaitEvent(e->read_stream, e->ev_slot[slot], 0));
  rank_select_kernel<<<1, 256, 0, e->read_stream>>>(e->d.ring_ids + off, e->d.ring_te + off, e->d.ring_cnt + slot,
                                                    h * e->hnet.locN, (h + 1) * e->hnet.locN, s);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(e->h_pin, e->d.flags, 4, cudaMemcpyDeviceToHost, e->read_stream));
  CK(cudaMemcpyAsync(e->h_pin + 1, &s->count, 4, cudaMemcpyDeviceToHost, e->read_stream));
  CK(cudaStreamSynchronize(e->read_stream));
  rc = flags_error(e->h_pin[0]);
  if (rc) return rc;
  const uint32_t n = e->h_pin[1];
  *count = n;
  const uint32_t k = std::min(n, cap);
  if (k && ids) CK(cudaMemcpyAsync(ids, s->ids, 4ull * k, cudaMemcpyDeviceToHost, e->read_stream));
  if (k && te) CK(cudaMemcpyAsync(te, s->te, 8ull * k, cudaMemcpyDeviceToHost, e->read_stream));
  if (k && (ids || te)) CK(cudaStreamSynchronize(e->read_stream));
  return 0;
}
