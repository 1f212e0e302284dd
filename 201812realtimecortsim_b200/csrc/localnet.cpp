// localnet.cpp -- the DAL process trio of DPSNN over the B200 engine, and
// the reference's per-rank output files (spikes, ratesPerPop,
// FiringsInChronoWindow) written from the engine's spike lists, and the
// synapse periodic probe files (synPeriodicProbe_A/B, DPSNN_stat.c:429-449)
// written from the engine's LTP probe, and the STDP event files (STDPevent,
// DPSNN_stat.c:451-477) written from the engine's STDP event log.
//
// Output formats restate DPSNN_stat.c (file names :66-83, spikes :290-308,
// ratesPerPop :227-275, open/close windows :594-745) and
// DPSNN_localNet_sim.c (per-population counts :229-253, chrono window
// statistics :1001-1036).  The stopWatch semantics are those of
// DPSNN_stopWatch.c:15-44.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dpsnn_b200.h"
#include "dpsnn_localnet.h"

namespace {

[[noreturn]] void die(const char *what) {
  printf("ERROR %s: %s\n", what, dpsnn_last_error());
  fflush(stdout);
  exit(0);  // the reference exits with status 0 on every error
}

// One emulated rank's stat files and chrono-window counters.
struct RankStat {
  FILE *spikes = nullptr, *rates = nullptr;
  std::vector<uint32_t> per_pop;   // N_firingsPerPop (globCFT*nsub entries)
  uint32_t n_win = 0, min_win = (uint32_t)-1, max_win = 0, laps = 0;
  double mean = 0, var = 0, sigma = 0, cv = 0, m2 = 0;
};

struct LocalNet {
  dpsnn_params par;
  dpsnn_engine *eng = nullptr;
  int32_t ms = 0, max_ms = 0;
  uint32_t P = 1, locN = 0, npcm = 0, globCFT = 0;
  float locCFT = 1.0f;
  uint32_t chrono = 0, chrono_start = 0, chrono_stop = 0;
  std::vector<RankStat> rank;
  std::vector<uint32_t> ids;
  std::vector<double> te;
  // synapse periodic probe (rank 0 only): files, window, and rank 0's
  // synapses with a presynaptic neuron of rank 0, as indices into its list
  bool probe = false;
  uint32_t probe_start_s = 0, probe_stop_s = 0;
  FILE *probe_a = nullptr, *probe_b = nullptr;
  std::vector<uint64_t> probe_idx;
  std::vector<uint32_t> syn_pre, syn_post;
  std::vector<uint8_t> syn_delay, syn_kind;
  // STDP event file (rank 0 only)
  bool stdp_ev = false;
  uint32_t stdp_start_s = 0, stdp_stop_s = 0, debug_ms = 0;
  FILE *stdp_f = nullptr;
  std::vector<uint32_t> ev_pre, ev_post;
  std::vector<float> ev_c;
};

LocalNet *g_net = nullptr;

bool stat_second(const dpsnn_params &p, uint32_t sec) {
  return sec >= p.startStatFiles_s && sec <= p.stopStatFiles_s && sec % p.moduloSec == 0;
}
bool rates_second(const dpsnn_params &p, uint32_t sec) {
  return stat_second(p, sec) && sec >= p.startRatesPerPop_s && sec <= p.stopRatesPerPop_s;
}

FILE *open_stat(const LocalNet &n, const char *prefix, uint32_t sec, uint32_t h) {
  char name[320];
  if (n.par.howManyOutputFiles == 1) {
    snprintf(name, sizeof name, "%s-sec%u-C%u-H%u-h%03u.dat", prefix, sec, n.globCFT, n.P, h);
  } else if (sec == 0) {
    snprintf(name, sizeof name, "%s-start-C%u-H%u-h%u.dat", prefix, n.globCFT, n.P, h);
  } else if (sec % 2 == 0) {
    snprintf(name, sizeof name, "%s-lasteven-C%u-H%u-h%u.dat", prefix, n.globCFT, n.P, h);
  } else {
    snprintf(name, sizeof name, "%s-lastodd-C%u-H%u-h%u.dat", prefix, n.globCFT, n.P, h);
  }
  FILE *f = fopen(name, "w");
  if (!f) {
    printf("ERROR NULL fp\n");
    fflush(stdout);
    exit(0);
  }
  return f;
}

void close_stat(FILE *&f) {
  if (f && fclose(f) != 0) {
    printf("ERROR fclose!=0 in stat_sfclose\n");
    fflush(stdout);
    exit(0);
  }
  f = nullptr;
}

void open_second(LocalNet &n, uint32_t sec) {
  for (uint32_t h = 0; h < n.P; h++) {
    RankStat &r = n.rank[h];
    if (!n.par.spikes_writeDisable && stat_second(n.par, sec)) r.spikes = open_stat(n, "spikes", sec, h);
    if (!n.par.statRatesPerPop_writeDisable && rates_second(n.par, sec))
      r.rates = open_stat(n, "ratesPerPop", sec, h);
  }
  if (n.probe && stat_second(n.par, sec) && sec >= n.probe_start_s && sec <= n.probe_stop_s) {
    n.probe_a = open_stat(n, "synPeriodicProbe_A", sec, 0);
    n.probe_b = open_stat(n, "synPeriodicProbe_B", sec, 0);
  }
  if (n.stdp_ev && stat_second(n.par, sec) && sec >= n.stdp_start_s && sec <= n.stdp_stop_s)
    n.stdp_f = open_stat(n, "STDPevent", sec, 0);
}

void close_second(LocalNet &n) {
  for (RankStat &r : n.rank) {
    close_stat(r.spikes);
    close_stat(r.rates);
  }
  close_stat(n.probe_a);
  close_stat(n.probe_b);
  close_stat(n.stdp_f);
}

// The STDP event lines of the step just run (statSTDPeventClass::write,
// DPSNN_stat.c:451-477), in the order the reference makes them.
void write_stdp_events(LocalNet &n) {
  uint32_t t = 0, cnt = 0;
  if (dpsnn_stdp_events(n.eng, &t, n.ev_pre.data(), n.ev_post.data(), n.ev_c.data(), (uint32_t)n.ev_pre.size(),
                        &cnt))
    die("statSTDPevent");
  if (t != (uint32_t)n.ms) {
    printf("ERROR STDP events of step %u read at step %d\n", t, n.ms);
    fflush(stdout);
    exit(0);
  }
  const uint32_t ms = (uint32_t)n.ms;
  if (n.debug_ms != 0 && !(ms >= n.debug_ms && ms <= n.debug_ms + 20)) return;
  for (uint32_t i = 0; i < cnt; i++)
    fprintf(n.stdp_f, "%8u %7d %7d %2.7f \n", ms, (int)n.ev_pre[i], (int)n.ev_post[i], n.ev_c[i]);
  fflush(n.stdp_f);
}

// The two probe files of an x999 ms step that ran the plasticity update:
// rank 0's synapses from rank-0 neurons in backward-list order, in the
// instrumentedSynapse::report format (DPSNN_synapse.h:63-80), before the
// update (A) and after it, before the decay of the time derivative (B).
void write_probe(LocalNet &n) {
  const uint64_t S = n.syn_pre.size();
  std::vector<int16_t> wb(S), wa(S);
  std::vector<float> tb(S), ta(S);
  uint32_t t = 0;
  if (dpsnn_ltp_probe(n.eng, 0, &t, wb.data(), tb.data(), wa.data(), ta.data())) die("longTermPlasticity");
  if (t != (uint32_t)n.ms) {
    printf("ERROR synapse probe of step %u read at step %d\n", t, n.ms);
    fflush(stdout);
    exit(0);
  }
  const float w2f = n.par.min_syn_weight_f / -32767;
  for (int side = 0; side < 2; side++) {
    FILE *f = side ? n.probe_b : n.probe_a;
    const int16_t *w = side ? wa.data() : wb.data();
    const float *td = side ? ta.data() : tb.data();
    for (uint64_t k : n.probe_idx) {
      fprintf(f, "%d %d %d %d %d %f ", (int)n.syn_pre[k], (int)n.syn_post[k], (int)(n.syn_post[k] / n.locN),
              (int)n.syn_delay[k], (int)n.syn_kind[k], (float)(w[k] * w2f));
      fprintf(f, "%f", td[k]);
      fprintf(f, "\n");
    }
    fflush(f);
  }
}

uint32_t subpop_in_module(const dpsnn_params &p, uint32_t in_cm) {
  uint32_t s = 0;
  while (s < p.nsub) {
    if (in_cm < p.count[s]) break;
    in_cm -= p.count[s];
    s++;
  }
  return s;
}

// The per-step outputs of one rank: its spike lines, its per-population
// counts and, every ratesSampling ms, its rate line; then the chrono window.
void rank_outputs(LocalNet &n, uint32_t h, const uint32_t *ids, const double *te, uint32_t cnt) {
  const dpsnn_params &p = n.par;
  RankStat &r = n.rank[h];
  const uint32_t ms = (uint32_t)n.ms;
  if (r.spikes)
    for (uint32_t i = 0; i < cnt; i++) {
      fprintf(r.spikes, "%d %.7g\n", (int)ids[i], te[i]);
      fflush(r.spikes);
    }
  const uint32_t first_pop = (h * n.locN / n.npcm) * p.nsub;
  for (uint32_t i = 0; i < cnt; i++) {
    const uint32_t col = ids[i] / n.npcm;
    const uint32_t pop = col * p.nsub + subpop_in_module(p, ids[i] - col * n.npcm);
    r.per_pop[pop - first_pop]++;
  }
  if (r.rates && ms % p.ratesSampling == 0) {
    fprintf(r.rates, "%d ", (int)(ms - p.ratesSampling));
    for (uint32_t tot = 0; (float)tot < n.locCFT * (float)p.nsub; tot += p.nsub)
      for (uint32_t s = 0; s < p.nsub; s++)
        fprintf(r.rates, "%.7g ",
                ((float)(r.per_pop[tot + s]) * 1000.0) / ((float)(p.count[s]) * (float)(p.ratesSampling)));
    fprintf(r.rates, " \n");
    fflush(r.rates);
    std::fill(r.per_pop.begin(), r.per_pop.end(), 0u);
  }
  if (ms >= n.chrono_start && ms < n.chrono_stop) {
    r.n_win += cnt;
    r.laps++;
    r.min_win = cnt < r.min_win ? cnt : r.min_win;
    r.max_win = cnt > r.max_win ? cnt : r.max_win;
    const double delta = cnt - r.mean;
    r.mean += (double)(delta / r.laps);
    r.m2 += (double)((double)delta * (double)((double)cnt - (double)r.mean));
    r.var = (double)(r.m2 / (r.laps - 1));
    r.sigma = (double)(sqrt(r.var));
    r.cv = (double)(r.sigma / r.mean);
  }
}

void write_chrono_window(const LocalNet &n, uint32_t h) {
  const RankStat &r = n.rank[h];
  char name[80];
  snprintf(name, sizeof name, "FiringsInChronoWindow_h%u.stat", h);
  FILE *f = fopen(name, "w");
  if (!f) return;
  const double rate = double((double)r.n_win * 1000) / double((double)r.laps * (double)n.locN);
  fprintf(f,
          "FIRING-h=%.3d     Firings in ms %6d-%6d = %-11d min = %-11d max = %-11d mean = %-11f variance = "
          "%-11f sigma = %-11f coeffOfVariation = %-11f samples = %d\n",
          (int)h, (int)n.chrono_start, (int)n.chrono_stop, (int)r.n_win, (int)r.min_win, (int)r.max_win, r.mean,
          r.var, r.sigma, r.cv, (int)r.laps);
  fprintf(f, "FIRING-h=%.3d  FiringRate in ms %6d-%6d = %-11f\n", (int)h, (int)n.chrono_start,
          (int)n.chrono_stop, rate);
  fclose(f);
}

// The Perseo .ini description of each rank's modules (writeIniFiles,
// DPSNN_writeIniFiles.c:31-158; the reference compiles the call out of its
// stock build, DPSNN_localNet_init.c:245-247): PerseoConFile_h<h>.txt with one
// line per (source population, target population, stencil cell) of non-zero
// connection probability, PerseoModFile_h<h>.txt with one line per local
// sub-population.  Connection probabilities mirror the explicit stencil
// (DPSNN_LIFCAconnectome.cpp); the bath efficacy is generateSourceNeuCExt
// (:871-887).
void write_ini_files(const LocalNet &n) {
  const dpsnn_params &p = n.par;
  const uint32_t S = p.stencil_dim, st = 2 * S - 1, M = S - 1, nsub = p.nsub;
  if (floorf(n.locCFT) != n.locCFT) return;
  const uint32_t lcft = (uint32_t)floorf(n.locCFT);
  auto prob = [&](uint32_t s, uint32_t t, uint32_t x, uint32_t y) -> float {
    const uint32_t dx = x >= M ? x - M : M - x, dy = y >= M ? y - M : M - y;
    return p.spec[((size_t)(s * nsub + t) * S + dx) * S + dy];
  };
  for (uint32_t h = 0; h < n.P; h++) {
    char fc[40], fm[40];
    snprintf(fc, sizeof fc, "PerseoConFile_h%u.txt", h);
    snprintf(fm, sizeof fm, "PerseoModFile_h%u.txt", h);
    FILE *fpc = fopen(fc, "w"), *fpm = fopen(fm, "w");
    if (!fpc || !fpm) {
      printf("ERROR NULL fp\n");
      fflush(stdout);
      exit(0);
    }
    const uint32_t first = h * n.locN, last = first + n.locN - 1;
    const uint32_t fx = (first / n.npcm) % p.cfx, fy = (first / n.npcm) / p.cfx;
    const uint32_t lx = (last / n.npcm) % p.cfx, ly = (last / n.npcm) / p.cfx;
    for (uint32_t cx = fx; cx <= lx; cx++)
      for (uint32_t cy = fy; cy <= ly; cy++) {
        const uint32_t this_cf = cx + cy * p.cfx, loc_cf = this_cf % lcft;
        const uint32_t src_cf = loc_cf + lcft * h;
        for (uint32_t sx = 0; sx < st; sx++)
          for (uint32_t sy = 0; sy < st; sy++) {
            const int32_t tx = (int32_t)cx + (int32_t)sx - (int32_t)M, ty = (int32_t)cy + (int32_t)sy - (int32_t)M;
            if (tx < 0 || tx >= (int32_t)p.cfx || ty < 0 || ty >= (int32_t)p.cfy) continue;
            const uint32_t tgt_cf = (uint32_t)tx + p.cfx * (uint32_t)ty;
            for (uint32_t tp = 0; tp < nsub; tp++)
              for (uint32_t sp = 0; sp < nsub; sp++) {
                const float cp = prob(sp, tp, sx, sy);
                const double dmin = (double)p.DMin[sp * nsub + tp] + 0.5, dmax = (double)p.DMax[sp * nsub + tp] + 0.5;
                if (cp > 0.0)
                  fprintf(fpc, " %5d %5d     %g   %g   %g   '%s'   %8g   %g\n", (int)(nsub * tgt_cf + tp),
                          (int)(nsub * src_cf + sp), (double)cp, dmin, dmax, "Fixed",
                          (double)p.J[sp * nsub + tp], (double)p.DJ[sp * nsub + tp]);
              }
          }
        uint32_t bx = cx, by = cy;   // generateSourceNeuCExt: mirrored, clamped
        if (bx >= p.cfx / 2) bx = p.cfx - 1 - bx;
        if (by >= p.cfy / 2) by = p.cfy - 1 - by;
        if (bx >= S) bx = S - 1;
        if (by >= S) by = S - 1;
        const float cext = (float)p.bath[bx * S + by];
        for (uint32_t sp = 0; sp < nsub; sp++)
          fprintf(fpm, " %6d   %g   %g   %g   %7g   %g   %g   %g   %g   %g   %4g   %4g   %d \n", (int)p.count[sp],
                  (double)p.JExt[sp], (double)p.DJExt[sp], (double)cext, (double)p.NuExt[sp], (double)p.Tau[sp],
                  (double)p.Theta[sp], (double)p.H[sp], (double)p.Tarp[sp], (double)p.AlphaC[sp],
                  (double)p.TauC[sp], (double)p.gC[sp], 0);
      }
    fclose(fpc);
    fclose(fpm);
  }
}

uint32_t env_u32_or(const char *name, uint32_t dflt) {
  const char *s = getenv(name);
  return s ? (uint32_t)atoi(s) : dflt;
}

}  // namespace

dpsnn_params getParameters(const uint32_t loc_h) {
  (void)loc_h;
  dpsnn_params par;
  if (dpsnn_params_from_env(nullptr, &par)) die("getParameters");
  return par;
}

void localNetProcess_init(DALProcess *p) {
  (void)p;
  if (g_net) {
    printf("ERROR localNetProcess_init called twice\n");
    fflush(stdout);
    exit(0);
  }
  LocalNet *n = new LocalNet();
  if (dpsnn_params_from_env(nullptr, &n->par)) die("getParameters");
  const dpsnn_params &q = n->par;
  n->P = q.glob_h;
  n->globCFT = q.cfx * q.cfy;
  n->npcm = 0;
  for (uint32_t s = 0; s < q.nsub; s++) n->npcm += q.count[s];
  n->locN = n->npcm * n->globCFT / n->P;
  n->locCFT = ((float)n->globCFT / (float)n->P);
  if (env_u32_or("DPSNN_WRITE_INI_FILES", 0) == 1) write_ini_files(*n);
  dpsnn_options opt;
  memset(&opt, 0, sizeof opt);
  opt.device = (int)env_u32_or("DPSNN_DEVICE", 0);
  if (dpsnn_create(&n->par, &opt, &n->eng)) die("localNetClass::init");
  // statClass::prep (DPSNN_stat.c:553-561): only rank 0 writes the probe
  n->probe = env_u32_or("env_statSynPeriodicProbe_writeDisable", 1) == 0;
  n->probe_start_s = env_u32_or("env_startSynPeriodicProbe_s", 0);
  n->probe_stop_s = env_u32_or("env_stopSynPeriodicProbe_s", 0);
  if (n->probe && q.start_plasticity_ms <= q.stop_plasticity_ms && q.start_plasticity_ms < q.total_sim_time_ms) {
    if (dpsnn_enable_ltp_probe(n->eng)) die("statSynPeriodicProbe");
    const uint64_t S = dpsnn_rank_synapse_count(n->eng, 0);
    n->syn_pre.resize(S);
    n->syn_post.resize(S);
    n->syn_delay.resize(S);
    n->syn_kind.resize(S);
    if (dpsnn_backward_synapses(n->eng, 0, n->syn_pre.data(), n->syn_post.data(), n->syn_delay.data(),
                                n->syn_kind.data(), nullptr, nullptr))
      die("statSynPeriodicProbe");
    for (uint64_t k = 0; k < S; k++)
      if (n->syn_pre[k] < n->locN) n->probe_idx.push_back(k);
  }
  // statClass::prep (DPSNN_stat.c:546-551): only rank 0 writes STDP events
  n->stdp_ev = env_u32_or("env_statSTDPevent_writeDisable", 1) == 0 && q.start_plasticity_ms <= q.stop_plasticity_ms &&
               q.start_plasticity_ms < q.total_sim_time_ms;
  n->stdp_start_s = env_u32_or("env_startSTDPevent_s", 0);
  n->stdp_stop_s = env_u32_or("env_stopSTDPevent_s", 0);
  n->debug_ms = env_u32_or("env_debugPrintEnable_ms", 0);
  if (n->stdp_ev) {
    if (dpsnn_enable_stdp_events(n->eng)) die("statSTDPevent");
    n->ev_pre.resize(DPSNN_STDP_LOG_CAP);
    n->ev_post.resize(DPSNN_STDP_LOG_CAP);
    n->ev_c.resize(DPSNN_STDP_LOG_CAP);
  }
  n->max_ms = (int32_t)q.total_sim_time_ms;
  n->chrono = env_u32_or("env_chrono", 0);
  n->chrono_start = env_u32_or("env_startPartialChrono_ms", 0);
  n->chrono_stop = n->chrono_start + env_u32_or("env_partialChronoWindow_ms", 0);
  n->rank.resize(n->P);
  for (RankStat &r : n->rank) r.per_pop.assign((size_t)n->globCFT * q.nsub, 0u);
  n->ids.resize(dpsnn_glob_n(n->eng));
  n->te.resize(dpsnn_glob_n(n->eng));
  g_net = n;
}

int localNetProcess_fire(DALProcess *p) {
  (void)p;
  LocalNet *n = g_net;
  if (!n) {
    printf("ERROR localNetProcess_fire before init\n");
    fflush(stdout);
    exit(0);
  }
  if (n->ms > n->max_ms) {
    printf("ERROR programmed max sim time ms exceeded\n");
    exit(0);
  }
  if (n->ms == n->max_ms) return 1;
  const uint32_t sec = (uint32_t)n->ms / 1000;
  if (n->ms % 1000 == 0) open_second(*n, sec);
  if (dpsnn_step(n->eng, 1)) die("completeTimeStep_ms");
  uint32_t cnt = 0;
  if (dpsnn_spikes(n->eng, (uint32_t)n->ms, n->ids.data(), n->te.data(), (uint32_t)n->ids.size(), &cnt))
    die("completeTimeStep_ms");
  // the list is rank-major and ascending: split it at the rank boundaries
  uint32_t a = 0;
  for (uint32_t h = 0; h < n->P; h++) {
    const uint32_t end_id = (h + 1) * n->locN;
    uint32_t b = a;
    while (b < cnt && n->ids[b] < end_id) b++;
    rank_outputs(*n, h, n->ids.data() + a, n->te.data() + a, b - a);
    a = b;
  }
  if (n->stdp_f) write_stdp_events(*n);
  // longTermPlasticity runs at x999 ms inside the plasticity window
  // (DPSNN_localNet_sim.c:281-284) and writes the probe
  const dpsnn_params &q = n->par;
  if (n->ms % 1000 == 999 && n->probe_a && !n->syn_pre.empty() && (uint32_t)n->ms >= q.start_plasticity_ms &&
      (uint32_t)n->ms <= q.stop_plasticity_ms)
    write_probe(*n);
  if (n->ms % 1000 == 999) close_second(*n);
  n->ms++;
  return 0;
}

void localNetProcess_finish(DALProcess *p) {
  (void)p;
  LocalNet *n = g_net;
  if (!n) return;
  if (n->chrono == 1)
    for (uint32_t h = 0; h < n->P; h++) write_chrono_window(*n, h);
  close_second(*n);
  dpsnn_destroy(n->eng);
  delete n;
  g_net = nullptr;
}

struct dpsnn_engine *localNetProcess_engine(void) { return g_net ? g_net->eng : nullptr; }
