// params.cpp -- the reference's inputs: env_* variables and the four text
// files, parsed with the reference's rules into a dpsnn_params.
//
// Restates getParameters (DPSNN_getParameters.c:23-831), readColumnFile
// (:834-898), readPlasticityParametersFile (:900-1053, including its habit of
// keeping the last line read), and the file parsers of describeConnectome
// (DPSNN_LIFCAconnectome.cpp:16-131, :240-398).  Numbers go through atof()
// into float, as the reference stores them.  Where the reference prints
// "ERROR ..." and exits, this returns DPSNN_E_PARAM with the same text.
//
// The compile-time limits of the reference build (Makefile:18-30: miniLocN,
// makeMaxGlobH, makeStencil_Max) are checked with the Makefile's values; the
// environment variables DPSNN_MAX_LOC_N, DPSNN_MAX_GLOB_H and
// DPSNN_MAX_STENCIL raise them for networks the GPU engine can hold but the
// reference build cannot.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "dpsnn_internal.h"

namespace {

thread_local std::vector<float> g_spec;
thread_local std::vector<uint32_t> g_bath;

uint32_t limit_from_env(const char *name, uint32_t def) {
  const char *v = getenv(name);
  return v ? (uint32_t)strtoul(v, nullptr, 10) : def;
}

std::string path_in(const char *dir, const char *file) {
  if (!dir || !*dir) return file;
  std::string p(dir);
  if (p.back() != '/') p += '/';
  return p + file;
}

// Tokenise one line the way the reference does (strtok on " \t\n", stop at
// a token starting with '#').
std::vector<std::string> tokens(char *buf) {
  std::vector<std::string> out;
  char *save = nullptr;
  for (char *tk = strtok_r(buf, " \t\n", &save); tk; tk = strtok_r(nullptr, " \t\n", &save)) {
    if (tk[0] == '#') break;
    out.emplace_back(tk);
  }
  return out;
}

int need_env(const char *name, const char **out) {
  *out = getenv(name);
  if (!*out) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: missing %s param in DPSNN_script", name);
  return 0;
}

int env_u32(const char *name, uint32_t *v) {
  const char *s;
  int rc = need_env(name, &s);
  if (rc) return rc;
  *v = (uint32_t)atoi(s);
  return 0;
}

int env_bool(const char *name, uint32_t *v) {
  const char *s;
  int rc = need_env(name, &s);
  if (rc) return rc;
  int x = atoi(s);
  if (x != 0 && x != 1) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: invalid %s param in DPSNN_script", name);
  *v = (uint32_t)x;
  return 0;
}

}  // namespace

extern "C" int dpsnn_params_from_env(const char *workdir, dpsnn_params *p) {
  if (!p) return dpsnn_fail(DPSNN_E_PARAM, "null params");
  memset(p, 0, sizeof *p);
  const uint32_t max_loc_n = limit_from_env("DPSNN_MAX_LOC_N", 32000);    // miniLocN
  const uint32_t max_glob_h = limit_from_env("DPSNN_MAX_GLOB_H", 256);    // makeMaxGlobH
  const uint32_t max_stencil = limit_from_env("DPSNN_MAX_STENCIL", 96);   // makeStencil_Max
  const char *s;
  int rc;
  uint32_t overall;
  if ((rc = env_u32("env_overallConnectivity", &overall))) return rc;
  if (overall != 0)
    return dpsnn_fail(DPSNN_E_PARAM, "env_overallConnectivity=%u: only the explicit stencil (0) is supported", overall);
  if ((rc = env_u32("env_stencilDim", &p->stencil_dim))) return rc;
  if (p->stencil_dim == 0 || p->stencil_dim > max_stencil)
    return dpsnn_fail(DPSNN_E_PARAM, "ERROR: env_stencilDim = %u out of %u range in DPSNN_script", p->stencil_dim,
                      max_stencil);
  if (2 * p->stencil_dim - 1 > max_stencil)
    return dpsnn_fail(DPSNN_E_PARAM, "ERROR: stencilX_Max = %u out of %u range, due to env_stencilDim set in DPSNN_script",
                      2 * p->stencil_dim - 1, max_stencil);
  if ((rc = env_u32("env_globH", &p->glob_h))) return rc;
  if (p->glob_h == 0 || p->glob_h > max_glob_h)
    return dpsnn_fail(DPSNN_E_PARAM, "ERROR: env_globH = %u out of range: [from 1 to %u] in DPSNN_script", p->glob_h,
                      max_glob_h);
  uint32_t syngen;
  if ((rc = env_u32("env_synGen", &syngen))) return rc;
  if (syngen != 2) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: unsupported synGen %u requested by DPSNN_script", syngen);

  // ---- column.txt (readColumnFile + initSubPopParamStruct)
  {
    std::string fn = path_in(workdir, "column.txt");
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) return dpsnn_fail(DPSNN_E_PARAM, "ERROR opening file column.txt ");
    char buf[200];
    while (fgets(buf, sizeof buf, f)) {
      std::vector<std::string> tk = tokens(buf);
      if (tk.empty()) continue;
      float v[12] = {(float)p->nsub, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (size_t k = 0; k < tk.size() && k < 12; k++) v[k] = (float)atof(tk[k].c_str());
      uint32_t sp = (uint32_t)v[0];
      if (sp >= DPSNN_MAX_SUBPOP) {
        fclose(f);
        return dpsnn_fail(DPSNN_E_PARAM, "ERROR in subPop initialization: wrong subPop identifier in column.txt file ");
      }
      p->count[sp] = (uint32_t)v[1];
      p->JExt[sp] = v[2];
      p->DJExt[sp] = v[3];
      p->NuExt[sp] = v[4];
      p->Tau[sp] = v[5];
      p->Theta[sp] = v[6];
      p->H[sp] = v[7];
      p->Tarp[sp] = v[8];
      p->AlphaC[sp] = v[9];
      p->TauC[sp] = v[10];
      p->gC[sp] = v[11];
      p->nsub++;
    }
    fclose(f);
    if (p->nsub == 0) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: lnp_par.neuronsPerCM <=0 in DPSNN_getParameters");
  }
  uint32_t npcm = 0;
  for (uint32_t k = 0; k < p->nsub; k++) npcm += p->count[k];
  if (npcm == 0) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: lnp_par.neuronsPerCM <=0 in DPSNN_getParameters");
  if (!getenv("env_CFX") || !getenv("env_CFY"))
    return dpsnn_fail(DPSNN_E_PARAM,
                      "ERROR: please set the env_CFX and env_CFY values in DPSNN_script (grid of Cortical Modules)");
  p->cfx = (uint32_t)atoi(getenv("env_CFX"));
  p->cfy = (uint32_t)atoi(getenv("env_CFY"));
  uint32_t cft = p->cfx * p->cfy;
  if (cft == 0 || cft > 96 * 96 + 1) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: globCFT more then %d", 96 * 96 + 1);
  if ((p->glob_h > cft && (p->glob_h % cft) != 0) || (cft > p->glob_h && (cft % p->glob_h) != 0))
    return dpsnn_fail(DPSNN_E_PARAM, "ERROR:#processes and #cort. columns must be  multiple OR equal");
  if (p->glob_h > cft)
    return dpsnn_fail(DPSNN_E_PARAM, "ERROR:a Cortical Module can be divided by max 1 processes");
  uint32_t loc_n = npcm * (cft / p->glob_h);
  if (loc_n > max_loc_n) return dpsnn_fail(DPSNN_E_PARAM, "ERROR too many neurons requested ");

  const char *mw;
  if ((rc = need_env("env_minSynWeight_f", &mw)))
    return dpsnn_fail(DPSNN_E_PARAM, "MISSING env_minSynWeigth in DPSNN launch script");
  p->min_syn_weight_f = (float)atof(mw);
  if (p->min_syn_weight_f >= 0 || p->min_syn_weight_f < -6.0)
    return dpsnn_fail(DPSNN_E_PARAM, "env_minSynWeigth out of range -6.000000 - 0.0");
  if ((rc = env_u32("env_D", &p->D))) return rc;
  if ((rc = env_u32("env_totalSimTime_ms", &p->total_sim_time_ms))) return rc;
  if ((rc = env_u32("env_startPlasticity_ms", &p->start_plasticity_ms))) return rc;
  if ((rc = env_u32("env_stopPlasticity_ms", &p->stop_plasticity_ms))) return rc;
  if ((rc = env_u32("env_moduloSec", &p->moduloSec))) return rc;
  if ((rc = env_u32("env_startStatFiles_s", &p->startStatFiles_s))) return rc;
  if ((rc = env_u32("env_stopStatFiles_s", &p->stopStatFiles_s))) return rc;
  if ((rc = env_bool("env_spikes_writeDisable", &p->spikes_writeDisable))) return rc;
  uint32_t tmp;
  if ((rc = env_bool("env_statSTDPevent_writeDisable", &tmp))) return rc;
  if ((rc = env_bool("env_statSynPeriodicProbe_writeDisable", &tmp))) return rc;
  if ((rc = env_bool("env_statRatesPerPop_writeDisable", &p->statRatesPerPop_writeDisable))) return rc;
  if ((rc = env_u32("env_startRatesPerPop_s", &p->startRatesPerPop_s))) return rc;
  if ((rc = env_u32("env_stopRatesPerPop_s", &p->stopRatesPerPop_s))) return rc;
  if ((rc = env_u32("env_startSynPeriodicProbe_s", &tmp))) return rc;
  if ((rc = env_u32("env_stopSynPeriodicProbe_s", &tmp))) return rc;
  if ((rc = env_u32("env_startSTDPevent_s", &tmp))) return rc;
  if ((rc = env_u32("env_stopSTDPevent_s", &tmp))) return rc;
  if ((rc = env_u32("env_ratesSampling", &p->ratesSampling))) return rc;
  if (p->moduloSec == 0) return dpsnn_fail(DPSNN_E_PARAM, "env_moduloSec must be > 0");
  if (p->ratesSampling == 0) return dpsnn_fail(DPSNN_E_PARAM, "env_ratesSampling must be > 0");
  if (!(s = getenv("env_globalSeed"))) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: missing env_globalSeed param");
  {
    int32_t seed = atoi(s);
    p->global_seed = seed < 0 ? (uint32_t)time(nullptr) : (uint32_t)seed;
  }
  s = getenv("env_howManyOutputFiles");
  p->howManyOutputFiles = s ? (uint32_t)atoi(s) : 0;
  if (p->howManyOutputFiles > 1) p->howManyOutputFiles = 0;
  // the delay distribution is a compile-time choice in the reference
  // (-DDelayUniform, DPSNN_LIFCAcorticalModuleGen.cpp:133-137)
  s = getenv("DPSNN_DELAY_DISTRIBUTION");
  p->delay_exponential = 0;
  if (s && strcmp(s, "exponential") == 0) p->delay_exponential = 1;
  else if (s && strcmp(s, "uniform") != 0)
    return dpsnn_fail(DPSNN_E_PARAM, "DPSNN_DELAY_DISTRIBUTION must be uniform or exponential");
  if ((rc = env_u32("env_collectivesAlgo", &tmp))) return rc;
  if ((rc = env_u32("env_pktLength", &tmp))) return rc;

  // ---- plasticity.txt (readPlasticityParametersFile)
  {
    std::string fn = path_in(workdir, "plasticity.txt");
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) {
      p->stdp_antiCausalCoeff = -1.0f;
      p->stdp_multiplier = 0.001f;
      p->stdp_tau_ms = 20.0f;
      p->stdp_causalMax = 0.1f;
      p->stdp_antiCausalMax = 0.12f;
      p->stdp_tauDecay_s = 1.0f;
      p->stdp_drift = 0.0f;
    } else {
      float v[20] = {0};
      size_t ntok = 0;
      char buf[200];
      while (fgets(buf, sizeof buf, f)) {  // keeps the last line read
        std::vector<std::string> tk = tokens(buf);
        ntok = tk.size();
        for (size_t k = 0; k < tk.size() && k < 20; k++) v[k] = (float)atof(tk[k].c_str());
      }
      fclose(f);
      if (ntok == 0 || ntok >= 20)
        return dpsnn_fail(DPSNN_E_PARAM, "ERROR: Plasticity.txt %zu columns (empty or too much params)", ntok);
      if (v[0] != 1) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: uknown algo in Plasticity.txt (first col)");
      if (ntok != 8) return dpsnn_fail(DPSNN_E_PARAM, "ERROR: wrong number %zu columns Plasticity.txt (expected 9)", ntok);
      p->stdp_antiCausalCoeff = v[1];
      p->stdp_multiplier = v[2];
      p->stdp_tau_ms = v[3];
      p->stdp_causalMax = v[4];
      p->stdp_antiCausalMax = v[5];
      p->stdp_tauDecay_s = v[6];
      p->stdp_drift = v[7];
    }
    if (p->stdp_tau_ms * 3 > 128)
      return dpsnn_fail(DPSNN_E_PARAM, "initLongTermPlasticity POSSIBLE ERROR: 3*tauSTDP>DSD__maxSTDPspan_ms");
    if (p->stdp_tau_ms <= 0) return dpsnn_fail(DPSNN_E_PARAM, "initLongTermPlasticity ERROR: tauSTDP <= 0");
    if (p->stdp_multiplier < 0) return dpsnn_fail(DPSNN_E_PARAM, "initLongTermPlasticity ERROR: STDPmultiplier < 0");
  }

  // ---- connectivity.txt (initConnectivityParam, explicit stencil)
  const uint32_t S = p->stencil_dim, nsub = p->nsub;
  g_spec.assign((size_t)nsub * nsub * S * S, 0.0f);
  {
    std::string fn = path_in(workdir, "connectivity.txt");
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) return dpsnn_fail(DPSNN_E_PARAM, "ERROR opening file connectivity.txt ");
    std::vector<char> buf(10 * 96 * 96 + 16);
    while (fgets(buf.data(), (int)buf.size(), f)) {
      std::vector<std::string> tk = tokens(buf.data());
      if (tk.empty()) continue;
      if (tk.size() - 6 != (size_t)S * S) {
        fclose(f);
        return dpsnn_fail(DPSNN_E_PARAM,
                          "ERROR: inconsistency in the number of elements of connectivity.txt file. Please check if the "
                          "connectivity matrix size matches the stencilDim set in the Makefile.");
      }
      std::vector<float> v(tk.size());
      for (size_t k = 0; k < tk.size(); k++) v[k] = (float)atof(tk[k].c_str());
      uint32_t sp = (uint32_t)v[0], tp = (uint32_t)v[1];
      if (sp >= nsub || tp >= nsub) {
        fclose(f);
        return dpsnn_fail(DPSNN_E_PARAM,
                          "ERROR in connectivity initialization: wrong subPop identifier in connectivity.txt file ");
      }
      p->J[sp * nsub + tp] = v[2];
      p->DJ[sp * nsub + tp] = v[3];
      p->DMin[sp * nsub + tp] = v[4];
      p->DMax[sp * nsub + tp] = v[5];
      size_t idx = 6;
      for (uint32_t y = 0; y < S; y++)
        for (uint32_t x = 0; x < S; x++) g_spec[((size_t)(sp * nsub + tp) * S + x) * S + y] = v[idx++];
    }
    fclose(f);
  }
  // ---- bathEfficacy.txt (initBathEfficacyTemplate)
  g_bath.assign((size_t)S * S, 0);
  {
    std::string fn = path_in(workdir, "bathEfficacy.txt");
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) return dpsnn_fail(DPSNN_E_PARAM, "ERROR opening file bathEfficacy.txt ");
    std::vector<char> buf(100000);
    uint32_t y = 0;
    while (fgets(buf.data(), (int)buf.size(), f)) {
      std::vector<std::string> tk = tokens(buf.data());
      if (tk.empty()) continue;
      if (tk.size() != S || y >= S) {
        fclose(f);
        return dpsnn_fail(DPSNN_E_PARAM,
                          "ERROR: number of elements in bathEfficacy.txt file doesn't match the stencil size stencilDim "
                          "set in the Makefile.");
      }
      for (uint32_t x = 0; x < S; x++) g_bath[(size_t)x * S + y] = (uint32_t)atoi(tk[x].c_str());
      y++;
    }
    fclose(f);
  }
  p->spec = g_spec.data();
  p->bath = g_bath.data();
  return 0;
}
