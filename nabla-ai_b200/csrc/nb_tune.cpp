// nb_tune.cpp — launch tuning of a context and the autotuner (no reference
// counterpart).
//
// The tuned choices change launch shapes (threads per brick and CTAs per SM),
// the multigrid halo staging, the mixed form's smoother and sweeps, the exact
// coarse-solve threshold, the cluster-resident V-cycle tail and PDL.
// None of them changes the discretisation: FP64 results move only by the
// summation order of the grid reductions (grid size, cluster tail), mixed results by the
// preconditioner (sweeps, coarse solve) within the solve tolerance.
//
// The autotuner times candidates on scratch copies of a sample case with
// CUDA events on the case's stream, by coordinate descent from the default,
// and caches the winner per (GPU, SM count, mesh kind, precision, levels,
// size class) in a text file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "nb_ctx.h"

using namespace nb;

namespace {

bool tuning_ok(const nb_tuning& t, std::string& why) {
  if (t.mg_ctas_per_sm < 1 || t.mg_ctas_per_sm > 16) why = "mg_ctas_per_sm must be in 1..16";
  else if (t.rhs_ctas_per_sm < 1 || t.rhs_ctas_per_sm > 4) why = "rhs_ctas_per_sm must be in 1..4";
  else if (t.halo_mode != 0 && t.halo_mode != 1) why = "halo_mode must be 0 or 1";
  else if (t.sweeps < 1 || t.sweeps > 3) why = "sweeps must be in 1..3";
  else if (t.coarse_direct_max < 0 || t.coarse_direct_max > 512) why = "coarse_direct_max must be in 0..512";
  else if (t.pdl != 0 && t.pdl != 1) why = "pdl must be 0 or 1";
  else if (t.threads_per_brick != 128 && t.threads_per_brick != 256 && t.threads_per_brick != 512)
    why = "threads_per_brick must be 128, 256 or 512";
  else if (t.smoother != 0 && t.smoother != 1) why = "smoother must be 0 or 1";
  else if (t.tail_bricks < 0 || t.tail_bricks > 4096) why = "tail_bricks must be in 0..4096";
  else if (t.warm_start < 0 || t.warm_start > 3) why = "warm_start must be in 0..3";
  else if (t.vgrid != 0 && t.vgrid != 1) why = "vgrid must be 0 or 1";
  else if (t.coarse_bf16 != 0 && t.coarse_bf16 != 1) why = "coarse_bf16 must be 0 or 1";
  else if (t.ghost_map != 0 && t.ghost_map != 1) why = "ghost_map must be 0 or 1";
  else return true;
  return false;
}

std::string tune_key(nb_ctx* ctx, const nb_case* c) {
  cudaDeviceProp prop{};
  NB_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
  std::string name = prop.name;
  for (char& ch : name)
    if (ch == ' ' || ch == '\t') ch = '_';
  int amr = 0, prec = 0, lev = 1;
  case_kind(c, &amr, &prec, &lev);
  const double cells = static_cast<double>(nb_case_cell_count(c));
  const int size_class = cells > 0 ? static_cast<int>(std::floor(std::log2(cells))) : 0;
  std::ostringstream k;
  k << name << "/sm" << ctx->nsm << "/" << (amr ? "octree" : "uniform") << "/"
    << (prec == NB_PRECISION_MIXED ? "mixed" : "fp64") << "/L" << lev << "/c2^" << size_class;
  std::string s = k.str();
  if (s.size() > 127) s.resize(127);
  return s;
}

// One cache line: key and the thirteen fields, then ms per step.
bool parse_line(const std::string& line, std::string& key, nb_tuning& t, double& ms) {
  std::istringstream in(line);
  if (!(in >> key >> t.mg_ctas_per_sm >> t.rhs_ctas_per_sm >> t.halo_mode >> t.sweeps >> t.coarse_direct_max >>
        t.pdl >> t.threads_per_brick >> t.smoother >> t.tail_bricks >>
        t.warm_start >> t.vgrid >> t.coarse_bf16 >> t.ghost_map >> ms))
    return false;
  std::string why;
  return tuning_ok(t, why);
}

std::string format_line(const std::string& key, const nb_tuning& t, double ms) {
  char buf[320];
  std::snprintf(buf, sizeof buf, "%s %d %d %d %d %d %d %d %d %d %d %d %d %d %.6g", key.c_str(), t.mg_ctas_per_sm,
                t.rhs_ctas_per_sm, t.halo_mode, t.sweeps, t.coarse_direct_max, t.pdl, t.threads_per_brick, t.smoother,
                t.tail_bricks, t.warm_start, t.vgrid, t.coarse_bf16, t.ghost_map, ms);
  return buf;
}

bool blank(const std::string& line) {
  for (char ch : line)
    if (ch != ' ' && ch != '\t' && ch != '\r') return ch == '#';
  return true;
}

}  // namespace

extern "C" {

void nb_tuning_default(nb_tuning* t) {
  if (!t) return;
  t->mg_ctas_per_sm = 4;
  t->rhs_ctas_per_sm = 4;
  t->halo_mode = 0;
  t->sweeps = 2;
  t->coarse_direct_max = 256;
  t->pdl = 1;
  t->threads_per_brick = 512;
  t->smoother = 1;
  t->tail_bricks = 8;
  t->warm_start = 3;
  t->vgrid = 0;
  t->coarse_bf16 = 0;
  t->ghost_map = 1;
}

nb_status nb_ctx_set_tuning(nb_ctx* ctx, const nb_tuning* t) {
  if (!ctx || !t) return NB_ERR_BAD_ARG;
  std::string why;
  if (!tuning_ok(*t, why)) return fail(ctx, NB_ERR_BAD_ARG, "nb_ctx_set_tuning: " + why);
  ctx->tune = *t;
  // cached Poisson hierarchies are rebuilt with the new tuning on next use
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    ctx->mg_cache.clear();
    return NB_OK;
  });
}

nb_status nb_ctx_get_tuning(const nb_ctx* ctx, nb_tuning* t) {
  if (!ctx || !t) return NB_ERR_BAD_ARG;
  *t = ctx->tune;
  return NB_OK;
}

int nb_tune_cache_lookup(const char* cache_path, const char* key, nb_tuning* t, double* ms) {
  if (!cache_path || !key || !t) return -1;
  std::ifstream in(cache_path);
  if (!in) return 0;  // no cache yet
  std::string line;
  while (std::getline(in, line)) {
    if (blank(line)) continue;
    std::string k;
    nb_tuning v{};
    double m = 0.0;
    if (!parse_line(line, k, v, m)) return -1;
    if (k == key) {
      *t = v;
      if (ms) *ms = m;
      return 1;
    }
  }
  return 0;
}

nb_status nb_tune_cache_store(const char* cache_path, const char* key, const nb_tuning* t, double ms) {
  if (!cache_path || !key || !t || !*key || std::strpbrk(key, " \t\r\n")) return NB_ERR_BAD_ARG;
  std::string why;
  if (!tuning_ok(*t, why)) return NB_ERR_BAD_ARG;
  std::vector<std::string> lines;
  {
    std::ifstream in(cache_path);
    std::string line;
    while (in && std::getline(in, line)) {
      std::string k;
      nb_tuning v{};
      double m = 0.0;
      if (!blank(line) && parse_line(line, k, v, m) && k == key) continue;  // replaced below
      lines.push_back(line);
    }
  }
  lines.push_back(format_line(key, *t, ms));
  // write a sibling file and rename it over the cache (readers never see a partial file)
  const std::string tmp = std::string(cache_path) + ".tmp";
  {
    std::ofstream out(tmp, std::ios::trunc);
    if (!out) return NB_ERR_BAD_ARG;
    for (const std::string& l : lines) out << l << "\n";
    if (!out) return NB_ERR_BAD_ARG;
  }
  if (std::rename(tmp.c_str(), cache_path) != 0) return NB_ERR_BAD_ARG;
  return NB_OK;
}

nb_status nb_autotune(nb_ctx* ctx, nb_case* sample, int steps, const char* cache_path, nb_tune_report* rep) {
  if (!ctx || !sample || !rep || steps < 1) return NB_ERR_BAD_ARG;
  std::memset(rep, 0, sizeof *rep);
  const nb_tuning saved = ctx->tune;
  std::string key;
  nb_status st = guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    key = tune_key(ctx, sample);
    return NB_OK;
  });
  if (st != NB_OK) return st;
  std::snprintf(rep->key, sizeof rep->key, "%s", key.c_str());
  if (cache_path) {
    nb_tuning t{};
    double ms = 0.0;
    const int found = nb_tune_cache_lookup(cache_path, key.c_str(), &t, &ms);
    if (found < 0) return fail(ctx, NB_ERR_BAD_ARG, std::string("nb_autotune: malformed cache file ") + cache_path);
    if (found == 1) {
      ctx->tune = t;
      rep->best = t;
      rep->best_ms = rep->default_ms = ms;
      rep->from_cache = 1;
      return NB_OK;
    }
  }
  int amr = 0, prec = 0, lev = 1;
  case_kind(sample, &amr, &prec, &lev);

  // ms per step of candidate t (< 0: rejected), on a scratch copy of the sample
  auto time_one = [&](const nb_tuning& t, double* ms) -> nb_status {
    *ms = -1.0;
    ctx->tune = t;
    nb_case* c = nullptr;
    nb_status s = clone_case(sample, &c);
    ctx->tune = saved;
    if (s != NB_OK) return s;
    double dt = 0.0;
    nb_step_report r{};
    s = nb_case_compute_dt(c, &dt);
    if (s == NB_OK) s = nb_step(c, dt, &r);  // warm-up: builds the step graph
    bool ok = s == NB_OK && r.converged && r.divergence_max <= 1e-8;
    if (ok) {
      s = guarded(ctx, [&] {
        cudaStream_t cs = static_cast<cudaStream_t>(nb_case_stream(c));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        NB_CUDA(cudaEventCreate(&e0));
        NB_CUDA(cudaEventCreate(&e1));
        NB_CUDA(cudaEventRecord(e0, cs));
        nb_status s2 = nb_step_many(c, dt, steps, &r);
        NB_CUDA(cudaEventRecord(e1, cs));
        NB_CUDA(cudaEventSynchronize(e1));
        float el = 0.0f;
        NB_CUDA(cudaEventElapsedTime(&el, e0, e1));
        NB_CUDA(cudaEventDestroy(e0));
        NB_CUDA(cudaEventDestroy(e1));
        if (s2 == NB_OK && r.converged && r.divergence_max <= 1e-8) *ms = el / steps;
        return s2;
      });
    }
    nb_case_destroy(c);
    ++rep->candidates;
    if (s == NB_OK && *ms < 0.0) ++rep->rejected;
    return s;
  };

  nb_tuning best;
  nb_tuning_default(&best);
  double best_ms = 0.0;
  st = time_one(best, &best_ms);
  if (st != NB_OK) return st;
  if (best_ms < 0.0)
    return fail(ctx, NB_ERR_NOT_CONVERGED, "nb_autotune: the sample does not converge to divergence <= 1e-8");
  rep->default_ms = best_ms;
  auto consider = [&](const nb_tuning& cand) -> nb_status {
    double ms = 0.0;
    const nb_status s = time_one(cand, &ms);
    if (s == NB_OK && ms >= 0.0 && ms < 0.98 * best_ms) {
      best = cand;
      best_ms = ms;
    }
    return s;
  };
  // threads per brick, keeping the resident threads per SM
  for (int32_t v : {256, 128}) {
    nb_tuning cand = best;
    cand.threads_per_brick = v;
    cand.mg_ctas_per_sm = std::min(16, best.mg_ctas_per_sm * best.threads_per_brick / v);
    if ((st = consider(cand)) != NB_OK) return st;
  }
  // multigrid CTAs per SM: 1/4 .. 1 of a full SM (2048 threads)
  {
    const int full = 2048 / best.threads_per_brick;
    for (int32_t v : {full / 4, full / 2, 3 * full / 4, full}) {
      if (v == best.mg_ctas_per_sm) continue;
      nb_tuning cand = best;
      cand.mg_ctas_per_sm = v;
      if ((st = consider(cand)) != NB_OK) return st;
    }
  }
  struct Knob {
    int32_t nb_tuning::*field;
    std::vector<int32_t> values;
  };
  std::vector<Knob> knobs = {{&nb_tuning::vgrid, {0, 1}},
                             {&nb_tuning::tail_bricks, {0, 8, 32, 128}},
                             {&nb_tuning::rhs_ctas_per_sm, {1, 2, 3, 4}},
                             {&nb_tuning::halo_mode, {0, 1}},
                             {&nb_tuning::pdl, {0, 1}}};
  if (prec == NB_PRECISION_MIXED) {
    knobs.push_back({&nb_tuning::smoother, {0, 1}});
    knobs.push_back({&nb_tuning::sweeps, {1, 2, 3}});
    knobs.push_back({&nb_tuning::warm_start, {0, 1, 2, 3}});
    knobs.push_back({&nb_tuning::coarse_bf16, {0, 1}});
  }
  if (amr && lev > 1) knobs.push_back({&nb_tuning::coarse_direct_max, {0, 256, 512}});
  for (const Knob& k : knobs)
    for (int32_t v : k.values) {
      if (best.*(k.field) == v) continue;
      nb_tuning cand = best;
      cand.*(k.field) = v;
      if ((st = consider(cand)) != NB_OK) return st;
    }
  ctx->tune = best;
  rep->best = best;
  rep->best_ms = best_ms;
  if (cache_path && nb_tune_cache_store(cache_path, key.c_str(), &best, best_ms) != NB_OK)
    return fail(ctx, NB_ERR_BAD_ARG, std::string("nb_autotune: cannot write cache file ") + cache_path);
  return NB_OK;
}

}  // extern "C"
