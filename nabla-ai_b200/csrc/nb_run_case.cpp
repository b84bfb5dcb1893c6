// nb_run_case.cpp — the case run loop of `nabla_solve run` on the GPU
// (runCase, core/src/flow/case.cpp:349-401), over the library's own C ABI.
//
// The loop, the stop rules, the file names and the diagnostics.jsonl record
// (one JSON object per step, keys in the reference's order, numbers written by
// a default-formatted std::ostream as the reference writes them) are the
// reference's, so the consumers of a run directory read either. The first line
// of a fresh file is a provenance record naming this library.
#include <filesystem>
#include <fstream>
#include <string>

#include "nb_ctx.h"

namespace {

constexpr const char* kSolverName = "nabla_b200";
constexpr const char* kSolverVersion = "1.0.0";

void append_step(std::ofstream& f, const nb_step_report& r) {
  f << "{\"step\":" << r.step << ",\"t\":" << r.t << ",\"dt\":" << r.dt << ",\"cfl\":" << r.cfl
    << ",\"momentum_residual\":" << r.momentum_residual << ",\"continuity_residual\":" << r.continuity_residual
    << ",\"divergence_max\":" << r.divergence_max << ",\"mass_error\":" << r.mass_error << ",\"cd\":" << r.cd
    << ",\"cl\":" << r.cl << ",\"poisson_iters\":" << r.poisson_iters << ",\"poisson_residual\":" << r.poisson_residual
    << ",\"cells\":" << r.cell_count << ",\"accepted\":" << (r.accepted ? "true" : "false") << "}\n";
}

struct CaseHolder {
  nb_case* c = nullptr;
  ~CaseHolder() {
    if (c) nb_case_destroy(c);
  }
};

}  // namespace

extern "C" {

nb_status nb_run_case(nb_ctx* ctx, const nb_grid_desc* grid, const nb_flow_config* cfg, const nb_run_options* opt,
                      nb_run_summary* out) {
  if (!ctx || !grid || !cfg || !opt || !opt->run_dir || opt->max_steps < 0) return NB_ERR_BAD_ARG;
  CaseHolder h;
  nb_status st = nb_case_create(ctx, grid, cfg, opt->precision, &h.c);
  if (st != NB_OK) return st;
  if ((st = nb_case_initialize(h.c)) != NB_OK) return st;
  const std::string dir = opt->run_dir;
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  if (ec) return nb::fail(ctx, NB_ERR_BAD_ARG, "nb_run_case: cannot create " + dir + ": " + ec.message());
  const bool restart = opt->restart_from && *opt->restart_from;
  if (restart && (st = nb_case_read_checkpoint(h.c, opt->restart_from)) != NB_OK) return st;
  std::ofstream diag(dir + "/diagnostics.jsonl", restart ? std::ios::app : std::ios::trunc);
  if (!diag) return nb::fail(ctx, NB_ERR_BAD_ARG, "nb_run_case: cannot open " + dir + "/diagnostics.jsonl");
  if (!restart)
    diag << "{\"event\":\"meta\",\"solver\":\"" << kSolverName << "\",\"solver_version\":\"" << kSolverVersion
         << "\",\"git_sha\":\"unknown\"}\n";
  nb_run_summary sum{};
  nb_step_report last{};
  for (int s = 0; s < opt->max_steps; ++s) {
    if ((st = nb_step(h.c, 0.0, &last)) != NB_OK) return st;  // dt from computeDt, as NSSolver::step()
    append_step(diag, last);
    diag.flush();
    if (opt->snapshot_every > 0 && last.step % opt->snapshot_every == 0) {
      const std::string p = dir + "/snapshot_" + std::to_string(last.step) + ".vtu";
      if ((st = nb_case_write_vtu(h.c, p.c_str())) != NB_OK) return st;
    }
    if (opt->checkpoint_every > 0 && last.step % opt->checkpoint_every == 0) {
      const std::string p = dir + "/checkpoint_" + std::to_string(last.step) + ".ckpt";
      if ((st = nb_case_write_checkpoint(h.c, p.c_str())) != NB_OK) return st;
    }
    if (opt->stop_time > 0.0 && last.t >= opt->stop_time) break;
    if (opt->steady_tol > 0.0 && last.step > 20 && last.momentum_residual < opt->steady_tol) {
      sum.steady = 1;
      break;
    }
  }
  if ((st = nb_case_write_vtu(h.c, (dir + "/final.vtu").c_str())) != NB_OK) return st;
  if ((st = nb_case_write_checkpoint(h.c, (dir + "/final.ckpt").c_str())) != NB_OK) return st;
  sum.steps = last.step;
  sum.time = last.t;
  sum.momentum_residual = last.momentum_residual;
  sum.continuity_residual = last.continuity_residual;
  sum.mass_error = last.mass_error;
  sum.cd = last.cd;
  sum.cl = last.cl;
  sum.cells = static_cast<uint64_t>(grid->nx) * grid->ny * grid->nz;
  if (out) *out = sum;
  return NB_OK;
}

}  // extern "C"
