// nabla_b200.hpp — C++20 host API over the C ABI of nabla_b200.h.
//
// Header-only. Mirrors the reference's flow-solver surface so a C++ caller
// switches by changing types, not call sites:
//   nabla_b200::MgPoisson  ~ nabla::flow::PoissonSolver / MgPoisson
//                            (core/include/nabla/flow/poisson.hpp:20-33, :69-92)
//   nabla_b200::NSSolver   ~ nabla::flow::NSSolver
//                            (core/include/nabla/flow/ns_solver.hpp:58-156)
// Error behaviour follows the reference core: failures throw
// std::runtime_error (here nabla_b200::Error, which also carries the nb_status);
// Poisson non-convergence is reported in Report::converged, not thrown.
// Fields cross as std::vector<double> in the reference's lexicographic MAC
// layouts; inside, the state stays resident on the GPU between steps and the
// face accessors download on demand (cached until the next step or setState).
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "nabla_b200.h"

namespace nabla_b200 {

class Error : public std::runtime_error {
 public:
  Error(nb_status s, const std::string& what) : std::runtime_error(what), status_(s) {}
  [[nodiscard]] nb_status status() const { return status_; }

 private:
  nb_status status_;
};

// One CUDA device. Owns the library context (streams, MG hierarchy cache).
class Context {
 public:
  explicit Context(int device = 0) {
    nb_ctx* h = nullptr;
    const nb_status s = nb_ctx_create(device, &h);
    if (s != NB_OK) {
      const std::string msg = h ? nb_last_error(h) : nb_status_string(s);
      if (h) nb_ctx_destroy(h);
      throw Error(s, "nabla_b200: context creation failed: " + msg);
    }
    h_.reset(h);
  }
  [[nodiscard]] nb_ctx* get() const { return h_.get(); }
  void check(nb_status s, const char* what) const {
    if (s != NB_OK) throw Error(s, std::string("nabla_b200: ") + what + ": " + nb_last_error(h_.get()));
  }
  [[nodiscard]] uint64_t launches() const { return nb_ctx_launch_count(h_.get()); }

 private:
  struct Del {
    void operator()(nb_ctx* p) const { nb_ctx_destroy(p); }
  };
  std::unique_ptr<nb_ctx, Del> h_;
};

inline std::size_t cell_count(const nb_grid_desc& g) {
  return static_cast<std::size_t>(g.nx) * static_cast<std::size_t>(g.ny) * static_cast<std::size_t>(g.nz);
}

// MG-PCG pressure solve behind the PoissonSolver seam.
class MgPoisson {
 public:
  struct Report {
    int iterations = 0;
    double residual = 0.0;
    bool converged = false;
  };
  MgPoisson(std::shared_ptr<Context> ctx, double tol = 1e-10, int max_iters = 200,
            int precision = NB_PRECISION_FP64)
      : ctx_(std::move(ctx)), tol_(tol), max_iters_(max_iters), precision_(precision) {}

  // x is resized by the callee, as PoissonSolver::solve does.
  Report solve(const nb_grid_desc& grid, const std::vector<double>& b, std::vector<double>& x) {
    const std::size_t n = cell_count(grid);
    if (b.size() != n) throw Error(NB_ERR_BAD_ARG, "nabla_b200: MgPoisson::solve: b has the wrong size");
    x.assign(n, 0.0);
    nb_poisson_report r{};
    ctx_->check(nb_poisson_solve(ctx_->get(), &grid, b.data(), x.data(), tol_, max_iters_, precision_, &r),
                "MgPoisson::solve");
    return Report{r.iterations, r.residual, r.converged != 0};
  }
  [[nodiscard]] std::string name() const {
    return precision_ == NB_PRECISION_MIXED ? "b200-mg-pcg-mixed" : "b200-mg-pcg";
  }
  [[nodiscard]] double tol() const { return tol_; }
  [[nodiscard]] int max_iters() const { return max_iters_; }

 private:
  std::shared_ptr<Context> ctx_;
  double tol_;
  int max_iters_;
  int precision_;
};

// SSP-RK3 MAC step with MG-PCG projection; the state lives on the GPU.
class NSSolver {
 public:
  NSSolver(std::shared_ptr<Context> ctx, const nb_grid_desc& grid, const nb_flow_config& cfg,
           int precision = NB_PRECISION_FP64)
      : ctx_(std::move(ctx)), grid_(grid), cfg_(cfg) {
    if (grid.solid) {
      solid_.assign(grid.solid, grid.solid + cell_count(grid));
      grid_.solid = solid_.data();
    }
    nb_case* h = nullptr;
    ctx_->check(nb_case_create(ctx_->get(), &grid_, &cfg_, precision, &h), "NSSolver");
    h_.reset(h);
    nu_ = cfg.velocity_scale * cfg.ref_length / cfg.reynolds;
  }

  void initialize() {
    ctx_->check(nb_case_initialize(h_.get()), "NSSolver::initialize");
    invalidate();
  }
  nb_step_report step() { return step(0.0); }
  nb_step_report step(double dt) {
    nb_step_report r{};
    ctx_->check(nb_step(h_.get(), dt, &r), "NSSolver::step");
    invalidate();
    return r;
  }
  [[nodiscard]] double computeDt() const {
    double dt = 0.0;
    ctx_->check(nb_case_compute_dt(h_.get(), &dt), "NSSolver::computeDt");
    return dt;
  }
  [[nodiscard]] double time() const { return clock().t; }
  [[nodiscard]] int stepIndex() const { return clock().step; }
  [[nodiscard]] double dtLast() const { return clock().dt_last; }
  [[nodiscard]] double nu() const { return nu_; }
  [[nodiscard]] const nb_grid_desc& grid() const { return grid_; }
  [[nodiscard]] const nb_flow_config& config() const { return cfg_; }

  [[nodiscard]] const std::vector<double>& uFace() const { return fetch().u; }
  [[nodiscard]] const std::vector<double>& vFace() const { return fetch().v; }
  [[nodiscard]] const std::vector<double>& wFace() const { return fetch().w; }
  [[nodiscard]] const std::vector<double>& pressure() const { return fetch().p; }
  [[nodiscard]] std::vector<double> cellPressure() const { return fetch().p; }

  void setState(std::vector<double> u, std::vector<double> v, std::vector<double> w, std::vector<double> p,
                int step, double t, double dt_last) {
    const std::size_t nx = grid_.nx, ny = grid_.ny, nz = grid_.nz;
    if (u.size() != (nx + 1) * ny * nz || v.size() != nx * (ny + 1) * nz || w.size() != nx * ny * (nz + 1) ||
        p.size() != nx * ny * nz)
      throw Error(NB_ERR_BAD_ARG, "nabla_b200: NSSolver::setState: size mismatch");
    ctx_->check(nb_case_set_state(h_.get(), u.data(), v.data(), w.data(), p.data(), step, t, dt_last),
                "NSSolver::setState");
    invalidate();
  }
  [[nodiscard]] uint64_t deviceBytes() const { return nb_case_device_bytes(h_.get()); }
  [[nodiscard]] nb_case* handle() const { return h_.get(); }
  // writeCheckpoint / readCheckpoint (core/src/flow/case.cpp:274-319): the NBFCK01 file.
  void writeCheckpoint(const std::string& path) const {
    ctx_->check(nb_case_write_checkpoint(h_.get(), path.c_str()), "writeCheckpoint");
  }
  void readCheckpoint(const std::string& path) {
    ctx_->check(nb_case_read_checkpoint(h_.get(), path.c_str()), "readCheckpoint");
    invalidate();
  }

 private:
  struct Clock {
    int step = 0;
    double t = 0.0, dt_last = 0.0;
  };
  struct Fields {
    std::vector<double> u, v, w, p;
  };
  [[nodiscard]] Clock clock() const {
    Clock c;
    ctx_->check(nb_case_get_clock(h_.get(), &c.step, &c.t, &c.dt_last), "NSSolver clock");
    return c;
  }
  const Fields& fetch() const {
    if (!cache_) {
      const std::size_t nx = grid_.nx, ny = grid_.ny, nz = grid_.nz;
      auto f = std::make_unique<Fields>();
      f->u.resize((nx + 1) * ny * nz);
      f->v.resize(nx * (ny + 1) * nz);
      f->w.resize(nx * ny * (nz + 1));
      f->p.resize(nx * ny * nz);
      ctx_->check(nb_case_get_state(h_.get(), f->u.data(), f->v.data(), f->w.data(), f->p.data()),
                  "NSSolver state download");
      cache_ = std::move(f);
    }
    return *cache_;
  }
  void invalidate() { cache_.reset(); }
  struct Del {
    void operator()(nb_case* p) const { nb_case_destroy(p); }
  };
  std::shared_ptr<Context> ctx_;
  nb_grid_desc grid_;
  nb_flow_config cfg_;
  std::vector<uint8_t> solid_;
  std::unique_ptr<nb_case, Del> h_;
  double nu_ = 0.0;
  mutable std::unique_ptr<Fields> cache_;
};

// runCase (core/src/flow/case.cpp:349-401) on the GPU: the run loop of
// `nabla_solve run` with diagnostics.jsonl and checkpoints in opt.run_dir.
inline nb_run_summary runCase(const std::shared_ptr<Context>& ctx, const nb_grid_desc& grid,
                              const nb_flow_config& flow, const nb_run_options& opt) {
  nb_run_summary s{};
  ctx->check(nb_run_case(ctx->get(), &grid, &flow, &opt, &s), "runCase");
  return s;
}

}  // namespace nabla_b200
