// nabla_adaptive_cuda.hpp — the B200 library behind the adaptive control
// plane's flow seam, for a maintainer of nabla_core to include.
//
//   nabla::adaptive::CudaSolverBackend : SolverBackend
//       (core/include/nabla/adaptive/run.hpp:11-32) with the flow advanced on
//       the GPU: BaselineBackend's behaviour (core/src/adaptive/run.cpp:23-65)
//       on a uniform grid, or an octree-native case on a brick mesh. step(),
//       the telemetry getters and sample() keep their meaning; sampleMany()
//       answers any number of points with one kernel launch.
//   nabla::adaptive::sampleFlowCuda(Octree&, const CudaSolverBackend&)
//       sampleFlow (core/src/adaptive/run.cpp:84-95) with one batched sample
//       per field instead of one virtual call per cell and field.
//
// Needs the reference's include directory (core/include) and this project's
// include/ on the include path, and links libnabla_b200.so.
#pragma once

#include <memory>
#include <utility>
#include <vector>

#include "nabla/adaptive/run.hpp"
#include "nabla_flow_cuda.hpp"

namespace nabla::adaptive {

class CudaSolverBackend : public SolverBackend {
 public:
  // Uniform grid: the GPU form of BaselineBackend(grid, cfg).
  CudaSolverBackend(std::shared_ptr<nabla_b200::Context> ctx, const flow::UniformGrid& grid,
                    const flow::FlowConfig& cfg, int precision = NB_PRECISION_FP64)
      : ctx_(std::move(ctx)), cells_(grid.cellCount()) {
    const nb_grid_desc g = flow::to_b200(grid);
    const nb_flow_config c = flow::to_b200(cfg);
    nb_case* h = nullptr;
    ctx_->check(nb_case_create(ctx_->get(), &g, &c, precision, &h), "CudaSolverBackend");
    h_.reset(h);
    ctx_->check(nb_case_initialize(h), "CudaSolverBackend::initialize");
    nu_ = cfg.velocityScale * cfg.refLength / cfg.reynolds;
  }
  // Octree-native: a case on a brick mesh (nb_amr_mesh_create) with its
  // initial state already set by the caller through nb_amr_case_set_state.
  CudaSolverBackend(std::shared_ptr<nabla_b200::Context> ctx, nb_case* octree_case, std::size_t uniform_cells,
                    double nu)
      : ctx_(std::move(ctx)), h_(octree_case), cells_(uniform_cells), nu_(nu) {}

  void step() override { ctx_->check(nb_step(h_.get(), 0.0, &last_), "CudaSolverBackend::step"); }

  double sample(int component, Vec3 p) const override {
    const double xyz[3] = {p.x, p.y, p.z};
    double v = 0.0;
    ctx_->check(nb_case_sample(h_.get(), component, 1, xyz, &v), "CudaSolverBackend::sample");
    return v;
  }
  // out[i] = sample(component, pts[i]) for every point, in one launch.
  void sampleMany(int component, const std::vector<Vec3>& pts, std::vector<double>& out) const {
    std::vector<double> xyz(pts.size() * 3);
    for (std::size_t i = 0; i < pts.size(); ++i) {
      xyz[3 * i] = pts[i].x;
      xyz[3 * i + 1] = pts[i].y;
      xyz[3 * i + 2] = pts[i].z;
    }
    out.resize(pts.size());
    ctx_->check(nb_case_sample(h_.get(), component, static_cast<int64_t>(pts.size()), xyz.data(), out.data()),
                "CudaSolverBackend::sampleMany");
  }

  double cd() const override { return last_.cd; }
  double cl() const override { return last_.cl; }
  double momentumResidual() const override { return last_.momentum_residual; }
  double nu() const override { return nu_; }
  std::size_t uniformCells() const override { return cells_; }
  double t() const override { return last_.t; }
  double dt() const override { return last_.dt; }
  double cfl() const override { return last_.cfl; }
  double continuityResidual() const override { return last_.continuity_residual; }
  double divergenceMax() const override { return last_.divergence_max; }
  double massError() const override { return last_.mass_error; }
  int poissonIters() const override { return last_.poisson_iters; }
  double poissonResidual() const override { return last_.poisson_residual; }

  [[nodiscard]] nb_case* handle() const { return h_.get(); }

 private:
  struct Del {
    void operator()(nb_case* p) const { nb_case_destroy(p); }
  };
  std::shared_ptr<nabla_b200::Context> ctx_;
  std::unique_ptr<nb_case, Del> h_;
  std::size_t cells_ = 0;
  double nu_ = 0.0;
  nb_step_report last_{};
};

// sampleFlow (core/src/adaptive/run.cpp:84-95): every cell's u, v, w, p from
// the backend at the cell centre, one batched launch per field.
inline void sampleFlowCuda(Octree& tree, const CudaSolverBackend& backend) {
  std::vector<Vec3> centres(tree.cellCount());
  for (std::size_t i = 0; i < centres.size(); ++i) centres[i] = tree.cellCenter(i);
  std::vector<double>* fields[4] = {&tree.u(), &tree.v(), &tree.w(), &tree.p()};
  for (int c = 0; c < 4; ++c) backend.sampleMany(c, centres, *fields[c]);
}

}  // namespace nabla::adaptive
