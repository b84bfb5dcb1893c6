// nabla_flow_cuda.hpp — the reference-side binding: the B200 library behind
// the reference core's own seams, for a maintainer of nabla_core to include.
//
//   nabla::flow::CudaMgPoisson : PoissonSolver
//       drops into NSSolver's constructor argument
//       (core/include/nabla/flow/ns_solver.hpp:60-61) exactly like MgPoisson
//       (core/include/nabla/flow/poisson.hpp:69-92): same solve() contract
//       (x resized by the callee, Report{iterations, residual, converged},
//       non-convergence reported, not thrown).
//   nabla::flow::CudaNSSolver
//       the whole step on the GPU, with NSSolver's public surface
//       (ns_solver.hpp:58-96) and its types (UniformGrid, FlowConfig,
//       StepReport), so runCase (core/src/flow/case.cpp:349-371) can hold
//       either one.
//
// Needs the reference's include directory (core/include) and this project's
// include/ on the include path, and links libnabla_b200.so. Nothing here is
// compiled into libnabla_b200.so itself.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "nabla/flow/grid.hpp"
#include "nabla/flow/ns_solver.hpp"
#include "nabla/flow/poisson.hpp"
#include "nabla_b200.hpp"

namespace nabla::flow {

// UniformGrid -> nb_grid_desc. The descriptor points into g.solid, so it is
// valid while g is.
inline nb_grid_desc to_b200(const UniformGrid& g) {
  nb_grid_desc d{};
  d.nx = g.nx;
  d.ny = g.ny;
  d.nz = g.nz;
  d.origin[0] = g.origin.x;
  d.origin[1] = g.origin.y;
  d.origin[2] = g.origin.z;
  d.dx = g.dx;
  d.dy = g.dy;
  d.dz = g.dz;
  for (int f = 0; f < 6; ++f) {
    const FaceBC& s = g.face[f];
    d.face[f].type = static_cast<int32_t>(s.type);
    d.face[f].profile = static_cast<int32_t>(s.profile);
    d.face[f].inlet_axis = s.inletAxis;
    d.face[f].inlet_speed = s.inletSpeed;
    d.face[f].wall_velocity[0] = s.wallVelocity.x;
    d.face[f].wall_velocity[1] = s.wallVelocity.y;
    d.face[f].wall_velocity[2] = s.wallVelocity.z;
  }
  d.solid = g.solid.size() == g.cellCount() ? g.solid.data() : nullptr;
  return d;
}

inline nb_flow_config to_b200(const FlowConfig& c) {
  nb_flow_config o{};
  o.reynolds = c.reynolds;
  o.ref_length = c.refLength;
  o.velocity_scale = c.velocityScale;
  o.density = c.density;
  o.cfl = c.cfl;
  o.body_force[0] = c.bodyForce.x;
  o.body_force[1] = c.bodyForce.y;
  o.body_force[2] = c.bodyForce.z;
  o.convection = c.convection == ConvectionScheme::Weno5 ? NB_CONV_WENO5 : NB_CONV_CENTRAL;
  o.poisson_max_iters = c.poissonMaxIters;
  o.poisson_tol = c.poissonTol;
  o.tol_continuity = c.tolContinuity;
  o.tol_mass = c.tolMass;
  o.ref_area = c.refArea;
  return o;
}

inline StepReport from_b200(const nb_step_report& r) {
  StepReport s;
  s.step = r.step;
  s.t = r.t;
  s.dt = r.dt;
  s.cfl = r.cfl;
  s.momentumResidual = r.momentum_residual;
  s.continuityResidual = r.continuity_residual;
  s.divergenceMax = r.divergence_max;
  s.massError = r.mass_error;
  s.poissonIters = r.poisson_iters;
  s.poissonResidual = r.poisson_residual;
  s.cd = r.cd;
  s.cl = r.cl;
  s.cellCount = static_cast<std::size_t>(r.cell_count);
  s.accepted = r.accepted != 0;
  return s;
}

class CudaMgPoisson : public PoissonSolver {
 public:
  explicit CudaMgPoisson(std::shared_ptr<nabla_b200::Context> ctx, double tol = 1e-9, int maxCycles = 100,
                         int precision = NB_PRECISION_FP64)
      : mg_(std::move(ctx), tol, maxCycles, precision) {}
  Report solve(const UniformGrid& grid, const std::vector<double>& b, std::vector<double>& x) override {
    const nb_grid_desc d = to_b200(grid);
    const nabla_b200::MgPoisson::Report r = mg_.solve(d, b, x);
    Report o;
    o.iterations = r.iterations;
    o.residual = r.residual;
    o.converged = r.converged;
    return o;
  }
  [[nodiscard]] std::string name() const override { return "cuda-" + mg_.name(); }

 private:
  nabla_b200::MgPoisson mg_;
};

class CudaNSSolver {
 public:
  CudaNSSolver(std::shared_ptr<nabla_b200::Context> ctx, UniformGrid grid, FlowConfig config,
               int precision = NB_PRECISION_FP64)
      : grid_(std::move(grid)), cfg_(config), ns_(std::move(ctx), to_b200(grid_), to_b200(cfg_), precision) {}

  void initialize() { ns_.initialize(); }
  StepReport step() { return from_b200(ns_.step()); }
  StepReport step(double dt) { return from_b200(ns_.step(dt)); }
  [[nodiscard]] double time() const { return ns_.time(); }
  [[nodiscard]] int stepIndex() const { return ns_.stepIndex(); }
  [[nodiscard]] double dtLast() const { return ns_.dtLast(); }
  [[nodiscard]] double nu() const { return ns_.nu(); }
  [[nodiscard]] const UniformGrid& grid() const { return grid_; }
  [[nodiscard]] const FlowConfig& config() const { return cfg_; }
  [[nodiscard]] const std::vector<double>& uFace() const { return ns_.uFace(); }
  [[nodiscard]] const std::vector<double>& vFace() const { return ns_.vFace(); }
  [[nodiscard]] const std::vector<double>& wFace() const { return ns_.wFace(); }
  [[nodiscard]] const std::vector<double>& pressure() const { return ns_.pressure(); }
  [[nodiscard]] std::vector<double> cellPressure() const { return ns_.cellPressure(); }
  void setState(std::vector<double> u, std::vector<double> v, std::vector<double> w, std::vector<double> p,
                int step, double t, double dtLast) {
    ns_.setState(std::move(u), std::move(v), std::move(w), std::move(p), step, t, dtLast);
  }
  [[nodiscard]] double computeDt() const { return ns_.computeDt(); }

 private:
  UniformGrid grid_;
  FlowConfig cfg_;
  nabla_b200::NSSolver ns_;
};

}  // namespace nabla::flow
