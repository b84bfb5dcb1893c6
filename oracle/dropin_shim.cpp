// dropin_shim.cpp — TEST INFRASTRUCTURE ONLY: runs the reference's own
// NSSolver (core/src/flow/ns_solver.cpp, compiled in place by oracle/Makefile)
// with the B200 library plugged in through the reference-side binding
// nabla-ai_b200/integration/nabla_flow_cuda.hpp, so the GPU tests can show
// the drop-in at the reference's seams:
//   mode 0  NSSolver + the reference's MgPoisson (CPU)
//   mode 1  NSSolver + CudaMgPoisson (PoissonSolver seam, poisson.hpp:20-33)
//   mode 2  CudaNSSolver (the whole step on the GPU, NSSolver's surface)
// and the adaptive seam (SolverBackend, core/include/nabla/adaptive/run.hpp)
// with CudaSolverBackend from nabla-ai_b200/integration/nabla_adaptive_cuda.hpp.
// Built into oracle/_ref/libnabla_dropin.so; loaded only by tests/.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "nabla/flow/grid.hpp"
#include "nabla/flow/ns_solver.hpp"
#include "nabla/flow/poisson.hpp"
#include "nabla/mesh/octree.hpp"
#include "nabla_adaptive_cuda.hpp"
#include "nabla_flow_cuda.hpp"

using namespace nabla;

namespace {

thread_local std::string g_err;

std::shared_ptr<nabla_b200::Context> context() {
  static std::shared_ptr<nabla_b200::Context> ctx = std::make_shared<nabla_b200::Context>(0);
  return ctx;
}

flow::UniformGrid grid_of(const nb_grid_desc* d) {
  flow::UniformGrid g;
  g.nx = d->nx;
  g.ny = d->ny;
  g.nz = d->nz;
  g.origin = {d->origin[0], d->origin[1], d->origin[2]};
  g.dx = d->dx;
  g.dy = d->dy;
  g.dz = d->dz;
  for (int f = 0; f < 6; ++f) {
    const nb_face_bc& s = d->face[f];
    g.face[f].type = static_cast<flow::BoundaryType>(s.type);
    g.face[f].profile = static_cast<flow::InletProfile>(s.profile);
    g.face[f].inletAxis = s.inlet_axis;
    g.face[f].inletSpeed = s.inlet_speed;
    g.face[f].wallVelocity = {s.wall_velocity[0], s.wall_velocity[1], s.wall_velocity[2]};
  }
  g.allocate();
  if (d->solid) std::memcpy(g.solid.data(), d->solid, g.cellCount());
  return g;
}

flow::FlowConfig config_of(const nb_flow_config* c) {
  flow::FlowConfig f;
  f.reynolds = c->reynolds;
  f.refLength = c->ref_length;
  f.velocityScale = c->velocity_scale;
  f.density = c->density;
  f.cfl = c->cfl;
  f.bodyForce = {c->body_force[0], c->body_force[1], c->body_force[2]};
  f.convection = c->convection == NB_CONV_WENO5 ? flow::ConvectionScheme::Weno5 : flow::ConvectionScheme::Central;
  f.poissonTol = c->poisson_tol;
  f.poissonMaxIters = c->poisson_max_iters;
  f.tolContinuity = c->tol_continuity;
  f.tolMass = c->tol_mass;
  f.refArea = c->ref_area;
  return f;
}

template <class NS>
void run(NS& ns, int nsteps, double dt, double* u, double* v, double* w, double* p, int* iters, double* dts) {
  const flow::UniformGrid& g = ns.grid();
  const std::size_t nx = g.nx, ny = g.ny, nz = g.nz;
  std::vector<double> U(u, u + (nx + 1) * ny * nz), V(v, v + nx * (ny + 1) * nz), W(w, w + nx * ny * (nz + 1)),
      P(p, p + nx * ny * nz);
  ns.setState(std::move(U), std::move(V), std::move(W), std::move(P), 0, 0.0, 0.0);
  for (int s = 0; s < nsteps; ++s) {
    const flow::StepReport r = dt > 0.0 ? ns.step(dt) : ns.step();
    if (iters) iters[s] = r.poissonIters;
    if (dts) dts[s] = r.dt;
  }
  std::memcpy(u, ns.uFace().data(), ns.uFace().size() * 8);
  std::memcpy(v, ns.vFace().data(), ns.vFace().size() * 8);
  std::memcpy(w, ns.wFace().data(), ns.wFace().size() * 8);
  std::memcpy(p, ns.pressure().data(), ns.pressure().size() * 8);
}

}  // namespace

extern "C" {

const char* dropin_last_error() { return g_err.c_str(); }

// Steps (u, v, w, p) in place, nsteps times (dt <= 0: CFL dt), with the
// solver selected by `mode`; iters[s] / dts[s] receive each step's Poisson
// cycles and dt (either may be NULL).
int dropin_run(const nb_grid_desc* grid, const nb_flow_config* cfg, int mode, int nsteps, double dt, double* u,
               double* v, double* w, double* p, int* iters, double* dts) {
  try {
    const flow::UniformGrid g = grid_of(grid);
    const flow::FlowConfig fc = config_of(cfg);
    if (mode == 0) {
      flow::NSSolver ns(g, fc, nullptr);
      run(ns, nsteps, dt, u, v, w, p, iters, dts);
    } else if (mode == 1) {
      auto mg = std::make_shared<flow::CudaMgPoisson>(context(), fc.poissonTol, fc.poissonMaxIters);
      flow::NSSolver ns(g, fc, mg);
      run(ns, nsteps, dt, u, v, w, p, iters, dts);
    } else {
      flow::CudaNSSolver ns(context(), g, fc);
      run(ns, nsteps, dt, u, v, w, p, iters, dts);
    }
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// One PoissonSolver::solve through the seam: mode 0 the reference's
// MgPoisson, mode 1 CudaMgPoisson.
int dropin_poisson(const nb_grid_desc* grid, const double* b, double* x, double tol, int max_cycles, int mode,
                   int* iters, double* residual, int* converged) {
  try {
    const flow::UniformGrid g = grid_of(grid);
    std::unique_ptr<flow::PoissonSolver> s;
    if (mode == 0) s = std::make_unique<flow::MgPoisson>(tol, max_cycles);
    else s = std::make_unique<flow::CudaMgPoisson>(context(), tol, max_cycles);
    const std::vector<double> B(b, b + g.cellCount());
    std::vector<double> X;
    const flow::PoissonSolver::Report r = s->solve(g, B, X);
    std::memcpy(x, X.data(), X.size() * 8);
    *iters = r.iterations;
    *residual = r.residual;
    *converged = r.converged ? 1 : 0;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// CudaSolverBackend after nsteps steps against the reference's NSSolver
// stepped alike and read the way BaselineBackend::sample reads it
// (core/src/adaptive/run.cpp:49-62). For each component c = 0..3 and point q:
// one[c*n+q] = sample(), many[c*n+q] = sampleMany(), ref[c*n+q] = reference.
// tele = backend t, dt, cfl, momentum residual, divergence max, poisson iters,
// then the reference StepReport's same fields. tree_err = max |sampleFlowCuda -
// per-cell sample()| over a uniformly refined reference Octree (3 levels).
int dropin_backend(const nb_grid_desc* grid, const nb_flow_config* cfg, int nsteps, int64_t n, const double* xyz,
                   double* one, double* many, double* ref, double* tele, double* tree_err) {
  try {
    const flow::UniformGrid g = grid_of(grid);
    const flow::FlowConfig c = config_of(cfg);
    adaptive::CudaSolverBackend be(context(), g, c);
    flow::NSSolver ns(g, c, std::make_shared<flow::MgPoisson>(c.poissonTol, c.poissonMaxIters));
    ns.initialize();
    flow::StepReport last;
    for (int s = 0; s < nsteps; ++s) {
      be.step();
      last = ns.step();
    }
    std::vector<adaptive::Vec3> pts(static_cast<size_t>(n));
    for (int64_t q = 0; q < n; ++q) pts[q] = {xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]};
    const std::vector<double> pc = ns.cellPressure();
    for (int comp = 0; comp < 4; ++comp) {
      std::vector<double> m;
      be.sampleMany(comp, pts, m);
      for (int64_t q = 0; q < n; ++q) {
        one[comp * n + q] = be.sample(comp, pts[q]);
        many[comp * n + q] = m[q];
        int i = static_cast<int>((pts[q].x - g.origin.x) / g.dx);
        int j = static_cast<int>((pts[q].y - g.origin.y) / g.dy);
        int k = static_cast<int>((pts[q].z - g.origin.z) / g.dz);
        i = std::clamp(i, 0, g.nx - 1);
        j = std::clamp(j, 0, g.ny - 1);
        k = std::clamp(k, 0, g.nz - 1);
        ref[comp * n + q] = comp == 0   ? ns.cellU(i, j, k)
                            : comp == 1 ? ns.cellV(i, j, k)
                            : comp == 2 ? ns.cellW(i, j, k)
                                        : pc[g.cidx(i, j, k)];
      }
    }
    const double mine[6] = {be.t(), be.dt(), be.cfl(), be.momentumResidual(), be.divergenceMax(),
                            static_cast<double>(be.poissonIters())};
    const double theirs[6] = {last.t, last.dt, last.cfl, last.momentumResidual, last.divergenceMax,
                              static_cast<double>(last.poissonIters)};
    for (int q = 0; q < 6; ++q) {
      tele[q] = mine[q];
      tele[6 + q] = theirs[q];
    }
    mesh::Octree tree({g.origin.x, g.origin.y, g.origin.z}, {g.nx * g.dx, g.ny * g.dy, g.nz * g.dz}, 6);
    tree.refineUniform(3);
    adaptive::sampleFlowCuda(tree, be);
    double err = 0.0;
    for (std::size_t i = 0; i < tree.cellCount(); ++i) {
      const adaptive::Vec3 ctr = tree.cellCenter(i);
      const double got[4] = {tree.u()[i], tree.v()[i], tree.w()[i], tree.p()[i]};
      for (int comp = 0; comp < 4; ++comp) err = std::max(err, std::abs(got[comp] - be.sample(comp, ctr)));
    }
    *tree_err = err;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

}  // extern "C"
