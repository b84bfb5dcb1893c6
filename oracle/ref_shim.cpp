// ref_shim.cpp — TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A C ABI over the reference's own CPU classes, compiled together with the
// reference sources in place (see oracle/Makefile) into oracle/_ref/libnabla_ref.so.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
//
// Wrapped reference entry points (paths relative to the reference project):
//   nabla::flow::NSSolver            core/include/nabla/flow/ns_solver.hpp:58-156
//   nabla::flow::CgPoisson::applyA   core/src/flow/poisson.cpp:102-134
//   nabla::flow::CgPoisson::solve    core/src/flow/poisson.cpp:136-252
//   nabla::flow::MgPoisson::solve    core/src/flow/multigrid.cpp:206-355
//   nabla::flow::OctreePoisson       core/src/flow/octree_poisson.cpp:64-197
//   nabla::mesh::Octree              core/src/mesh/octree.cpp
//   nabla::mesh::mortonEncode/Decode core/include/nabla/mesh/morton.hpp:19-48
//   nabla::flow::makeChannel etc.    core/src/flow/case.cpp:25-134
//   writeCheckpoint / readCheckpoint core/src/flow/case.cpp:274-323
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "nabla/flow/case.hpp"
#include "nabla/flow/grid.hpp"
#include "nabla/flow/ns_solver.hpp"
#include "nabla/flow/octree_poisson.hpp"
#include "nabla/flow/poisson.hpp"
#include "nabla/mesh/morton.hpp"
#include "nabla/mesh/octree.hpp"
#include "nabla_b200.h"

using namespace nabla;

namespace {

thread_local std::string g_err;

flow::UniformGrid toGrid(const nb_grid_desc* d) {
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
  if (d->solid) {
    std::memcpy(g.solid.data(), d->solid, g.cellCount());
  }
  return g;
}

void fromGrid(const flow::UniformGrid& g, nb_grid_desc* d) {
  std::memset(d, 0, sizeof(*d));
  d->nx = g.nx;
  d->ny = g.ny;
  d->nz = g.nz;
  d->origin[0] = g.origin.x;
  d->origin[1] = g.origin.y;
  d->origin[2] = g.origin.z;
  d->dx = g.dx;
  d->dy = g.dy;
  d->dz = g.dz;
  for (int f = 0; f < 6; ++f) {
    d->face[f].type = static_cast<int32_t>(g.face[f].type);
    d->face[f].profile = static_cast<int32_t>(g.face[f].profile);
    d->face[f].inlet_axis = g.face[f].inletAxis;
    d->face[f].inlet_speed = g.face[f].inletSpeed;
    d->face[f].wall_velocity[0] = g.face[f].wallVelocity.x;
    d->face[f].wall_velocity[1] = g.face[f].wallVelocity.y;
    d->face[f].wall_velocity[2] = g.face[f].wallVelocity.z;
  }
}

flow::FlowConfig toCfg(const nb_flow_config* c) {
  flow::FlowConfig f;
  f.reynolds = c->reynolds;
  f.refLength = c->ref_length;
  f.velocityScale = c->velocity_scale;
  f.density = c->density;
  f.cfl = c->cfl;
  f.bodyForce = {c->body_force[0], c->body_force[1], c->body_force[2]};
  f.convection = c->convection == NB_CONV_WENO5 ? flow::ConvectionScheme::Weno5
                                                : flow::ConvectionScheme::Central;
  f.poissonTol = c->poisson_tol;
  f.poissonMaxIters = c->poisson_max_iters;
  f.tolContinuity = c->tol_continuity;
  f.tolMass = c->tol_mass;
  f.refArea = c->ref_area;
  return f;
}

void fromCfg(const flow::FlowConfig& f, nb_flow_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->reynolds = f.reynolds;
  c->ref_length = f.refLength;
  c->velocity_scale = f.velocityScale;
  c->density = f.density;
  c->cfl = f.cfl;
  c->body_force[0] = f.bodyForce.x;
  c->body_force[1] = f.bodyForce.y;
  c->body_force[2] = f.bodyForce.z;
  c->convection = f.convection == flow::ConvectionScheme::Weno5 ? NB_CONV_WENO5 : NB_CONV_CENTRAL;
  c->poisson_tol = f.poissonTol;
  c->poisson_max_iters = f.poissonMaxIters;
  c->tol_continuity = f.tolContinuity;
  c->tol_mass = f.tolMass;
  c->ref_area = f.refArea;
}

void toReport(const flow::StepReport& r, nb_step_report* o) {
  std::memset(o, 0, sizeof(*o));
  o->step = r.step;
  o->poisson_iters = r.poissonIters;
  o->t = r.t;
  o->dt = r.dt;
  o->cfl = r.cfl;
  o->momentum_residual = r.momentumResidual;
  o->continuity_residual = r.continuityResidual;
  o->divergence_max = r.divergenceMax;
  o->mass_error = r.massError;
  o->poisson_residual = r.poissonResidual;
  o->cd = r.cd;
  o->cl = r.cl;
  o->cell_count = r.cellCount;
  o->accepted = r.accepted ? 1 : 0;
  o->converged = 1;
}

struct RefNS {
  std::shared_ptr<flow::MgPoisson> mg;
  std::unique_ptr<flow::NSSolver> ns;
};

struct RefOctree {
  std::unique_ptr<mesh::Octree> t;
};

}  // namespace

#define SHIM_TRY try {
#define SHIM_CATCH                 \
  }                                \
  catch (const std::exception& e) { \
    g_err = e.what();              \
    return 1;                      \
  }

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// Draws of std::uniform_real_distribution<double>(lo, hi) over std::mt19937 /
// std::mt19937_64 (the generators the reference tests seed; standard library,
// not reference code), so tests can rebuild the reference tests' inputs.
void ref_uniform(int bits64, uint64_t seed, double lo, double hi, uint64_t n, double* out) {
  std::uniform_real_distribution<double> dist(lo, hi);
  if (bits64) {
    std::mt19937_64 rng(seed);
    for (uint64_t i = 0; i < n; ++i) out[i] = dist(rng);
  } else {
    std::mt19937 rng(static_cast<std::mt19937::result_type>(seed));
    for (uint64_t i = 0; i < n; ++i) out[i] = dist(rng);
  }
}

// ---- case builders (core/src/flow/case.cpp:25-134) ----
int ref_make_case(int kind, int a, int b, double reynolds, double vel, nb_grid_desc* grid,
                  uint8_t* solid_out, nb_flow_config* cfg) {
  SHIM_TRY
  flow::CaseSpec s;
  if (kind == 0) {
    s = flow::makeLidCavity(a, reynolds, vel);
  } else if (kind == 1) {
    s = flow::makeChannel(a, b, reynolds, vel);
  } else {
    s = flow::makeWallMountedCube(a, reynolds);
  }
  fromGrid(s.grid, grid);
  if (solid_out) {
    std::memcpy(solid_out, s.grid.solid.data(), s.grid.cellCount());
  }
  fromCfg(s.flow, cfg);
  return 0;
  SHIM_CATCH
}

// ---- NSSolver ----
void* ref_ns_create(const nb_grid_desc* grid, const nb_flow_config* cfg) {
  try {
    auto* h = new RefNS();
    const flow::FlowConfig fc = toCfg(cfg);
    h->mg = std::make_shared<flow::MgPoisson>(fc.poissonTol, fc.poissonMaxIters);
    h->ns = std::make_unique<flow::NSSolver>(toGrid(grid), fc, h->mg);
    return h;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void ref_ns_destroy(void* h) { delete static_cast<RefNS*>(h); }

int ref_ns_initialize(void* h) {
  SHIM_TRY
  static_cast<RefNS*>(h)->ns->initialize();
  return 0;
  SHIM_CATCH
}

int ref_ns_set_state(void* h, const double* u, const double* v, const double* w, const double* p,
                     int step, double t, double dtLast) {
  SHIM_TRY
  auto& ns = *static_cast<RefNS*>(h)->ns;
  std::vector<double> U(u, u + ns.uFace().size()), V(v, v + ns.vFace().size()),
      W(w, w + ns.wFace().size()), P(p, p + ns.pressure().size());
  ns.setState(std::move(U), std::move(V), std::move(W), std::move(P), step, t, dtLast);
  return 0;
  SHIM_CATCH
}

int ref_ns_get_state(void* h, double* u, double* v, double* w, double* p) {
  SHIM_TRY
  auto& ns = *static_cast<RefNS*>(h)->ns;
  if (u) std::memcpy(u, ns.uFace().data(), ns.uFace().size() * 8);
  if (v) std::memcpy(v, ns.vFace().data(), ns.vFace().size() * 8);
  if (w) std::memcpy(w, ns.wFace().data(), ns.wFace().size() * 8);
  if (p) std::memcpy(p, ns.pressure().data(), ns.pressure().size() * 8);
  return 0;
  SHIM_CATCH
}

double ref_ns_compute_dt(void* h) { return static_cast<RefNS*>(h)->ns->computeDt(); }

int ref_ns_step(void* h, double dt, nb_step_report* rep) {
  SHIM_TRY
  auto& ns = *static_cast<RefNS*>(h)->ns;
  const flow::StepReport r = dt > 0.0 ? ns.step(dt) : ns.step();
  if (rep) toReport(r, rep);
  return 0;
  SHIM_CATCH
}

int ref_ns_write_checkpoint(void* h, const char* path) {
  SHIM_TRY
  flow::writeCheckpoint(*static_cast<RefNS*>(h)->ns, path);
  return 0;
  SHIM_CATCH
}

int ref_ns_read_checkpoint(void* h, const char* path) {
  SHIM_TRY
  flow::readCheckpoint(*static_cast<RefNS*>(h)->ns, path);
  return 0;
  SHIM_CATCH
}

// runCase (core/src/flow/case.cpp:349-401) with the given grid, flow config
// and run options; summary = steps, time, momentum, continuity, mass, cd, cl.
int ref_run_case(const nb_grid_desc* grid, const nb_flow_config* cfg, const char* run_dir, int max_steps,
                 double stop_time, double steady_tol, int checkpoint_every, const char* restart_from,
                 double* summary, int* steady) {
  SHIM_TRY
  flow::CaseSpec spec;
  spec.grid = toGrid(grid);
  spec.flow = toCfg(cfg);
  spec.run.runDir = run_dir;
  spec.run.maxSteps = max_steps;
  spec.run.stopTime = stop_time;
  spec.run.steadyTol = steady_tol;
  spec.run.checkpointEvery = checkpoint_every;
  spec.run.restartFrom = restart_from ? restart_from : "";
  spec.run.quiet = true;
  const flow::RunSummary s = flow::runCase(spec);
  const double v[7] = {static_cast<double>(s.steps), s.time, s.momentumResidual, s.continuityResidual,
                       s.massError, s.cd, s.cl};
  for (int q = 0; q < 7; ++q) summary[q] = v[q];
  *steady = s.steady ? 1 : 0;
  return 0;
  SHIM_CATCH
}

// loadCase (core/src/flow/case.cpp:136-170): the spec's grid (solid mask into
// `solid`, cap bytes), flow config and run options; run = max_steps,
// snapshot_every, checkpoint_every; runf = stop_time, steady_tol.
int ref_load_case(const char* path, nb_grid_desc* grid, uint8_t* solid, uint64_t cap, nb_flow_config* cfg,
                  char* run_dir, int run_dir_cap, int* run, double* runf) {
  SHIM_TRY
  const flow::CaseSpec s = flow::loadCase(path);
  fromGrid(s.grid, grid);
  const size_t n = s.grid.cellCount();
  if (s.grid.solid.size() == n && n <= cap) std::memcpy(solid, s.grid.solid.data(), n);
  grid->solid = nullptr;
  fromCfg(s.flow, cfg);
  std::snprintf(run_dir, static_cast<size_t>(run_dir_cap), "%s", s.run.runDir.c_str());
  run[0] = s.run.maxSteps;
  run[1] = s.run.snapshotEvery;
  run[2] = s.run.checkpointEvery;
  runf[0] = s.run.stopTime;
  runf[1] = s.run.steadyTol;
  return 0;
  SHIM_CATCH
}

// ---- Poisson ----
int ref_apply_a(const nb_grid_desc* grid, const double* x, double* out) {
  SHIM_TRY
  const flow::UniformGrid g = toGrid(grid);
  std::vector<double> X(x, x + g.cellCount()), O;
  flow::CgPoisson::applyA(g, X, O);
  std::memcpy(out, O.data(), O.size() * 8);
  return 0;
  SHIM_CATCH
}

int ref_build_diagonal(const nb_grid_desc* grid, double* diag) {
  SHIM_TRY
  const flow::UniformGrid g = toGrid(grid);
  std::vector<double> D;
  flow::CgPoisson::buildDiagonal(g, D);
  std::memcpy(diag, D.data(), D.size() * 8);
  return 0;
  SHIM_CATCH
}

int ref_poisson_solve(int which, const nb_grid_desc* grid, const double* b, double* x, double tol,
                      int maxit, nb_poisson_report* rep) {
  SHIM_TRY
  const flow::UniformGrid g = toGrid(grid);
  std::vector<double> B(b, b + g.cellCount()), X;
  flow::PoissonSolver::Report r;
  if (which == 0) {
    flow::CgPoisson s(tol, maxit);
    r = s.solve(g, B, X);
  } else {
    flow::MgPoisson s(tol, maxit);
    r = s.solve(g, B, X);
  }
  std::memcpy(x, X.data(), X.size() * 8);
  rep->iterations = r.iterations;
  rep->converged = r.converged ? 1 : 0;
  rep->residual = r.residual;
  return 0;
  SHIM_CATCH
}

// ---- Morton (core/include/nabla/mesh/morton.hpp:19-48) ----
uint64_t ref_morton_encode(uint32_t x, uint32_t y, uint32_t z) { return mesh::mortonEncode(x, y, z); }
void ref_morton_decode(uint64_t code, uint32_t* x, uint32_t* y, uint32_t* z) {
  mesh::mortonDecode(code, *x, *y, *z);
}

// ---- Octree (core/src/mesh/octree.cpp) ----
void* ref_octree_create(const double* origin, const double* extent, int maxLevel) {
  try {
    auto* h = new RefOctree();
    h->t = std::make_unique<mesh::Octree>(mesh::Vec3{origin[0], origin[1], origin[2]},
                                          mesh::Vec3{extent[0], extent[1], extent[2]}, maxLevel);
    return h;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void ref_octree_destroy(void* h) { delete static_cast<RefOctree*>(h); }
int ref_octree_refine_uniform(void* h, int times) {
  SHIM_TRY
  static_cast<RefOctree*>(h)->t->refineUniform(times);
  return 0;
  SHIM_CATCH
}
int ref_octree_refine_box(void* h, const double* lo, const double* hi, int times) {
  SHIM_TRY
  static_cast<RefOctree*>(h)->t->refineBox(mesh::Vec3{lo[0], lo[1], lo[2]},
                                           mesh::Vec3{hi[0], hi[1], hi[2]}, times);
  return 0;
  SHIM_CATCH
}
int ref_octree_refine_morton(void* h, uint64_t key) {
  SHIM_TRY
  static_cast<RefOctree*>(h)->t->refineByMorton(key);
  return 0;
  SHIM_CATCH
}
int ref_octree_coarsen(void* h, uint64_t key, int level) {
  try {
    return static_cast<RefOctree*>(h)->t->coarsen(key, level) ? 1 : 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ref_octree_is_balanced(void* h) { return static_cast<RefOctree*>(h)->t->isBalanced() ? 1 : 0; }
uint64_t ref_octree_cell_count(void* h) { return static_cast<RefOctree*>(h)->t->cellCount(); }
void ref_octree_cells(void* h, uint64_t* morton, uint8_t* level, uint8_t* mask) {
  const mesh::Octree& t = *static_cast<RefOctree*>(h)->t;
  for (std::size_t i = 0; i < t.cellCount(); ++i) {
    if (morton) morton[i] = t.morton(i);
    if (level) level[i] = static_cast<uint8_t>(t.level(i));
    if (mask) mask[i] = static_cast<uint8_t>(t.mask(i));
  }
}
void ref_octree_set_mask(void* h, uint64_t i, int mask) {
  static_cast<RefOctree*>(h)->t->setMask(i, static_cast<mesh::CellMask>(mask));
}
void ref_octree_cell_center(void* h, uint64_t i, double* c) {
  const mesh::Vec3 v = static_cast<RefOctree*>(h)->t->cellCenter(i);
  c[0] = v.x;
  c[1] = v.y;
  c[2] = v.z;
}
// Writes up to 4 neighbour indices; returns the count.
int ref_octree_face_neighbors(void* h, uint64_t i, int dir, uint64_t* out) {
  const std::vector<std::size_t> nb = static_cast<RefOctree*>(h)->t->faceNeighbors(i, dir);
  for (std::size_t k = 0; k < nb.size(); ++k) out[k] = nb[k];
  return static_cast<int>(nb.size());
}
int ref_octree_apply_a(void* h, const double* x, double* out) {
  SHIM_TRY
  const mesh::Octree& t = *static_cast<RefOctree*>(h)->t;
  std::vector<double> X(x, x + t.cellCount()), O;
  flow::OctreePoisson::applyA(t, X, O);
  std::memcpy(out, O.data(), O.size() * 8);
  return 0;
  SHIM_CATCH
}
int ref_octree_build_diagonal(void* h, double* diag) {
  SHIM_TRY
  const mesh::Octree& t = *static_cast<RefOctree*>(h)->t;
  std::vector<double> D;
  flow::OctreePoisson::buildDiagonal(t, D);
  std::memcpy(diag, D.data(), D.size() * 8);
  return 0;
  SHIM_CATCH
}
int ref_octree_solve(void* h, const double* b, double* x, double tol, int maxit,
                     nb_poisson_report* rep) {
  SHIM_TRY
  const mesh::Octree& t = *static_cast<RefOctree*>(h)->t;
  std::vector<double> B(b, b + t.cellCount()), X;
  flow::OctreePoisson s(tol, maxit);
  const auto r = s.solve(t, B, X);
  std::memcpy(x, X.data(), X.size() * 8);
  rep->iterations = r.iterations;
  rep->converged = r.converged ? 1 : 0;
  rep->residual = r.residual;
  return 0;
  SHIM_CATCH
}

}  // extern "C"
