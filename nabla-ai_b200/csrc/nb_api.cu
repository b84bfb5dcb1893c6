// nb_api.cu — the extern "C" boundary (include/nabla_b200.h) over the device
// solver: context, resident cases, the SSP-RK3 step driver and the Poisson
// seam. Host orchestration only; all arithmetic on the solution runs in the
// kernels of nb_flow.cu, nb_amr_flow.cu and nb_mg.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "nb_amr_faces.h"
#include "nb_amr_flow.cuh"
#include "nb_amr_mesh.h"
#include "nb_ctx.h"
#include "nb_maps.h"
#include "nb_flow.cuh"
#include "nb_mg.cuh"

using namespace nb;

// Results of one step, written by the step's kernels.
struct StepBlock {
  StepScalars sc;
  AmrStepScalars asc;  // octree-AMR cases
  double rep[3][6];  // per projection: MgSolver report
  double dt;
  unsigned long long execs;  // MG loop-body executions so far
};

struct GraphSlot {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t fixed_kernels = 0;
  uint64_t body_kernels = 0;
};

struct nb_case {
  nb_ctx* ctx = nullptr;
  nb_grid_desc grid{};
  std::vector<uint8_t> solid;
  nb_flow_config cfg{};
  int precision = NB_PRECISION_FP64;
  double nu = 0.0;
  std::unique_ptr<MgSolver> mg;
  FlowView F{};
  cudaStream_t stream = nullptr;
  double* uvw[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int cur = 0;
  double* uvw0[3] = {nullptr, nullptr, nullptr};
  double* p = nullptr;
  double* b = nullptr;
  // Mixed form: each RK stage's pressure (phi / dt) of the last two steps,
  // [stage][0 latest, 1 the one before], and how many steps it holds (0..2,
  // device): the history warm start (nb_tuning.warm_start = 2).
  double* hist[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  int* d_nhist = nullptr;
  double* staging = nullptr;
  size_t staging_elems = 0;
  BcOp* bc_out = nullptr;  // applyVelocityBC(enforceOutflow = true), phase 1
  BcOp* bc_in = nullptr;   // applyVelocityBC(enforceOutflow = false), phase 1
  BcOp* bc_solid = nullptr;  // phase 2: zero faces touching a solid
  int n_out = 0, n_in = 0, n_solid = 0, serial_out = 0, serial_in = 0;
  RedBuf rb{};
  StepBlock* d_blk = nullptr;  // per-step results (device)
  StepBlock* h_blk = nullptr;  // pinned host copy
  double* h_dt = nullptr;      // pinned dt staging
  GraphSlot graphs[2][2];      // [state parity][cfl dt]
  uint64_t body_kernels = 0;
  unsigned long long last_execs = 0;
  std::vector<void*> allocs;
  uint64_t bytes = 0;
  bool has_solid = false;
  uint64_t nfluid = 0;
  int rhs_grid = 592;  // CTAs of the momentum kernel (tuning)
  int step = 0;
  double t = 0.0, dt_last = 0.0;
  // ---- octree-AMR cases (the mesh outlives the case) ----
  bool amr = false;
  nb_amr_mesh* mesh = nullptr;
  AmrFaceMaps fm;
  AmrFlowView AF{};
  long long* d_sync[3] = {nullptr, nullptr, nullptr};
  int nsync[3] = {0, 0, 0};
  // a step launched and not yet waited for (nb_step_async / nb_step_wait)
  bool pending = false, pend_cfl = false, pend_direct = false;

  void* alloc(size_t n) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, n ? n : 16);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      throw ApiError{NB_ERR_OOM, "device allocation of " + std::to_string(n) + " bytes failed"};
    }
    allocs.push_back(q);
    bytes += n;
    return q;
  }
  ~nb_case() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& row : graphs)
      for (GraphSlot& g : row) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
      }
    for (void* q : allocs) cudaFree(q);
    if (h_blk) cudaFreeHost(h_blk);
    if (h_dt) cudaFreeHost(h_dt);
    mg.reset();
    if (stream) cudaStreamDestroy(stream);
  }
};

void nb::ensure_staging(nb_ctx* ctx, size_t elems) {
  if (ctx->stage_bytes >= elems * sizeof(double)) return;
  if (ctx->stage_a) cudaFree(ctx->stage_a);
  if (ctx->stage_b) cudaFree(ctx->stage_b);
  ctx->stage_a = ctx->stage_b = nullptr;
  ctx->stage_bytes = 0;
  NB_CUDA(cudaMalloc(&ctx->stage_a, elems * sizeof(double)));
  NB_CUDA(cudaMalloc(&ctx->stage_b, elems * sizeof(double)));
  ctx->stage_bytes = elems * sizeof(double);
}

namespace {

bool grid_ok(const nb_grid_desc* g, std::string& why) {
  if (!g) { why = "grid is NULL"; return false; }
  if (g->nx < 1 || g->ny < 1 || g->nz < 1) { why = "grid dimensions must be >= 1"; return false; }
  if (!(g->dx > 0.0) || !(g->dy > 0.0) || !(g->dz > 0.0)) { why = "grid spacing must be > 0"; return false; }
  if (static_cast<long long>(g->nx) * g->ny * g->nz > (1ll << 31) / 2) { why = "grid too large"; return false; }
  for (int f = 0; f < 6; ++f)
    if (g->face[f].type < NB_BC_WALL || g->face[f].type > NB_BC_PERIODIC) { why = "bad boundary type"; return false; }
  for (int a = 0; a < 3; ++a)
    if ((g->face[2 * a].type == NB_BC_PERIODIC) != (g->face[2 * a + 1].type == NB_BC_PERIODIC)) {
      why = "periodic faces must come in pairs";
      return false;
    }
  return true;
}

// Host mirror of the device storage index (brick slot or trailing slab).
long long h_cell(const HostLevel& L, int i, int j, int k) {
  const int b = L.lut[((k >> 3) * L.nby + (j >> 3)) * L.nbx + (i >> 3)];
  return static_cast<long long>(b) * BR3 + (((k & 7) << 6) | ((j & 7) << 3) | (i & 7));
}
long long h_face(const HostLevel& L, long long nb, int comp, int i, int j, int k) {
  if (comp == 0 && i == L.nx) return nb + j + static_cast<long long>(L.ny) * k;
  if (comp == 1 && j == L.ny) return nb + i + static_cast<long long>(L.nx) * k;
  if (comp == 2 && k == L.nz) return nb + i + static_cast<long long>(L.nx) * j;
  return h_cell(L, i, j, k);
}

// inletVelocityAt (core/src/flow/ns_solver.cpp:71-93)
double h_inlet(const nb_grid_desc& g, int face, int a, int comp) {
  const nb_face_bc& fb = g.face[face];
  double mag = fb.inlet_speed;
  if (fb.profile == NB_PROFILE_PARABOLIC) {
    const double H = g.ny * g.dy;
    const double yc = g.origin[1] + 0.5 * H;
    const double y = g.origin[1] + (a + 0.5) * g.dy;
    const double r = (y - yc) / (0.5 * H);
    mag = 1.5 * fb.inlet_speed * (1.0 - r * r);
  }
  return fb.inlet_axis == comp ? mag : 0.0;
}

bool h_solid(const nb_case& c, int i, int j, int k) {
  const nb_grid_desc& g = c.grid;
  if (i < 0 || i >= g.nx || j < 0 || j >= g.ny || k < 0 || k >= g.nz) return false;
  return c.solid[static_cast<size_t>(i) + static_cast<size_t>(g.nx) * (j + static_cast<size_t>(g.ny) * k)] != 0;
}

// applyVelocityBC (core/src/flow/ns_solver.cpp:221-309) as ordered face actions.
void build_bc(nb_case& c, bool outflow, std::vector<BcOp>& ops, std::vector<BcOp>& solid_ops) {
  const nb_grid_desc& g = c.grid;
  const HostLevel& L = c.mg->host0();
  const long long nb = c.F.nb;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  auto set = [&](int comp, long long idx, double v) { ops.push_back(BcOp{comp, 0, idx, 0, v}); };
  auto copy = [&](int comp, long long idx, long long src) { ops.push_back(BcOp{comp, 1, idx, src, 0.0}); };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int side = 0; side < 2; ++side) {
        const int face = side, i = side == 0 ? 0 : nx;
        const long long idx = h_face(L, nb, 0, i, j, k);
        switch (g.face[face].type) {
          case NB_BC_WALL: set(0, idx, 0.0); break;
          case NB_BC_INLET: set(0, idx, h_inlet(g, face, j, 0)); break;
          case NB_BC_OUTLET:
            if (outflow) copy(0, idx, h_face(L, nb, 0, side == 0 ? 1 : nx - 1, j, k));
            break;
          default: break;
        }
      }
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i)
      for (int side = 0; side < 2; ++side) {
        const int face = 2 + side, j = side == 0 ? 0 : ny;
        const long long idx = h_face(L, nb, 1, i, j, k);
        switch (g.face[face].type) {
          case NB_BC_WALL: set(1, idx, 0.0); break;
          case NB_BC_INLET: set(1, idx, h_inlet(g, face, i, 1)); break;
          case NB_BC_OUTLET:
            if (outflow) copy(1, idx, h_face(L, nb, 1, i, side == 0 ? 1 : ny - 1, k));
            break;
          default: break;
        }
      }
  if (nz > 1)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        for (int side = 0; side < 2; ++side) {
          const int face = 4 + side, k = side == 0 ? 0 : nz;
          const long long idx = h_face(L, nb, 2, i, j, k);
          switch (g.face[face].type) {
            case NB_BC_WALL: set(2, idx, 0.0); break;
            case NB_BC_INLET: set(2, idx, h_inlet(g, face, i, 2)); break;
            case NB_BC_OUTLET:
              if (outflow) copy(2, idx, h_face(L, nb, 2, i, j, side == 0 ? 1 : nz - 1));
              break;
            default: break;
          }
        }
  if (c.has_solid) {
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i)
          if (h_solid(c, i - 1, j, k) || h_solid(c, i, j, k))
            solid_ops.push_back(BcOp{0, 0, h_face(L, nb, 0, i, j, k), 0, 0.0});
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i)
          if (h_solid(c, i, j - 1, k) || h_solid(c, i, j, k))
            solid_ops.push_back(BcOp{1, 0, h_face(L, nb, 1, i, j, k), 0, 0.0});
    if (nz > 1)
      for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i)
            if (h_solid(c, i, j, k - 1) || h_solid(c, i, j, k))
              solid_ops.push_back(BcOp{2, 0, h_face(L, nb, 2, i, j, k), 0, 0.0});
  }
}

// A copy whose source is also written in the same list must run in order.
int needs_serial(const std::vector<BcOp>& ops) {
  std::map<std::pair<int, long long>, int> dst;
  for (const BcOp& o : ops) dst[{o.comp, o.idx}] = 1;
  for (const BcOp& o : ops)
    if (o.action == 1 && dst.count({o.comp, o.src})) return 1;
  return 0;
}

BcOp* upload_ops(nb_case& c, const std::vector<BcOp>& ops) {
  if (ops.empty()) return nullptr;
  BcOp* d = static_cast<BcOp*>(c.alloc(ops.size() * sizeof(BcOp)));
  NB_CUDA(cudaMemcpy(d, ops.data(), ops.size() * sizeof(BcOp), cudaMemcpyHostToDevice));
  return d;
}

void apply_bc(nb_case& c, double* const* f, bool outflow) {
  const int n = outflow ? c.n_out : c.n_in;
  if (n) {
    launch_bc(c.stream, outflow ? c.bc_out : c.bc_in, n, outflow ? c.serial_out : c.serial_in, f[0],
              f[1], f[2]);
    c.ctx->launches++;
  }
  if (c.n_solid) {
    launch_bc(c.stream, c.bc_solid, c.n_solid, 0, f[0], f[1], f[2]);
    c.ctx->launches++;
  }
}

// One flow-kernel launch: counted, and bracketed with events when profiled.
template <class Fn>
void flow_launch(nb_case& c, const char* fam, double bytes, Fn&& fn) {
  Profiler& P = c.ctx->prof;
  const bool on = P.on(fam);
  if (on) P.begin(c.stream);
  fn();
  if (on) P.end(c.stream, bytes);
  c.ctx->launches++;
}

double ncell_of(const nb_case& c) {
  if (c.amr) return static_cast<double>(c.fm.nbrick) * BR3;
  return static_cast<double>(c.grid.nx) * c.grid.ny * c.grid.nz;
}

void upload_lex(nb_case& c, int comp, const double* host, double* dst) {
  const long long n = lex_size(c.F, comp);
  NB_CUDA(cudaMemcpyAsync(c.staging, host, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  launch_convert(c.stream, c.F, comp, 0, c.staging, dst);
  c.ctx->launches++;
}

void download_lex(nb_case& c, int comp, const double* src, double* host) {
  const long long n = lex_size(c.F, comp);
  launch_convert(c.stream, c.F, comp, 1, src, c.staging);
  c.ctx->launches++;
  NB_CUDA(cudaMemcpyAsync(host, c.staging, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  NB_CUDA(cudaStreamSynchronize(c.stream));
}

// History of the stage pressures (mixed form only; 6 FP64 arrays per case).
void alloc_history(nb_case& c, size_t ncs) {
  if (c.precision != NB_PRECISION_MIXED) return;
  for (int st = 0; st < 3; ++st)
    for (int k = 0; k < 2; ++k) {
      c.hist[st][k] = static_cast<double*>(c.alloc(ncs * sizeof(double)));
      NB_CUDA(cudaMemset(c.hist[st][k], 0, ncs * sizeof(double)));
    }
  c.d_nhist = static_cast<int*>(c.alloc(2 * sizeof(int)));  // [0] steps held, [1] set_state's difference flag
  NB_CUDA(cudaMemset(c.d_nhist, 0, 2 * sizeof(int)));
}

// A new state makes the history meaningless (set_state, initialize, transfer).
void reset_history(nb_case& c) {
  if (c.d_nhist) NB_CUDA(cudaMemsetAsync(c.d_nhist, 0, sizeof(int), c.stream));
}

bool history_on(const nb_case& c) { return c.d_nhist && c.ctx->tune.warm_start >= 2; }

// Bitwise comparison of an uploaded array with the resident one: any
// difference (a NaN included) sets *differs.
__global__ void k_differs(long long n, const unsigned long long* __restrict__ a,
                          const unsigned long long* __restrict__ b, int* differs) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    if (a[i] != b[i]) {
      *differs = 1;
      return;
    }
}

__global__ void k_reset_if(const int* differs, int* nhist) {
  if (*differs) *nhist = 0;
}

// set_state of a case with a history: the state is uploaded into the scratch
// parity (and p into the rhs scratch), compared with the resident state, and
// the history cleared only if they differ; then the scratch becomes the
// state. A caller that reads the state back and uploads it unchanged (a host
// round trip every step) keeps the history.
void compare_and_swap_in(nb_case& c, size_t np) {
  const int nxt = 1 - c.cur;
  int* flag = c.d_nhist + 1;
  NB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), c.stream));
  for (int a = 0; a < 3; ++a) {
    const long long n = c.amr ? c.fm.store[a] : store_size(c.F, a);
    k_differs<<<148, 256, 0, c.stream>>>(n, reinterpret_cast<const unsigned long long*>(c.uvw[nxt][a]),
                                         reinterpret_cast<const unsigned long long*>(c.uvw[c.cur][a]), flag);
  }
  k_differs<<<148, 256, 0, c.stream>>>(static_cast<long long>(np), reinterpret_cast<const unsigned long long*>(c.b),
                                       reinterpret_cast<const unsigned long long*>(c.p), flag);
  k_reset_if<<<1, 1, 0, c.stream>>>(flag, c.d_nhist);
  c.ctx->launches += 5;
  NB_CUDA(cudaMemcpyAsync(c.p, c.b, np * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
  c.cur = nxt;
}

__global__ void k_history_tick(int* n) {
  if (*n < 2) *n += 1;
}

// After the correction of stage `stage` (p = phi / dt): latest -> previous,
// p -> latest.
void record_history(nb_case& c, int stage) {
  if (!history_on(c)) return;
  const size_t nbytes = static_cast<size_t>(ncell_of(c)) * sizeof(double);
  NB_CUDA(cudaMemcpyAsync(c.hist[stage][1], c.hist[stage][0], nbytes, cudaMemcpyDeviceToDevice, c.stream));
  NB_CUDA(cudaMemcpyAsync(c.hist[stage][0], c.p, nbytes, cudaMemcpyDeviceToDevice, c.stream));
}

// Mixed form with warm_start: the projection of RK stage `stage` starts from
// the pressure the last projection left (p = phi / dt), scaled to this
// stage's potential: the stage potentials are about dt P, dt P / 4 and
// 2 dt P / 3 for a pressure P (the divergence of the stage's u* is that of
// dt R, dt R / 4 and 2 dt R / 3), so p holds 2 P / 3 before stage 1 (the last
// step's stage 3), P before stage 2 and P / 4 before stage 3. The FP64 form
// starts from 0 as the reference does.
// With warm_start = 2 the stage's own pressures of the last two steps are
// extrapolated linearly in time (scaled by this step's dt) once the history
// holds them; until then the scaled last pressure above.
const WarmStart* warm_start(const nb_case& c, int stage, WarmStart* ws) {
  if (c.precision != NB_PRECISION_MIXED || !c.ctx->tune.warm_start) return nullptr;
  static constexpr double kAlpha[3] = {1.5, 0.25, 8.0 / 3.0};
  *ws = WarmStart{c.p, &c.d_blk->dt, kAlpha[stage]};
  if (history_on(c)) {
    ws->nhist = c.d_nhist;
    ws->h1 = c.hist[stage][0];
    if (c.ctx->tune.warm_start == 2) {  // 2 psi_s(n) - psi_s(n-1)
      ws->h2 = c.hist[stage][1];
      ws->k2 = -1.0;
      ws->h1 = c.hist[stage][0];
      ws->h3 = c.hist[stage][0];
      ws->k3 = 1.0;
    } else {  // psi_s(n) + alpha_s (p now - the previous stage's psi one step earlier)
      const int prev = (stage + 2) % 3;
      ws->h2 = c.hist[prev][0];
      ws->k2 = kAlpha[stage];
      ws->h3 = c.hist[prev][1];
      ws->k3 = -kAlpha[stage];
    }
  }
  return ws;
}

// NSSolver::project (core/src/flow/ns_solver.cpp:475-579) on the current fields.
// Graph form: the MG-PCG cycle loop is a device-side conditional node.
void project(nb_case& c, double* const* f, int stage, bool direct) {
  StepBlock* blk = c.d_blk;
  WarmStart wsv;
  const WarmStart* ws = warm_start(c, stage, &wsv);
  apply_bc(c, f, true);
  flow_launch(c, "div", ncell_of(c) * 33, [&] { launch_div(c.stream, c.F, f[0], f[1], f[2], c.b); });
  if (direct) {
    c.mg->solve_async(c.stream, c.b, c.cfg.poisson_tol, c.cfg.poisson_max_iters, blk->rep[stage], ws);
  } else {
    uint64_t nbody = 0;
    c.mg->capture_solve(c.stream, c.b, c.cfg.poisson_tol, c.cfg.poisson_max_iters, blk->rep[stage],
                        &nbody, ws);
    c.body_kernels = nbody;
  }
  flow_launch(c, "correct", ncell_of(c) * 65,
              [&] { launch_correct(c.stream, c.F, c.mg->phi(), &blk->dt, f[0], f[1], f[2], c.p); });
  record_history(c, stage);
  apply_bc(c, f, false);
}

double visc_of(const nb_case& c) {
  const nb_grid_desc& g = c.grid;
  const bool twoD = g.nz == 1;
  return 2.0 * c.nu * (1.0 / (g.dx * g.dx) + 1.0 / (g.dy * g.dy) + (twoD ? 0.0 : 1.0 / (g.dz * g.dz)));
}

double compute_dt(nb_case& c) {
  double* const* f = c.uvw[c.cur];
  if (c.amr) {
    flow_launch(c, "max_inv", ncell_of(c) * 25, [&] {
      launch_amr_max_inv(c.stream, c.AF, f[0], f[1], f[2], c.cfg.cfl, nullptr, c.rb, &c.d_blk->asc);
    });
  } else {
    flow_launch(c, "max_inv", ncell_of(c) * 25, [&] {
      launch_max_inv(c.stream, c.F, f[0], f[1], f[2], visc_of(c), c.cfg.cfl, nullptr, c.rb, &c.d_blk->sc);
    });
  }
  NB_CUDA(cudaMemcpyAsync(c.h_blk, c.d_blk, sizeof(StepBlock), cudaMemcpyDeviceToHost, c.stream));
  NB_CUDA(cudaStreamSynchronize(c.stream));
  return c.cfg.cfl / (c.amr ? c.h_blk->asc.maxinv : c.h_blk->sc.maxinv);
}

// ---- octree-AMR step ---------------------------------------------------------
// Derived coarse faces <- average of their fine sub-faces.
void amr_sync(nb_case& c, double* const* f) {
  for (int a = 0; a < 3; ++a)
    if (c.nsync[a])
      flow_launch(c, "sync", c.nsync[a] * 40.0, [&] { launch_amr_sync(c.stream, c.d_sync[a], c.nsync[a], f[a]); });
}

void amr_bc(nb_case& c, double* const* f, bool outflow) {
  apply_bc(c, f, outflow);
  amr_sync(c, f);
}

// NSSolver::project (ns_solver.cpp:475-579) on the composite mesh.
void project_amr(nb_case& c, double* const* f, int stage, bool direct) {
  StepBlock* blk = c.d_blk;
  WarmStart wsv;
  const WarmStart* ws = warm_start(c, stage, &wsv);
  amr_bc(c, f, true);
  flow_launch(c, "div", ncell_of(c) * 33, [&] { launch_amr_div(c.stream, c.AF, f[0], f[1], f[2], c.b); });
  if (direct) {
    c.mg->solve_async(c.stream, c.b, c.cfg.poisson_tol, c.cfg.poisson_max_iters, blk->rep[stage], ws);
  } else {
    uint64_t nbody = 0;
    c.mg->capture_solve(c.stream, c.b, c.cfg.poisson_tol, c.cfg.poisson_max_iters, blk->rep[stage],
                        &nbody, ws);
    c.body_kernels = nbody;
  }
  flow_launch(c, "correct", ncell_of(c) * 65,
              [&] { launch_amr_correct(c.stream, c.AF, c.mg->phi(), &blk->dt, f[0], f[1], f[2], c.p); });
  record_history(c, stage);
  amr_bc(c, f, false);
}

void issue_step_amr(nb_case& c, int cur, bool cfl_dt, bool direct) {
  StepBlock* blk = c.d_blk;
  double** A = c.uvw[cur];
  double** B = c.uvw[1 - cur];
  if (cfl_dt)
    flow_launch(c, "max_inv", ncell_of(c) * 25, [&] {
      launch_amr_max_inv(c.stream, c.AF, A[0], A[1], A[2], c.cfg.cfl, &blk->dt, c.rb, &blk->asc);
    });
  for (int q = 0; q < 3; ++q)
    NB_CUDA(cudaMemcpyAsync(c.uvw0[q], A[q], static_cast<size_t>(c.fm.store[q]) * 8, cudaMemcpyDeviceToDevice,
                            c.stream));
  amr_bc(c, A, true);
  const int mixed = c.precision == NB_PRECISION_MIXED;
  for (int stage = 1; stage <= 3; ++stage) {
    double** in = (stage == 2) ? B : A;
    double** out = (stage == 2) ? A : B;
    flow_launch(c, "rhs_rk", ncell_of(c) * 73, [&] {
      launch_amr_rhs_rk(c.stream, c.AF, stage, &blk->dt, in[0], in[1], in[2], c.uvw0[0], c.uvw0[1], c.uvw0[2],
                        out[0], out[1], out[2], mixed, c.rhs_grid);
    });
    amr_sync(c, out);
    project_amr(c, out, stage - 1, direct);
  }
  flow_launch(c, "diag", ncell_of(c) * 49, [&] {
    launch_amr_diag(c.stream, c.AF, B[0], B[1], B[2], c.uvw0[0], c.uvw0[1], c.uvw0[2], c.rb, &blk->asc);
  });
  NB_CUDA(cudaMemcpyAsync(&blk->execs, c.mg->body_execs(), sizeof(unsigned long long),
                          cudaMemcpyDeviceToDevice, c.stream));
  if (history_on(c)) {
    k_history_tick<<<1, 1, 0, c.stream>>>(c.d_nhist);
    c.ctx->launches++;
  }
}

// Issues one SSP-RK3 step (NSSolver::step, core/src/flow/ns_solver.cpp:765-824)
// starting from state parity `cur`. cfl_dt: dt = computeDt() on the device.
void issue_step(nb_case& c, int cur, bool cfl_dt, bool direct) {
  if (c.amr) {
    issue_step_amr(c, cur, cfl_dt, direct);
    return;
  }
  StepBlock* blk = c.d_blk;
  double** A = c.uvw[cur];
  double** B = c.uvw[1 - cur];
  if (cfl_dt)
    flow_launch(c, "max_inv", ncell_of(c) * 25, [&] {
      launch_max_inv(c.stream, c.F, A[0], A[1], A[2], visc_of(c), c.cfg.cfl, &blk->dt, c.rb, &blk->sc);
    });
  for (int q = 0; q < 3; ++q)
    NB_CUDA(cudaMemcpyAsync(c.uvw0[q], A[q], static_cast<size_t>(store_size(c.F, q)) * 8,
                            cudaMemcpyDeviceToDevice, c.stream));
  apply_bc(c, A, true);
  const int mixed = c.precision == NB_PRECISION_MIXED;
  for (int stage = 1; stage <= 3; ++stage) {
    double** in = (stage == 2) ? B : A;
    double** out = (stage == 2) ? A : B;
    flow_launch(c, "rhs_rk", ncell_of(c) * 73, [&] {
      launch_rhs_rk(c.stream, c.F, stage, &blk->dt, in[0], in[1], in[2], c.uvw0[0], c.uvw0[1], c.uvw0[2],
                    out[0], out[1], out[2], mixed, c.rhs_grid);
    });
    project(c, out, stage - 1, direct);
  }
  flow_launch(c, "diag", ncell_of(c) * 57, [&] {
    launch_diag(c.stream, c.F, B[0], B[1], B[2], c.uvw0[0], c.uvw0[1], c.uvw0[2], c.p, c.rb, &blk->sc);
  });
  NB_CUDA(cudaMemcpyAsync(&blk->execs, c.mg->body_execs(), sizeof(unsigned long long),
                          cudaMemcpyDeviceToDevice, c.stream));
  if (history_on(c)) {
    k_history_tick<<<1, 1, 0, c.stream>>>(c.d_nhist);
    c.ctx->launches++;
  }
}

void finish_step(nb_case& c, nb_step_report* rep);

// One step. Without profiling the step runs as one CUDA graph (built on first
// use per state parity and dt mode): one launch and one small read-back per step.
// launch_step issues it on the case stream; complete_step waits and finishes.
void launch_step(nb_case& c, double dt) {
  const bool cfl_dt = dt <= 0.0;
  if (!cfl_dt) {
    c.h_dt[0] = dt;
    NB_CUDA(cudaMemcpyAsync(&c.d_blk->dt, c.h_dt, sizeof(double), cudaMemcpyHostToDevice, c.stream));
  }
  const bool direct = !c.ctx->prof.family.empty();
  if (direct) {
    issue_step(c, c.cur, cfl_dt, true);
  } else {
    GraphSlot& gs = c.graphs[c.cur][cfl_dt ? 1 : 0];
    if (!gs.exec) {
      const uint64_t before = c.ctx->launches;
      NB_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
      try {
        issue_step(c, c.cur, cfl_dt, false);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(c.stream, &g);
        if (g) cudaGraphDestroy(g);
        c.ctx->launches = before;
        throw;
      }
      NB_CUDA(cudaStreamEndCapture(c.stream, &gs.graph));
      NB_CUDA(cudaGraphInstantiate(&gs.exec, gs.graph, 0));
      gs.fixed_kernels = c.ctx->launches - before;
      gs.body_kernels = c.body_kernels;
      c.ctx->launches = before;
    }
    NB_CUDA(cudaGraphLaunch(gs.exec, c.stream));
  }
  NB_CUDA(cudaMemcpyAsync(c.h_blk, c.d_blk, sizeof(StepBlock), cudaMemcpyDeviceToHost, c.stream));
  c.pending = true;
  c.pend_cfl = cfl_dt;
  c.pend_direct = direct;
}

void complete_step(nb_case& c, nb_step_report* rep) {
  NB_CUDA(cudaStreamSynchronize(c.stream));
  c.pending = false;
  if (!c.pend_direct) {
    const GraphSlot& gs = c.graphs[c.cur][c.pend_cfl ? 1 : 0];
    c.ctx->launches += gs.fixed_kernels + (c.h_blk->execs - c.last_execs) * gs.body_kernels;
  }
  finish_step(c, rep);
}

void do_step(nb_case& c, double dt, nb_step_report* rep) {
  launch_step(c, dt);
  complete_step(c, rep);
}

// True when a bounded device-side wait of the step's pressure solves gave up
// (a grid-resident V-cycle's barrier, stop code STOP_TIMEOUT).
bool step_timed_out(const nb_case& c) {
  for (int s = 0; s < 3; ++s)
    if (c.h_blk->rep[s][1] == static_cast<double>(STOP_TIMEOUT)) return true;
  return false;
}

// Host side of a finished step once c.h_blk holds its results: clock, state
// parity and the StepReport (ns_solver.cpp:797-823).
void finish_step(nb_case& c, nb_step_report* rep) {
  const StepBlock& hb = *c.h_blk;
  c.last_execs = hb.execs;
  const double dt = hb.dt;
  c.cur = 1 - c.cur;  // the stage-3 output is the new state
  c.step += 1;
  c.t += dt;
  c.dt_last = dt;
  if (!rep) return;
  nb_poisson_report pr[3];
  for (int s = 0; s < 3; ++s) pr[s] = MgSolver::report_from(hb.rep[s], c.cfg.poisson_tol);
  const nb_grid_desc& g = c.grid;
  const double nfaces =
      c.amr ? static_cast<double>(c.fm.owned[0] + c.fm.owned[1] + c.fm.owned[2])
            : static_cast<double>(lex_size(c.F, 0) + lex_size(c.F, 1) + lex_size(c.F, 2));
  StepScalars sc = hb.sc;
  if (c.amr) {
    sc = StepScalars{};
    sc.du2 = hb.asc.du2;
    sc.div2 = hb.asc.div2;
    sc.divmax = hb.asc.divmax;
    sc.mass = hb.asc.mass;
  }
  std::memset(rep, 0, sizeof(*rep));
  rep->step = c.step;
  rep->t = c.t;
  rep->dt = dt;
  rep->cfl = c.cfg.cfl;
  rep->momentum_residual = std::sqrt(sc.du2 / nfaces) / (dt * c.cfg.velocity_scale + 1e-300);
  rep->continuity_residual = c.nfluid ? std::sqrt(sc.div2 / static_cast<double>(c.nfluid)) : 0.0;
  rep->divergence_max = sc.divmax;
  const double ay = g.dx * g.dz;
  rep->mass_error = std::fabs(sc.mass) / (c.cfg.velocity_scale * (g.ny * ay) + 1e-300);
  rep->poisson_iters = pr[0].iterations + pr[1].iterations + pr[2].iterations;
  rep->poisson_residual = std::max(pr[0].residual, std::max(pr[1].residual, pr[2].residual));
  rep->converged = pr[0].converged && pr[1].converged && pr[2].converged;
  if (c.has_solid && !c.amr) {
    double aref = c.cfg.ref_area;
    if (aref <= 0.0) aref = c.cfg.ref_length * c.cfg.ref_length;
    const double q = 0.5 * c.cfg.density * c.cfg.velocity_scale * c.cfg.velocity_scale * aref + 1e-300;
    rep->cd = sc.fx / q;
    rep->cl = sc.fy / q;
  }
  rep->cell_count = c.amr ? static_cast<uint64_t>(c.fm.nbrick) * BR3 : static_cast<uint64_t>(g.nx) * g.ny * g.nz;
  rep->accepted = (rep->continuity_residual < c.cfg.tol_continuity && rep->mass_error < c.cfg.tol_mass) ? 1 : 0;
}

// ---- batches: one graph per step of a set of cases ---------------------------
void destroy_batch(BatchGraph& bg) {
  if (bg.exec) cudaGraphExecDestroy(bg.exec);
  if (bg.graph) cudaGraphDestroy(bg.graph);
  bg.exec = nullptr;
  bg.graph = nullptr;
}

void drop_batches_with(nb_ctx* ctx, const nb_case* c) {
  const uintptr_t id = reinterpret_cast<uintptr_t>(c);
  for (auto it = ctx->batch_cache.begin(); it != ctx->batch_cache.end();) {
    bool has = false;
    for (size_t q = 0; q < it->first.size(); q += 3) has = has || it->first[q] == id;
    if (has) {
      destroy_batch(it->second);
      it = ctx->batch_cache.erase(it);
    } else {
      ++it;
    }
  }
}

// One step of every case, as one graph: each case's whole step (its CFL dt or
// the fixed dt already in its step block, its three projections with their
// device-side MG-PCG loops, the report copy) is a branch captured from the
// case's own stream between a fork and a join on the context stream.
void batch_step(nb_ctx* ctx, nb_case* const* cs, int n, bool cfl_dt, nb_step_report* reps) {
  std::vector<uintptr_t> key;
  key.reserve(3 * static_cast<size_t>(n));
  for (int q = 0; q < n; ++q) {
    key.push_back(reinterpret_cast<uintptr_t>(cs[q]));
    key.push_back(static_cast<uintptr_t>(cs[q]->cur));
    key.push_back(cfl_dt ? 1u : 0u);
  }
  auto it = ctx->batch_cache.find(key);
  if (it == ctx->batch_cache.end()) {
    BatchGraph bg;
    cudaEvent_t ev = nullptr;
    NB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    const uint64_t before = ctx->launches;
    NB_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    try {
      NB_CUDA(cudaEventRecord(ev, ctx->stream));
      for (int q = 0; q < n; ++q) {
        nb_case& c = *cs[q];
        NB_CUDA(cudaStreamWaitEvent(c.stream, ev, 0));
        issue_step(c, c.cur, cfl_dt, false);
        bg.body_kernels.push_back(c.body_kernels);
        NB_CUDA(cudaMemcpyAsync(c.h_blk, c.d_blk, sizeof(StepBlock), cudaMemcpyDeviceToHost, c.stream));
      }
      for (int q = 0; q < n; ++q) {
        NB_CUDA(cudaEventRecord(ev, cs[q]->stream));
        NB_CUDA(cudaStreamWaitEvent(ctx->stream, ev, 0));
      }
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(ctx->stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaEventDestroy(ev);
      ctx->launches = before;
      throw;
    }
    NB_CUDA(cudaStreamEndCapture(ctx->stream, &bg.graph));
    cudaEventDestroy(ev);
    const cudaError_t e = cudaGraphInstantiate(&bg.exec, bg.graph, 0);
    if (e != cudaSuccess) {
      destroy_batch(bg);
      ctx->launches = before;
      NB_CUDA(e);
    }
    bg.fixed_kernels = ctx->launches - before;
    ctx->launches = before;
    it = ctx->batch_cache.emplace(key, std::move(bg)).first;
  }
  NB_CUDA(cudaGraphLaunch(it->second.exec, ctx->stream));
  NB_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->launches += it->second.fixed_kernels;
  for (int q = 0; q < n; ++q)
    ctx->launches += (cs[q]->h_blk->execs - cs[q]->last_execs) * it->second.body_kernels[q];
  for (int q = 0; q < n; ++q) finish_step(*cs[q], reps ? &reps[q] : nullptr);
}

MgSolver& ctx_solver(nb_ctx* ctx, const nb_grid_desc& g, int precision) {
  const auto key = std::make_pair(grid_signature(g), precision);
  auto it = ctx->mg_cache.find(key);
  if (it == ctx->mg_cache.end()) {
    auto s = std::make_unique<MgSolver>(g, precision, LaunchCounter{&ctx->launches, &ctx->prof}, &ctx->tune);
    it = ctx->mg_cache.emplace(key, std::move(s)).first;
  }
  return *it->second;
}

FlowView cell_view(const MgSolver& mg) {
  FlowView F{};
  F.L = mg.view0();
  F.nb = static_cast<long long>(F.L.nbrick) * BR3;
  return F;
}

}  // namespace

void nb::ctx_release(nb_ctx* ctx) {
  if (ctx->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->batch_cache) destroy_batch(kv.second);
  ctx->batch_cache.clear();
  ctx->mg_cache.clear();
  if (ctx->stage_a) cudaFree(ctx->stage_a);
  if (ctx->stage_b) cudaFree(ctx->stage_b);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

void nb::case_kind(const nb_case* c, int* amr, int* precision, int* levels) {
  *amr = c->amr ? 1 : 0;
  *precision = c->precision;
  *levels = c->amr ? c->mesh->lvl.tree.nlev : 1;
}

nb_ctx* nb::case_ctx(const nb_case* c) { return c->ctx; }

void nb::case_dims(const nb_case* c, int dims[3]) {
  dims[0] = c->grid.nx;
  dims[1] = c->grid.ny;
  dims[2] = c->grid.nz;
}

nb_amr_mesh* nb::case_mesh(const nb_case* c) { return c->amr ? c->mesh : nullptr; }

void nb::case_set_clock(nb_case* c, int step, double t, double dt_last) {
  c->step = step;
  c->t = t;
  c->dt_last = dt_last;
}

std::vector<uint8_t> nb::case_solid(const nb_case* c) {
  if (!c->amr) return c->solid;
  const std::vector<uint8_t>& ty = c->mesh->lvl.type;
  std::vector<uint8_t> out(ty.size());
  for (size_t q = 0; q < ty.size(); ++q) out[q] = ty[q] == CELL_SOLID ? 1 : 0;
  return out;
}

const nb_grid_desc& nb::case_grid(const nb_case* c) { return c->grid; }

nb_status nb::clone_case(nb_case* src, nb_case** out) {
  nb_ctx* ctx = src->ctx;
  nb_case* c = nullptr;
  nb_status st = src->amr ? nb_amr_case_create(ctx, src->mesh, &src->cfg, src->precision, &c)
                          : nb_case_create(ctx, &src->grid, &src->cfg, src->precision, &c);
  if (st != NB_OK) return st;
  // the current state, through the public accessors (host round trip)
  std::vector<double> f[4];
  if (src->amr) {
    int64_t sz[4];
    st = nb_amr_case_sizes(src, sz);
    for (int q = 0; q < 4 && st == NB_OK; ++q) f[q].resize(static_cast<size_t>(sz[q]));
    if (st == NB_OK) st = nb_amr_case_get_state(src, f[0].data(), f[1].data(), f[2].data(), f[3].data());
    if (st == NB_OK) st = nb_amr_case_set_state(c, f[0].data(), f[1].data(), f[2].data(), f[3].data());
  } else {
    const size_t nx = src->grid.nx, ny = src->grid.ny, nz = src->grid.nz;
    f[0].resize((nx + 1) * ny * nz);
    f[1].resize(nx * (ny + 1) * nz);
    f[2].resize(nx * ny * (nz + 1));
    f[3].resize(nx * ny * nz);
    st = nb_case_get_state(src, f[0].data(), f[1].data(), f[2].data(), f[3].data());
    if (st == NB_OK)
      st = nb_case_set_state(c, f[0].data(), f[1].data(), f[2].data(), f[3].data(), src->step, src->t, src->dt_last);
  }
  if (st != NB_OK) {
    nb_case_destroy(c);
    return st;
  }
  *out = c;
  return NB_OK;
}

extern "C" {

const char* nb_status_string(nb_status s) {
  switch (s) {
    case NB_OK: return "ok";
    case NB_ERR_BAD_ARG: return "bad argument";
    case NB_ERR_OOM: return "out of device memory";
    case NB_ERR_NOT_CONVERGED: return "not converged";
    case NB_ERR_NAN: return "NaN detected";
    case NB_ERR_DEVICE_TIMEOUT: return "device wait timed out";
    case NB_ERR_CUDA: return "CUDA error";
    case NB_ERR_UNSUPPORTED: return "unsupported configuration";
  }
  return "unknown status";
}

nb_status nb_ctx_create(int device, nb_ctx** out) {
  if (!out) return NB_ERR_BAD_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    (void)cudaGetLastError();
    return NB_ERR_CUDA;
  }
  if (device < 0 || device >= n) return NB_ERR_BAD_ARG;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) return NB_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return NB_ERR_CUDA;
  auto* ctx = new nb_ctx();
  ctx->device = device;
  nb_tuning_default(&ctx->tune);
  const nb_status s = guarded(ctx, [&] {
    NB_CUDA(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device));
    NB_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    flow_kernel_setup();
    amr_flow_setup();
    return NB_OK;
  });
  if (s != NB_OK) {
    delete ctx;
    return s;
  }
  *out = ctx;
  return NB_OK;
}

void nb_ctx_destroy(nb_ctx* ctx) {
  if (ctx) ctx_release(ctx);
}

const char* nb_last_error(const nb_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

uint64_t nb_ctx_launch_count(const nb_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

void* nb_ctx_stream(const nb_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

nb_status nb_ctx_synchronize(nb_ctx* ctx) {
  if (!ctx) return NB_ERR_BAD_ARG;
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    NB_CUDA(cudaDeviceSynchronize());
    return NB_OK;
  });
}

nb_status nb_case_create(nb_ctx* ctx, const nb_grid_desc* grid, const nb_flow_config* cfg,
                         int precision, nb_case** out) {
  if (!ctx || !out || !cfg) return NB_ERR_BAD_ARG;
  *out = nullptr;
  std::string why;
  if (!grid_ok(grid, why)) return fail(ctx, NB_ERR_BAD_ARG, why);
  if (precision != NB_PRECISION_FP64 && precision != NB_PRECISION_MIXED)
    return fail(ctx, NB_ERR_BAD_ARG, "precision must be NB_PRECISION_FP64 or NB_PRECISION_MIXED");
  if (!(cfg->reynolds > 0.0)) return fail(ctx, NB_ERR_BAD_ARG, "reynolds must be > 0");
  auto c = std::make_unique<nb_case>();
  c->ctx = ctx;
  const nb_status s = guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    NB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->grid = *grid;
    const size_t ncell = static_cast<size_t>(grid->nx) * grid->ny * grid->nz;
    c->solid.assign(ncell, 0);
    if (grid->solid) std::memcpy(c->solid.data(), grid->solid, ncell);
    c->grid.solid = c->solid.data();
    c->cfg = *cfg;
    c->precision = precision;
    c->nu = cfg->velocity_scale * cfg->ref_length / cfg->reynolds;  // ns_solver.cpp:54
    for (uint8_t v : c->solid)
      if (v) { c->has_solid = true; break; }
    c->mg = std::make_unique<MgSolver>(c->grid, precision, LaunchCounter{&ctx->launches, &ctx->prof}, &ctx->tune);
    c->rhs_grid = std::min(std::max(ctx->tune.rhs_ctas_per_sm, 1), 4) * ctx->nsm;
    c->nfluid = c->mg->host0().nfluid;
    FlowView& F = c->F;
    F.L = c->mg->view0();
    F.nb = static_cast<long long>(F.L.nbrick) * BR3;
    for (int a = 0; a < 3; ++a) F.origin[a] = grid->origin[a];
    for (int f = 0; f < 6; ++f) {
      for (int a = 0; a < 3; ++a) F.wallv[f][a] = grid->face[f].wall_velocity[a];
      F.inlet_speed[f] = grid->face[f].inlet_speed;
      F.profile[f] = grid->face[f].profile;
      F.inlet_axis[f] = grid->face[f].inlet_axis;
    }
    for (int a = 0; a < 3; ++a) F.per[a] = grid->face[2 * a].type == NB_BC_PERIODIC;
    F.weno = cfg->convection == NB_CONV_WENO5;
    F.has_solid = c->has_solid;
    F.nu = c->nu;
    for (int a = 0; a < 3; ++a) F.bf[a] = cfg->body_force[a];
    F.density = cfg->density;
    F.velocity_scale = cfg->velocity_scale;
    for (int h = 0; h < 2; ++h)
      for (int q = 0; q < 3; ++q) {
        const size_t nb = static_cast<size_t>(store_size(F, q)) * sizeof(double);
        c->uvw[h][q] = static_cast<double*>(c->alloc(nb));
        NB_CUDA(cudaMemset(c->uvw[h][q], 0, nb));
      }
    for (int q = 0; q < 3; ++q) {
      const size_t nb = static_cast<size_t>(store_size(F, q)) * sizeof(double);
      c->uvw0[q] = static_cast<double*>(c->alloc(nb));
      NB_CUDA(cudaMemset(c->uvw0[q], 0, nb));
    }
    const size_t ncs = static_cast<size_t>(F.nb);
    c->p = static_cast<double*>(c->alloc(ncs * sizeof(double)));
    c->b = static_cast<double*>(c->alloc(ncs * sizeof(double)));
    NB_CUDA(cudaMemset(c->p, 0, ncs * sizeof(double)));
    NB_CUDA(cudaMemset(c->b, 0, ncs * sizeof(double)));
    alloc_history(*c, ncs);
    c->staging_elems = static_cast<size_t>(std::max({lex_size(F, 0), lex_size(F, 1), lex_size(F, 2)}));
    c->staging = static_cast<double*>(c->alloc(c->staging_elems * sizeof(double)));
    std::vector<BcOp> out_ops, in_ops, solid_ops, dummy;
    build_bc(*c, true, out_ops, solid_ops);
    build_bc(*c, false, in_ops, dummy);
    c->n_out = static_cast<int>(out_ops.size());
    c->n_in = static_cast<int>(in_ops.size());
    c->n_solid = static_cast<int>(solid_ops.size());
    c->serial_out = needs_serial(out_ops);
    c->serial_in = needs_serial(in_ops);
    c->bc_out = upload_ops(*c, out_ops);
    c->bc_in = upload_ops(*c, in_ops);
    c->bc_solid = upload_ops(*c, solid_ops);
    c->rb.max_blocks = 148 * 4;
    c->rb.partials = static_cast<double*>(c->alloc(RED_KMAX * c->rb.max_blocks * sizeof(double)));
    c->rb.counter = static_cast<unsigned*>(c->alloc(sizeof(unsigned)));
    NB_CUDA(cudaMemset(c->rb.counter, 0, sizeof(unsigned)));
    c->d_blk = static_cast<StepBlock*>(c->alloc(sizeof(StepBlock)));
    NB_CUDA(cudaMemset(c->d_blk, 0, sizeof(StepBlock)));
    NB_CUDA(cudaMallocHost(&c->h_blk, sizeof(StepBlock)));
    NB_CUDA(cudaMallocHost(&c->h_dt, sizeof(double)));
    // the uploads and memsets above ran on the legacy stream; the case's own
    // stream is non-blocking, so steps of other cases keep running meanwhile
    NB_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    return NB_OK;
  });
  if (s != NB_OK) return s;
  ctx_retain(ctx);
  *out = c.release();
  return NB_OK;
}

void nb_case_destroy(nb_case* c) {
  if (!c) return;
  cudaSetDevice(c->ctx->device);
  if (c->ctx->stream) cudaStreamSynchronize(c->ctx->stream);
  drop_batches_with(c->ctx, c);
  nb_ctx* ctx = c->ctx;
  delete c;
  ctx_release(ctx);
}

// Steps every case of `cases` nsteps times; each step of all of them is one
// CUDA graph launch (see batch_step).
nb_status nb_batch_step(nb_ctx* ctx, nb_case* const* cases, int n, double dt, int nsteps,
                        nb_step_report* reports) {
  if (!ctx || !cases || n <= 0 || nsteps < 0) return NB_ERR_BAD_ARG;
  for (int q = 0; q < n; ++q) {
    if (!cases[q] || cases[q]->ctx != ctx) return fail(ctx, NB_ERR_BAD_ARG, "batch cases must belong to the context");
    if (cases[q]->pending) return fail(ctx, NB_ERR_BAD_ARG, "a batch case has a step in flight");
    for (int r = 0; r < q; ++r)
      if (cases[r] == cases[q]) return fail(ctx, NB_ERR_BAD_ARG, "a case appears twice in the batch");
  }
  if (!ctx->prof.family.empty()) return fail(ctx, NB_ERR_UNSUPPORTED, "batch steps run as graphs: switch profiling off");
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    const bool cfl_dt = dt <= 0.0;
    for (int s = 0; s < nsteps; ++s) {
      if (!cfl_dt)
        for (int q = 0; q < n; ++q) {
          cases[q]->h_dt[0] = dt;
          NB_CUDA(cudaMemcpyAsync(&cases[q]->d_blk->dt, cases[q]->h_dt, sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream));
        }
      batch_step(ctx, cases, n, cfl_dt, reports);
    }
    for (int q = 0; q < n; ++q)
      if (step_timed_out(*cases[q])) return fail(ctx, NB_ERR_DEVICE_TIMEOUT, "a device-side barrier wait gave up");
    if (reports)
      for (int q = 0; q < n; ++q)
        if (std::isnan(reports[q].momentum_residual)) return fail(ctx, NB_ERR_NAN, "NaN in the step diagnostics");
    return NB_OK;
  });
}

uint64_t nb_case_device_bytes(const nb_case* c) {
  return c ? c->bytes + c->mg->device_bytes() : 0;
}

void* nb_case_stream(const nb_case* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

nb_status nb_ctx_profile(nb_ctx* ctx, const char* family) {
  if (!ctx) return NB_ERR_BAD_ARG;
  ctx->prof.family = family ? family : "";
  return NB_OK;
}

nb_status nb_ctx_profile_read(nb_ctx* ctx, double* total_ms, uint64_t* launches, double* bytes) {
  if (!ctx) return NB_ERR_BAD_ARG;
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    const double ms = ctx->prof.drain(launches, bytes);
    if (total_ms) *total_ms = ms;
    return NB_OK;
  });
}

uint64_t nb_case_cell_count(const nb_case* c) {
  if (c && c->amr) return static_cast<uint64_t>(c->fm.nbrick) * BR3;
  return c ? static_cast<uint64_t>(c->grid.nx) * c->grid.ny * c->grid.nz : 0;
}

nb_status nb_case_set_state(nb_case* c, const double* u, const double* v, const double* w,
                            const double* p, int step, double t, double dt_last) {
  if (!c || !u || !v || !w || !p) return NB_ERR_BAD_ARG;
  if (c->amr) return fail(c->ctx, NB_ERR_UNSUPPORTED, "AMR cases take nb_amr_case_set_state");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    const bool keep = c->d_nhist != nullptr;  // stage, compare, then swap in
    double** f = c->uvw[keep ? 1 - c->cur : c->cur];
    upload_lex(*c, 0, u, f[0]);
    upload_lex(*c, 1, v, f[1]);
    upload_lex(*c, 2, w, f[2]);
    upload_lex(*c, 3, p, keep ? c->b : c->p);
    if (keep) compare_and_swap_in(*c, static_cast<size_t>(c->F.nb));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    c->step = step;
    c->t = t;
    c->dt_last = dt_last;
    return NB_OK;
  });
}

nb_status nb_case_get_state(nb_case* c, double* u, double* v, double* w, double* p) {
  if (!c) return NB_ERR_BAD_ARG;
  if (c->amr) return fail(c->ctx, NB_ERR_UNSUPPORTED, "AMR cases take nb_amr_case_get_state");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    double** f = c->uvw[c->cur];
    if (u) download_lex(*c, 0, f[0], u);
    if (v) download_lex(*c, 1, f[1], v);
    if (w) download_lex(*c, 2, f[2], w);
    if (p) download_lex(*c, 3, c->p, p);
    return NB_OK;
  });
}

nb_status nb_case_get_clock(nb_case* c, int* step, double* t, double* dt_last) {
  if (!c) return NB_ERR_BAD_ARG;
  if (step) *step = c->step;
  if (t) *t = c->t;
  if (dt_last) *dt_last = c->dt_last;
  return NB_OK;
}

// NSSolver::initialize (core/src/flow/ns_solver.cpp:95-112)
nb_status nb_case_initialize(nb_case* c) {
  if (!c) return NB_ERR_BAD_ARG;
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    reset_history(*c);
    if (c->amr) {  // zero interior, inlet speed on u as the initial guess
      double s = 0.0;
      for (int f = 0; f < 6; ++f)
        if (c->grid.face[f].type == NB_BC_INLET && c->grid.face[f].inlet_axis == 0) {
          s = c->grid.face[f].inlet_speed;
          break;
        }
      double** fl = c->uvw[c->cur];
      for (int a = 0; a < 3; ++a) {
        std::vector<double> F0(static_cast<size_t>(c->fm.store[a]), a == 0 ? s : 0.0);
        NB_CUDA(cudaMemcpyAsync(fl[a], F0.data(), F0.size() * 8, cudaMemcpyHostToDevice, c->stream));
        NB_CUDA(cudaStreamSynchronize(c->stream));
      }
      NB_CUDA(cudaMemsetAsync(c->p, 0, static_cast<size_t>(c->fm.nbrick) * BR3 * 8, c->stream));
      amr_bc(*c, fl, true);
      NB_CUDA(cudaStreamSynchronize(c->stream));
      c->step = 0;
      c->t = 0.0;
      c->dt_last = 0.0;
      return NB_OK;
    }
    const long long nu = lex_size(c->F, 0), nv = lex_size(c->F, 1), nw = lex_size(c->F, 2),
                    np = lex_size(c->F, 3);
    std::vector<double> U(nu, 0.0), V(nv, 0.0), W(nw, 0.0), P(np, 0.0);
    for (int f = 0; f < 6; ++f)
      if (c->grid.face[f].type == NB_BC_INLET && c->grid.face[f].inlet_axis == 0) {
        std::fill(U.begin(), U.end(), c->grid.face[f].inlet_speed);
        break;
      }
    double** fl = c->uvw[c->cur];
    upload_lex(*c, 0, U.data(), fl[0]);
    upload_lex(*c, 1, V.data(), fl[1]);
    upload_lex(*c, 2, W.data(), fl[2]);
    upload_lex(*c, 3, P.data(), c->p);
    apply_bc(*c, fl, true);
    NB_CUDA(cudaStreamSynchronize(c->stream));
    c->step = 0;
    c->t = 0.0;
    c->dt_last = 0.0;
    return NB_OK;
  });
}

// Per-brick refinement sensors of an octree case (host array nleaf x 4).
nb_status nb_amr_case_sensors(nb_case* c, double* out) {
  if (!c || !c->amr || !out) return NB_ERR_BAD_ARG;
  if (c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "nb_amr_case_sensors: the case has a step in flight");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    const size_t n = static_cast<size_t>(c->fm.nbrick) * 4;
    ensure_staging(c->ctx, n);
    double** f = c->uvw[c->cur];
    launch_amr_sensors(c->stream, c->AF, f[0], f[1], f[2], c->p, c->ctx->stage_a);
    ++c->ctx->launches;
    NB_CUDA(cudaMemcpyAsync(out, c->ctx->stage_a, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NB_OK;
  });
}

nb_status nb_amr_case_refine(nb_case* c, int sensor, double above, int32_t* out, int64_t cap, int64_t* n_out) {
  if (!c || !c->amr || sensor < 0 || sensor > 3 || !n_out) return NB_ERR_BAD_ARG;
  if (c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "nb_amr_case_refine: the case has a step in flight");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    const int n = c->fm.nbrick;
    ensure_staging(c->ctx, static_cast<size_t>(n) * 4);
    double** f = c->uvw[c->cur];
    launch_amr_sensors(c->stream, c->AF, f[0], f[1], f[2], c->p, c->ctx->stage_a);
    ++c->ctx->launches;
    const auto& L = c->mesh->lvl.tree.leaves;
    std::vector<int32_t> h(4 * static_cast<size_t>(n));
    for (int r = 0; r < n; ++r) {
      h[4 * r] = L[r].level;
      for (int a = 0; a < 3; ++a) h[4 * r + 1 + a] = L[r].b[a];
    }
    refine_from_sensors(c->ctx, c->stream, c->mesh->geom, h.data(), n, c->ctx->stage_a, sensor, above, out, cap,
                        n_out);
    return NB_OK;
  });
}

namespace {
bool same_geometry(const nb_amr_geom& a, const nb_amr_geom& b) {
  for (int q = 0; q < 3; ++q)
    if (a.nb0[q] != b.nb0[q] || a.h0[q] != b.h0[q] || a.origin[q] != b.origin[q]) return false;
  for (int f = 0; f < 6; ++f)
    if (a.face[f].type != b.face[f].type) return false;
  return a.lmax == b.lmax;
}
}  // namespace

// Conservative state transfer onto dst's mesh from src (meshes of one
// geometry, at most one level apart at every destination leaf).
nb_status nb_amr_case_transfer(nb_case* dst, nb_case* src) {
  if (!dst || !src || !dst->amr || !src->amr || dst->ctx != src->ctx) return NB_ERR_BAD_ARG;
  nb_ctx* ctx = dst->ctx;
  if (dst->pending || src->pending) return fail(ctx, NB_ERR_BAD_ARG, "nb_amr_case_transfer: a step is in flight");
  if (!same_geometry(dst->mesh->geom, src->mesh->geom))
    return fail(ctx, NB_ERR_BAD_ARG, "nb_amr_case_transfer: the meshes have different geometries");
  const AmrTree& ts = src->mesh->lvl.tree;
  // leaf of the source at (level, brick), with the level bounded to the source's levels
  auto has = [&](int L, int x, int y, int z) { return L >= 0 && L < ts.nlev && ts.find(L, x, y, z) >= 0; };
  for (const AmrLeaf& f : dst->mesh->lvl.tree.leaves) {
    bool ok = has(f.level, f.b[0], f.b[1], f.b[2]) || has(f.level - 1, f.b[0] >> 1, f.b[1] >> 1, f.b[2] >> 1);
    if (!ok) {
      ok = true;
      for (int d = 0; d < 8 && ok; ++d)
        ok = has(f.level + 1, 2 * f.b[0] + (d & 1), 2 * f.b[1] + ((d >> 1) & 1), 2 * f.b[2] + (d >> 2));
    }
    if (!ok) return fail(ctx, NB_ERR_BAD_ARG, "nb_amr_case_transfer: the meshes differ by more than one level");
  }
  std::vector<void*> tmp;
  const nb_status st = guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    reset_history(*dst);
    NB_CUDA(cudaStreamSynchronize(src->stream));
    const int* dslab[3];
    long long nstore[3];
    const double* fsrc[3];
    double* fdst[3];
    for (int a = 0; a < 3; ++a) {
      const std::vector<int>& sb = dst->fm.slab_brick[a];
      void* d = nullptr;
      NB_CUDA(cudaMalloc(&d, std::max<size_t>(1, sb.size()) * sizeof(int)));
      tmp.push_back(d);
      if (!sb.empty()) NB_CUDA(cudaMemcpy(d, sb.data(), sb.size() * sizeof(int), cudaMemcpyHostToDevice));
      dslab[a] = static_cast<const int*>(d);
      nstore[a] = dst->fm.store[a];
      fsrc[a] = src->uvw[src->cur][a];
      fdst[a] = dst->uvw[dst->cur][a];
    }
    launch_amr_transfer(dst->stream, dst->AF, src->AF, dslab, nstore, fsrc, fdst, src->p, dst->p);
    ctx->launches += 4;
    amr_sync(*dst, dst->uvw[dst->cur]);
    NB_CUDA(cudaStreamSynchronize(dst->stream));
    dst->step = src->step;
    dst->t = src->t;
    dst->dt_last = src->dt_last;
    return NB_OK;
  });
  for (void* d : tmp) cudaFree(d);
  return st;
}

// Cell-centred values at host points (SolverBackend::sample): points and
// results pass through the context's staging buffers.
nb_status nb_case_sample(nb_case* c, int component, int64_t n, const double* xyz, double* out) {
  if (!c || component < 0 || component > 3 || n < 0 || (n > 0 && (!xyz || !out))) return NB_ERR_BAD_ARG;
  if (c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "nb_case_sample: the case has a step in flight");
  if (n == 0) return NB_OK;
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    ensure_staging(c->ctx, static_cast<size_t>(n) * 3);
    double* dxyz = c->ctx->stage_a;
    double* dout = c->ctx->stage_b;
    NB_CUDA(cudaMemcpyAsync(dxyz, xyz, static_cast<size_t>(n) * 3 * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    double** f = c->uvw[c->cur];
    if (c->amr) launch_amr_sample(c->stream, c->AF, component, n, dxyz, f[0], f[1], f[2], c->p, dout);
    else launch_sample(c->stream, c->F, component, n, dxyz, f[0], f[1], f[2], c->p, dout);
    ++c->ctx->launches;
    NB_CUDA(cudaMemcpyAsync(out, dout, static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NB_OK;
  });
}

nb_status nb_case_compute_dt(nb_case* c, double* dt) {
  if (!c || !dt) return NB_ERR_BAD_ARG;
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    *dt = compute_dt(*c);
    return NB_OK;
  });
}

nb_status nb_step(nb_case* c, double dt, nb_step_report* rep) {
  if (!c) return NB_ERR_BAD_ARG;
  if (c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "a step of this case is in flight (nb_step_wait)");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    nb_step_report r{};
    do_step(*c, dt, &r);
    if (rep) *rep = r;
    if (step_timed_out(*c)) return fail(c->ctx, NB_ERR_DEVICE_TIMEOUT, "a device-side barrier wait gave up");
    if (std::isnan(r.momentum_residual) || std::isnan(r.continuity_residual))
      return fail(c->ctx, NB_ERR_NAN, "NaN in the step diagnostics");
    return NB_OK;
  });
}

nb_status nb_step_async(nb_case* c, double dt) {
  if (!c) return NB_ERR_BAD_ARG;
  if (c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "a step of this case is already in flight");
  if (!c->ctx->prof.family.empty()) return fail(c->ctx, NB_ERR_UNSUPPORTED, "asynchronous steps need profiling off");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    launch_step(*c, dt);
    return NB_OK;
  });
}

nb_status nb_step_wait(nb_case* c, nb_step_report* rep) {
  if (!c) return NB_ERR_BAD_ARG;
  if (!c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "no step of this case is in flight");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    nb_step_report r{};
    complete_step(*c, &r);
    if (rep) *rep = r;
    if (step_timed_out(*c)) return fail(c->ctx, NB_ERR_DEVICE_TIMEOUT, "a device-side barrier wait gave up");
    if (std::isnan(r.momentum_residual) || std::isnan(r.continuity_residual))
      return fail(c->ctx, NB_ERR_NAN, "NaN in the step diagnostics");
    return NB_OK;
  });
}

nb_status nb_step_ready(nb_case* c, int* ready) {
  if (!c || !ready) return NB_ERR_BAD_ARG;
  if (!c->pending) return fail(c->ctx, NB_ERR_BAD_ARG, "no step of this case is in flight");
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    const cudaError_t e = cudaStreamQuery(c->stream);
    if (e == cudaErrorNotReady) {
      *ready = 0;
      return NB_OK;
    }
    NB_CUDA(e);
    *ready = 1;
    return NB_OK;
  });
}

nb_status nb_step_many(nb_case* c, double dt, int nsteps, nb_step_report* rep) {
  if (!c || nsteps < 0) return NB_ERR_BAD_ARG;
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    nb_step_report r{};
    for (int i = 0; i < nsteps; ++i) {
      do_step(*c, dt, &r);
      if (step_timed_out(*c)) return fail(c->ctx, NB_ERR_DEVICE_TIMEOUT, "a device-side barrier wait gave up");
    }
    if (rep) *rep = r;
    if (std::isnan(r.momentum_residual)) return fail(c->ctx, NB_ERR_NAN, "NaN in the step diagnostics");
    return NB_OK;
  });
}

nb_status nb_poisson_solve(nb_ctx* ctx, const nb_grid_desc* grid, const double* b, double* x,
                           double tol, int max_cycles, int precision, nb_poisson_report* rep) {
  if (!ctx || !b || !x || max_cycles < 0) return NB_ERR_BAD_ARG;
  std::string why;
  if (!grid_ok(grid, why)) return fail(ctx, NB_ERR_BAD_ARG, why);
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    MgSolver& mg = ctx_solver(ctx, *grid, precision);
    const FlowView F = cell_view(mg);
    const size_t n = static_cast<size_t>(grid->nx) * grid->ny * grid->nz;
    ensure_staging(ctx, std::max(n, static_cast<size_t>(F.nb)));
    NB_CUDA(cudaMemcpyAsync(ctx->stage_a, b, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    NB_CUDA(cudaMemsetAsync(ctx->stage_b, 0, F.nb * sizeof(double), ctx->stream));
    launch_convert(ctx->stream, F, 3, 0, ctx->stage_a, ctx->stage_b);
    ctx->launches++;
    mg.solve_async(ctx->stream, ctx->stage_b, tol, max_cycles);
    const nb_poisson_report r = mg.fetch_report(ctx->stream);
    if (mg.timed_out()) throw ApiError{NB_ERR_DEVICE_TIMEOUT, "a device-side barrier wait gave up"};
    launch_convert(ctx->stream, F, 3, 1, mg.phi(), ctx->stage_a);
    ctx->launches++;
    NB_CUDA(cudaMemcpyAsync(x, ctx->stage_a, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NB_CUDA(cudaStreamSynchronize(ctx->stream));
    if (rep) *rep = r;
    return NB_OK;
  });
}

nb_status nb_apply_laplacian(nb_ctx* ctx, const nb_grid_desc* grid, const double* x, double* out) {
  if (!ctx || !x || !out) return NB_ERR_BAD_ARG;
  std::string why;
  if (!grid_ok(grid, why)) return fail(ctx, NB_ERR_BAD_ARG, why);
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    MgSolver& mg = ctx_solver(ctx, *grid, NB_PRECISION_FP64);
    const FlowView F = cell_view(mg);
    const size_t n = static_cast<size_t>(grid->nx) * grid->ny * grid->nz;
    ensure_staging(ctx, std::max(n, static_cast<size_t>(F.nb)) * 2);
    double* xa = ctx->stage_b;
    double* xo = ctx->stage_b + F.nb;
    NB_CUDA(cudaMemcpyAsync(ctx->stage_a, x, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    NB_CUDA(cudaMemsetAsync(xa, 0, F.nb * sizeof(double), ctx->stream));
    launch_convert(ctx->stream, F, 3, 0, ctx->stage_a, xa);
    mg.apply_a(ctx->stream, xa, xo);
    launch_convert(ctx->stream, F, 3, 1, xo, ctx->stage_a);
    ctx->launches += 2;
    NB_CUDA(cudaMemcpyAsync(out, ctx->stage_a, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NB_CUDA(cudaStreamSynchronize(ctx->stream));
    return NB_OK;
  });
}

}  // extern "C"

// ===========================================================================
// octree-AMR cases
// ===========================================================================
extern "C" {

// The momentum kernel's ghost map: the walker's recorded form for every halo
// point that the same-level fast path does not serve, built once per case on
// the case's stream (count, host scan, fill; no device-wide synchronisation,
// which would break another thread's graph capture). Without it (more than
// 2^31 entries or terms) the kernel walks those points at every stage.
static void build_ghost_map(nb_case& c, AmrFlowView& F) {
  const int nb = F.L.nbrick;
  int* dcount = static_cast<int*>(c.alloc(2 * static_cast<size_t>(nb) * sizeof(int)));
  launch_ghost_count(c.stream, F, dcount);
  NB_CUDA(cudaStreamSynchronize(c.stream));
  std::vector<int> cnt(2 * static_cast<size_t>(nb));
  NB_CUDA(cudaMemcpy(cnt.data(), dcount, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<int> eoff(static_cast<size_t>(nb) + 1), toff(static_cast<size_t>(nb));
  long long ne = 0, nt = 0;
  for (int b = 0; b < nb; ++b) {
    if (ne > INT32_MAX || nt > INT32_MAX) return;
    eoff[b] = static_cast<int>(ne);
    toff[b] = static_cast<int>(nt);
    ne += cnt[2 * static_cast<size_t>(b)];
    nt += cnt[2 * static_cast<size_t>(b) + 1];
  }
  if (ne > INT32_MAX || nt > INT32_MAX) return;
  eoff[nb] = static_cast<int>(ne);
  int* d_eoff = static_cast<int*>(c.alloc(eoff.size() * sizeof(int)));
  int* d_toff = static_cast<int*>(c.alloc(toff.size() * sizeof(int)));
  auto* d_ent = static_cast<uint2*>(c.alloc(static_cast<size_t>(ne) * sizeof(uint2)));
  auto* d_term = static_cast<int2*>(c.alloc(static_cast<size_t>(nt) * sizeof(int2)));
  NB_CUDA(cudaMemcpy(d_eoff, eoff.data(), eoff.size() * sizeof(int), cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(d_toff, toff.data(), toff.size() * sizeof(int), cudaMemcpyHostToDevice));
  launch_ghost_fill(c.stream, F, d_eoff, d_toff, d_ent, d_term);
  NB_CUDA(cudaStreamSynchronize(c.stream));
  F.gm_off = d_eoff;
  F.gm_ent = d_ent;
  F.gm_term = d_term;
}

nb_status nb_amr_case_create(nb_ctx* ctx, nb_amr_mesh* mesh, const nb_flow_config* cfg, int precision,
                             nb_case** out) {
  if (!ctx || !mesh || !cfg || !out) return NB_ERR_BAD_ARG;
  *out = nullptr;
  if (precision != NB_PRECISION_FP64 && precision != NB_PRECISION_MIXED)
    return fail(ctx, NB_ERR_BAD_ARG, "precision must be NB_PRECISION_FP64 or NB_PRECISION_MIXED");
  if (!(cfg->reynolds > 0.0)) return fail(ctx, NB_ERR_BAD_ARG, "reynolds must be > 0");
  auto c = std::make_unique<nb_case>();
  c->ctx = ctx;
  c->amr = true;
  c->mesh = mesh;
  const nb_status s = guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    NB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const AmrLevelHost& lv = mesh->lvl;
    const AmrTree& t = lv.tree;
    const nb_amr_geom& g = mesh->geom;
    c->cfg = *cfg;
    c->precision = precision;
    c->nu = cfg->velocity_scale * cfg->ref_length / cfg->reynolds;  // ns_solver.cpp:54
    // level-0 description: report normalisation and inlet data
    c->grid.nx = t.cells(0, 0);
    c->grid.ny = t.cells(0, 1);
    c->grid.nz = t.cells(0, 2);
    c->grid.dx = g.h0[0];
    c->grid.dy = g.h0[1];
    c->grid.dz = g.h0[2];
    for (int a = 0; a < 3; ++a) c->grid.origin[a] = g.origin[a];
    for (int f = 0; f < 6; ++f) c->grid.face[f] = g.face[f];
    for (uint8_t v : lv.type)
      if (v == CELL_SOLID) {
        c->has_solid = true;
        break;
      }
    c->nfluid = lv.nfluid;
    c->mg = std::make_unique<MgSolver>(lv, precision, LaunchCounter{&ctx->launches, &ctx->prof}, &ctx->tune);
    c->rhs_grid = std::min(std::max(ctx->tune.rhs_ctas_per_sm, 1), 4) * ctx->nsm;
    build_face_maps(t, c->fm);
    AmrFlowView& F = c->AF;
    auto up = [&](const void* src, size_t bytes) {
      void* d = c->alloc(bytes);
      if (src && bytes) NB_CUDA(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice));
      else NB_CUDA(cudaMemset(d, 0, bytes ? bytes : 16));
      return d;
    };
    // The flow kernels' own view of the leaves (per-level LUTs, coordinates,
    // levels, cell types). It does not come from the multigrid hierarchy,
    // whose finest level is a uniform view when the mesh has one level.
    LevelView& V = F.L;
    V = LevelView{};
    V.amr = 1;
    V.nbrick = static_cast<int>(t.leaves.size());
    V.nlev = t.nlev;
    for (int f = 0; f < 6; ++f) V.bc[f] = g.face[f].type;
    V.nx = t.cells(0, 0);
    V.ny = t.cells(0, 1);
    V.nz = t.cells(0, 2);
    // Level sizes up to the geometry's finest level (a state transfer reads
    // this view at the levels of a mesh one level finer); LUTs only for the
    // levels present.
    const int ltab = std::min(g.lmax + 1, AMR_MAXLEV);
    for (int L = 0; L < ltab; ++L) {
      if (L < t.nlev) V.lut_off[L] = t.lut_off[L];
      for (int a = 0; a < 3; ++a) {
        V.lnb[L][a] = t.lnb(L, a);
        V.lcells[L][a] = t.cells(L, a);
        V.lh2[L][a] = 1.0 / (t.h(L, a) * t.h(L, a));
      }
    }
    for (int a = 0; a < 3; ++a) V.dxyz[a] = t.h(0, a);
    V.lut = static_cast<const int*>(up(t.lut.data(), t.lut.size() * sizeof(int)));
    V.bcoord = static_cast<const int*>(up(lv.bcoord.data(), lv.bcoord.size() * sizeof(int)));
    V.type = static_cast<const uint8_t*>(up(lv.type.data(), lv.type.size()));
    V.blevel = static_cast<const int8_t*>(up(lv.blevel.data(), lv.blevel.size()));
    for (int a = 0; a < 3; ++a) F.origin[a] = g.origin[a];
    for (int L = 0; L < ltab; ++L)
      for (int a = 0; a < 3; ++a) F.h[L][a] = t.h(L, a);
    for (int f = 0; f < 6; ++f) {
      for (int a = 0; a < 3; ++a) F.wallv[f][a] = g.face[f].wall_velocity[a];
      F.inlet_speed[f] = g.face[f].inlet_speed;
      F.profile[f] = g.face[f].profile;
      F.inlet_axis[f] = g.face[f].inlet_axis;
    }
    for (int a = 0; a < 3; ++a) F.per[a] = g.face[2 * a].type == NB_BC_PERIODIC;
    F.nb = static_cast<long long>(c->fm.nbrick) * BR3;
    if (t.nlev > AMR_MAXLEV) throw ApiError{NB_ERR_UNSUPPORTED, "mesh has more octree levels than supported"};
    F.slab_id = static_cast<const int*>(up(c->fm.slab_id.data(), c->fm.slab_id.size() * sizeof(int)));
    F.rel_lo = static_cast<const int8_t*>(up(c->fm.rel_lo.data(), c->fm.rel_lo.size()));
    F.rel_hi = static_cast<const int8_t*>(up(c->fm.rel_hi.data(), c->fm.rel_hi.size()));
    F.nbr_lo = static_cast<const int*>(up(c->fm.nbr_lo.data(), c->fm.nbr_lo.size() * sizeof(int)));
    F.nbr_hi = static_cast<const int*>(up(c->fm.nbr_hi.data(), c->fm.nbr_hi.size() * sizeof(int)));
    F.weno = cfg->convection == NB_CONV_WENO5;
    F.nu = c->nu;
    for (int a = 0; a < 3; ++a) F.bf[a] = cfg->body_force[a];
    if (ctx->tune.ghost_map) build_ghost_map(*c, F);
    for (int h = 0; h < 2; ++h)
      for (int q = 0; q < 3; ++q) {
        const size_t nb = static_cast<size_t>(c->fm.store[q]) * sizeof(double);
        c->uvw[h][q] = static_cast<double*>(c->alloc(nb));
        NB_CUDA(cudaMemset(c->uvw[h][q], 0, nb));
      }
    for (int q = 0; q < 3; ++q) {
      const size_t nb = static_cast<size_t>(c->fm.store[q]) * sizeof(double);
      c->uvw0[q] = static_cast<double*>(c->alloc(nb));
      NB_CUDA(cudaMemset(c->uvw0[q], 0, nb));
    }
    const size_t ncs = static_cast<size_t>(F.nb);
    c->p = static_cast<double*>(c->alloc(ncs * sizeof(double)));
    c->b = static_cast<double*>(c->alloc(ncs * sizeof(double)));
    NB_CUDA(cudaMemset(c->p, 0, ncs * sizeof(double)));
    NB_CUDA(cudaMemset(c->b, 0, ncs * sizeof(double)));
    alloc_history(*c, ncs);
    for (int a = 0; a < 3; ++a) {
      c->nsync[a] = static_cast<int>(c->fm.sync[a].size() / 5);
      if (c->nsync[a])
        c->d_sync[a] =
            static_cast<long long*>(up(c->fm.sync[a].data(), c->fm.sync[a].size() * sizeof(long long)));
    }
    std::vector<BcOp> out_ops, in_ops, solid_ops, unused;
    build_amr_bc(t, c->fm, lv.type, g, true, out_ops, solid_ops);
    build_amr_bc(t, c->fm, lv.type, g, false, in_ops, unused);
    c->n_out = static_cast<int>(out_ops.size());
    c->n_in = static_cast<int>(in_ops.size());
    c->n_solid = static_cast<int>(solid_ops.size());
    c->serial_out = needs_serial(out_ops);
    c->serial_in = needs_serial(in_ops);
    c->bc_out = upload_ops(*c, out_ops);
    c->bc_in = upload_ops(*c, in_ops);
    c->bc_solid = upload_ops(*c, solid_ops);
    c->rb.max_blocks = 148 * 4;
    c->rb.partials = static_cast<double*>(c->alloc(RED_KMAX * c->rb.max_blocks * sizeof(double)));
    c->rb.counter = static_cast<unsigned*>(c->alloc(sizeof(unsigned)));
    NB_CUDA(cudaMemset(c->rb.counter, 0, sizeof(unsigned)));
    c->d_blk = static_cast<StepBlock*>(c->alloc(sizeof(StepBlock)));
    NB_CUDA(cudaMemset(c->d_blk, 0, sizeof(StepBlock)));
    NB_CUDA(cudaMallocHost(&c->h_blk, sizeof(StepBlock)));
    NB_CUDA(cudaMallocHost(&c->h_dt, sizeof(double)));
    // the uploads and memsets above ran on the legacy stream; the case's own
    // stream is non-blocking, so steps of other cases keep running meanwhile
    NB_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    return NB_OK;
  });
  if (s != NB_OK) return s;
  ctx_retain(ctx);
  *out = c.release();
  return NB_OK;
}

nb_status nb_amr_case_sizes(const nb_case* c, int64_t sizes[4]) {
  if (!c || !c->amr || !sizes) return NB_ERR_BAD_ARG;
  for (int a = 0; a < 3; ++a) sizes[a] = c->fm.store[a];
  sizes[3] = static_cast<int64_t>(c->fm.nbrick) * BR3;
  return NB_OK;
}

nb_status nb_amr_case_slabs(const nb_case* c, int axis, int32_t* bricks) {
  if (!c || !c->amr || axis < 0 || axis > 2 || !bricks) return NB_ERR_BAD_ARG;
  for (size_t s = 0; s < c->fm.slab_brick[axis].size(); ++s) bricks[s] = c->fm.slab_brick[axis][s];
  return NB_OK;
}

nb_status nb_amr_case_set_state(nb_case* c, const double* u, const double* v, const double* w, const double* p) {
  if (!c || !c->amr || !u || !v || !w || !p) return NB_ERR_BAD_ARG;
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    const bool keep = c->d_nhist != nullptr;  // stage, compare, then swap in
    double** f = c->uvw[keep ? 1 - c->cur : c->cur];
    const double* src[3] = {u, v, w};
    for (int a = 0; a < 3; ++a)
      NB_CUDA(cudaMemcpyAsync(f[a], src[a], static_cast<size_t>(c->fm.store[a]) * 8, cudaMemcpyHostToDevice,
                              c->stream));
    const size_t np = static_cast<size_t>(c->fm.nbrick) * BR3;
    NB_CUDA(cudaMemcpyAsync(keep ? c->b : c->p, p, np * 8, cudaMemcpyHostToDevice, c->stream));
    amr_sync(*c, f);
    if (keep) compare_and_swap_in(*c, np);
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NB_OK;
  });
}

nb_status nb_amr_case_get_state(nb_case* c, double* u, double* v, double* w, double* p) {
  if (!c || !c->amr) return NB_ERR_BAD_ARG;
  return guarded(c->ctx, [&] {
    NB_CUDA(cudaSetDevice(c->ctx->device));
    double** f = c->uvw[c->cur];
    double* dst[3] = {u, v, w};
    for (int a = 0; a < 3; ++a)
      if (dst[a])
        NB_CUDA(cudaMemcpyAsync(dst[a], f[a], static_cast<size_t>(c->fm.store[a]) * 8, cudaMemcpyDeviceToHost,
                                c->stream));
    if (p)
      NB_CUDA(cudaMemcpyAsync(p, c->p, static_cast<size_t>(c->fm.nbrick) * BR3 * 8, cudaMemcpyDeviceToHost,
                              c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NB_OK;
  });
}

}  // extern "C"
