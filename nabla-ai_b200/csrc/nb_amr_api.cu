// nb_amr_api.cu — C ABI of octree-AMR brick meshes and their pressure solve.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "nb_amr.h"
#include "nb_amr_level.h"
#include "nb_amr_mesh.h"
#include "nb_ctx.h"
#include "nb_mg.cuh"

using namespace nb;

namespace {

bool geom_ok(const nb_amr_geom* g, std::string& why) {
  if (!g) { why = "geometry is NULL"; return false; }
  for (int a = 0; a < 3; ++a) {
    if (g->nb0[a] < 1) { why = "nb0 must be >= 1"; return false; }
    if (!(g->h0[a] > 0.0)) { why = "h0 must be > 0"; return false; }
  }
  if (g->lmax < 0 || g->lmax >= AMR_MAXLEV) { why = "lmax out of range"; return false; }
  for (int a = 0; a < 3; ++a)
    if (static_cast<long long>(g->nb0[a]) << g->lmax > (1 << 17)) { why = "mesh too large"; return false; }
  for (int f = 0; f < 6; ++f)
    if (g->face[f].type < NB_BC_WALL || g->face[f].type > NB_BC_PERIODIC) { why = "bad boundary type"; return false; }
  for (int a = 0; a < 3; ++a)
    if ((g->face[2 * a].type == NB_BC_PERIODIC) != (g->face[2 * a + 1].type == NB_BC_PERIODIC)) {
      why = "periodic faces must come in pairs";
      return false;
    }
  return true;
}

AmrGeom to_geom(const nb_amr_geom& g) {
  AmrGeom o{};
  for (int a = 0; a < 3; ++a) {
    o.nb0[a] = g.nb0[a];
    o.h0[a] = g.h0[a];
    o.origin[a] = g.origin[a];
  }
  for (int f = 0; f < 6; ++f) o.bc[f] = g.face[f].type;
  o.lmax = g.lmax;
  return o;
}

std::vector<AmrLeaf> to_leaves(const int32_t* leaves, int64_t n) {
  std::vector<AmrLeaf> v(static_cast<size_t>(n));
  for (int64_t q = 0; q < n; ++q)
    v[q] = AmrLeaf{leaves[4 * q], {leaves[4 * q + 1], leaves[4 * q + 2], leaves[4 * q + 3]}};
  return v;
}

MgSolver& mesh_solver(nb_amr_mesh* m, int precision) {
  auto& s = m->mg[precision == NB_PRECISION_MIXED ? 1 : 0];
  if (!s)
    s = std::make_unique<MgSolver>(m->lvl, precision, LaunchCounter{&m->ctx->launches, &m->ctx->prof}, &m->ctx->tune);
  return *s;
}

}  // namespace

extern "C" {

nb_status nb_amr_refine(const nb_amr_geom* g, const int32_t* leaves, int64_t n, const uint8_t* flags,
                        int32_t* out, int64_t cap, int64_t* n_out) {
  std::string why;
  if (!geom_ok(g, why) || !leaves || n <= 0 || !flags || !n_out) return NB_ERR_BAD_ARG;
  try {
    std::string err;
    const std::vector<uint8_t> fl(flags, flags + n);
    const std::vector<AmrLeaf> res = refine_leaves(to_geom(*g), to_leaves(leaves, n), fl, err);
    if (!err.empty()) return NB_ERR_BAD_ARG;
    *n_out = static_cast<int64_t>(res.size());
    if (!out || cap < static_cast<int64_t>(res.size())) return NB_ERR_BAD_ARG;
    for (size_t q = 0; q < res.size(); ++q) {
      out[4 * q] = res[q].level;
      for (int a = 0; a < 3; ++a) out[4 * q + 1 + a] = res[q].b[a];
    }
    return NB_OK;
  } catch (const std::exception&) {
    return NB_ERR_BAD_ARG;
  }
}

nb_status nb_amr_coarsen(const nb_amr_geom* g, const int32_t* leaves, int64_t n, const uint8_t* flags,
                         int32_t* out, int64_t cap, int64_t* n_out) {
  std::string why;
  if (!geom_ok(g, why) || !leaves || n <= 0 || !flags || !n_out) return NB_ERR_BAD_ARG;
  try {
    std::string err;
    const std::vector<uint8_t> fl(flags, flags + n);
    const std::vector<AmrLeaf> res = coarsen_leaves(to_geom(*g), to_leaves(leaves, n), fl, err);
    if (!err.empty()) return NB_ERR_BAD_ARG;
    *n_out = static_cast<int64_t>(res.size());
    if (!out || cap < static_cast<int64_t>(res.size())) return NB_ERR_BAD_ARG;
    for (size_t q = 0; q < res.size(); ++q) {
      out[4 * q] = res[q].level;
      for (int a = 0; a < 3; ++a) out[4 * q + 1 + a] = res[q].b[a];
    }
    return NB_OK;
  } catch (const std::exception&) {
    return NB_ERR_BAD_ARG;
  }
}

nb_status nb_amr_mesh_create(nb_ctx* ctx, const nb_amr_geom* g, const int32_t* leaves, int64_t n,
                             const uint8_t* solid, nb_amr_mesh** out) {
  if (!ctx || !out || !leaves || n <= 0) return NB_ERR_BAD_ARG;
  *out = nullptr;
  std::string why;
  if (!geom_ok(g, why)) return fail(ctx, NB_ERR_BAD_ARG, why);
  auto m = std::make_unique<nb_amr_mesh>();
  m->ctx = ctx;
  m->geom = *g;
  const nb_status s = guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    std::string err;
    const std::vector<AmrLeaf> in = to_leaves(leaves, n);
    m->lvl.tree = tree_from_leaves(to_geom(*g), in, err);
    if (!err.empty()) throw ApiError{NB_ERR_BAD_ARG, "nb_amr_mesh_create: " + err};
    int wl = 0;
    for (const AmrLeaf& f : m->lvl.tree.leaves) wl = std::max(wl, f.level);
    m->lvl.wlmax = wl;
    amr_level_geometry(m->lvl);
    // solid flags arrive in the input order: map them to ranks
    m->lvl.type.assign(m->lvl.tree.leaves.size() * BR3, CELL_FLUID);
    if (solid) {
      for (int64_t q = 0; q < n; ++q) {
        const AmrLeaf& f = in[q];
        const int r = m->lvl.tree.find(f.level, f.b[0], f.b[1], f.b[2]);
        for (int l = 0; l < BR3; ++l)
          m->lvl.type[static_cast<size_t>(r) * BR3 + l] = solid[q * BR3 + l] ? CELL_SOLID : CELL_FLUID;
      }
    }
    amr_level_codes(m->lvl);
    return NB_OK;
  });
  if (s != NB_OK) return s;
  ctx_retain(ctx);
  *out = m.release();
  return NB_OK;
}

void nb_amr_mesh_destroy(nb_amr_mesh* m) {
  if (!m) return;
  nb_ctx* ctx = m->ctx;
  cudaSetDevice(ctx->device);
  delete m;
  ctx_release(ctx);
}

int64_t nb_amr_mesh_leaf_count(const nb_amr_mesh* m) {
  return m ? static_cast<int64_t>(m->lvl.tree.leaves.size()) : 0;
}

nb_status nb_amr_mesh_leaves(const nb_amr_mesh* m, int32_t* out) {
  if (!m || !out) return NB_ERR_BAD_ARG;
  const auto& L = m->lvl.tree.leaves;
  for (size_t q = 0; q < L.size(); ++q) {
    out[4 * q] = L[q].level;
    for (int a = 0; a < 3; ++a) out[4 * q + 1 + a] = L[q].b[a];
  }
  return NB_OK;
}

nb_status nb_amr_apply_laplacian(nb_ctx* ctx, nb_amr_mesh* m, const double* x, double* out) {
  if (!ctx || !m || !x || !out) return NB_ERR_BAD_ARG;
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    MgSolver& mg = mesh_solver(m, NB_PRECISION_FP64);
    const size_t n = m->lvl.tree.leaves.size() * BR3;
    ensure_staging(ctx, n);
    NB_CUDA(cudaMemcpyAsync(ctx->stage_a, x, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    mg.apply_a(ctx->stream, ctx->stage_a, ctx->stage_b);
    NB_CUDA(cudaMemcpyAsync(out, ctx->stage_b, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NB_CUDA(cudaStreamSynchronize(ctx->stream));
    return NB_OK;
  });
}

nb_status nb_amr_poisson_solve(nb_ctx* ctx, nb_amr_mesh* m, const double* b, double* x, double tol,
                               int max_cycles, int precision, nb_poisson_report* rep) {
  if (!ctx || !m || !b || !x || max_cycles < 0) return NB_ERR_BAD_ARG;
  if (precision != NB_PRECISION_FP64 && precision != NB_PRECISION_MIXED) return NB_ERR_BAD_ARG;
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    MgSolver& mg = mesh_solver(m, precision);
    const size_t n = m->lvl.tree.leaves.size() * BR3;
    ensure_staging(ctx, n);
    NB_CUDA(cudaMemcpyAsync(ctx->stage_a, b, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    mg.solve_async(ctx->stream, ctx->stage_a, tol, max_cycles);
    const nb_poisson_report r = mg.fetch_report(ctx->stream);
    if (mg.timed_out()) throw ApiError{NB_ERR_DEVICE_TIMEOUT, "a device-side barrier wait gave up"};
    NB_CUDA(cudaMemcpyAsync(x, mg.phi(), n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NB_CUDA(cudaStreamSynchronize(ctx->stream));
    if (rep) *rep = r;
    return NB_OK;
  });
}

}  // extern "C"
