// nb_ctx.h — the context object behind the C ABI and its error plumbing.
#pragma once
#include <map>
#include <memory>
#include <string>

#include "nb_internal.h"
#include "nb_mg.cuh"

struct nb_ctx {
  int device = 0;
  std::string err;
  uint64_t launches = 0;
  nb::Profiler prof;
  cudaStream_t stream = nullptr;
  // MgPoisson-style cache for the host-array Poisson seam (multigrid.cpp:211-220)
  std::map<std::pair<uint64_t, int>, std::unique_ptr<nb::MgSolver>> mg_cache;
  double* stage_a = nullptr;
  double* stage_b = nullptr;
  size_t stage_bytes = 0;
};

namespace nb {

inline nb_status fail(nb_ctx* ctx, nb_status s, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return s;
}

template <class Fn>
nb_status guarded(nb_ctx* ctx, Fn&& fn) {
  try {
    return fn();
  } catch (const ApiError& e) {
    return fail(ctx, e.status, e.what);
  } catch (const CudaError& e) {
    return fail(ctx, NB_ERR_CUDA, e.what);
  } catch (const std::exception& e) {
    return fail(ctx, NB_ERR_BAD_ARG, e.what());
  }
}

// Grows the context's two staging buffers to at least `elems` doubles each.
void ensure_staging(nb_ctx* ctx, size_t elems);

}  // namespace nb
