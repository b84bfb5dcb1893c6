// nb_ctx.h — the context object behind the C ABI and its error plumbing.
#pragma once
#include <atomic>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "nb_internal.h"
#include "nb_mg.cuh"

namespace nb {
// One step of a set of cases as a single CUDA graph: every case's step is an
// independent branch (captured from the case's own stream), so one launch
// advances all of them and their kernels overlap on the device.
struct BatchGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t fixed_kernels = 0;        // kernels outside the MG-PCG loop bodies
  std::vector<uint64_t> body_kernels;  // per case: kernels per loop-body execution
};
}  // namespace nb

struct nb_ctx {
  int device = 0;
  // the caller's handle plus one per live case and mesh: nb_ctx_destroy drops
  // the first, and the context is freed when the last of its objects goes, in
  // whatever order the caller (or a garbage collector) destroys them
  std::atomic<int> refs{1};
  std::string err;
  std::atomic<uint64_t> launches{0};  // atomic: cases may be built on one thread while others step
  nb::Profiler prof;
  cudaStream_t stream = nullptr;
  int nsm = 148;     // SMs of the device
  nb_tuning tune{};  // applies to objects created after it is set
  // batch graphs keyed by (case, state parity) pairs
  std::map<std::vector<uintptr_t>, nb::BatchGraph> batch_cache;
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

inline void ctx_retain(nb_ctx* ctx) { ctx->refs.fetch_add(1, std::memory_order_relaxed); }
// Frees the context when this was its last reference.
void ctx_release(nb_ctx* ctx);

// A scratch case with `sample`'s mesh or grid, configuration, precision and
// current state, built with the context's current tuning (autotuner).
nb_status clone_case(nb_case* sample, nb_case** out);
// Kind of a case for the tuning cache key.
void case_kind(const nb_case* c, int* amr, int* precision, int* levels);
// Case internals for the checkpoint files: owning context, uniform grid
// dimensions, octree mesh (nullptr for uniform cases), and the step clock.
nb_ctx* case_ctx(const nb_case* c);
void case_dims(const nb_case* c, int dims[3]);
nb_amr_mesh* case_mesh(const nb_case* c);
void case_set_clock(nb_case* c, int step, double t, double dt_last);
// Per-cell solid flags for output: uniform cases nx*ny*nz lexicographic (or
// empty when the grid has none), octree cases leaves*512 in storage order.
std::vector<uint8_t> case_solid(const nb_case* c);
// The grid description a uniform case was created with.
const nb_grid_desc& case_grid(const nb_case* c);

// Grows the context's two staging buffers to at least `elems` doubles each.
void ensure_staging(nb_ctx* ctx, size_t elems);

}  // namespace nb
