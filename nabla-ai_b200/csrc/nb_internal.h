// nb_internal.h — shared definitions of the sm_100a solver library.
//
// Storage model ("bricks"): a uniform cell grid nx*ny*nz is covered by
// ceil(n/8) bricks per axis of 8x8x8 cells. Bricks are ranked in Morton
// order of their brick coordinates (the reference's key,
// core/include/nabla/mesh/morton.hpp:19-48) and a dense lookup table maps brick
// coordinates to rank. A cell field is [nbrick][8][8][8] doubles (x fastest
// inside a brick). Cells of a partially covered brick that lie outside the
// grid are "void": typed NB_CELL_VOID, always zero, excluded from every sum.
//
// MAC faces: u(i,j,k) is the low-x face of cell (i,j,k) and is stored in the
// cell's slot; the domain's high face i == nx is stored in a trailing slab of
// ny*nz values appended to the brick array (v: nx*nz, w: nx*ny), so a face
// component is one contiguous allocation [nbrick*512 | slab].
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "nabla_b200.h"

namespace nb {

constexpr int BR = 8;       // brick edge (cells)
constexpr int BR3 = 512;    // cells per brick
constexpr int AMR_MAXLEV = 6;  // octree levels of a composite mesh
enum : uint8_t { CELL_FLUID = 0, CELL_SOLID = 1, CELL_VOID = 2 };

// ---------------------------------------------------------------------------
// Device view of one uniform brick level (passed by value to kernels).
// ---------------------------------------------------------------------------
struct LevelView {
  int nx, ny, nz;
  int nbx, nby, nbz, nbrick;
  int bc[6];          // NB_BC_* per domain face
  double h2[3];       // 1/h^2 per axis
  double dxyz[3];     // h per axis
  int twoD;           // nz == 1: no z coupling (poisson.cpp:61, ns_solver.cpp:316)
  const int* lut;     // [nbz][nby][nbx] -> brick rank
  const int* bcoord;  // [nbrick][3] brick coordinates
  const uint8_t* type;  // [nbrick*512] CELL_*
  // Per-cell stencil code (built on the host from the BCs and solids):
  // bit f (f = 2*axis + side, side 0 low / 1 high): face f couples to a fluid
  // neighbour; bit 6+f: face f is a Dirichlet outlet face; bits 12-13: CELL_*.
  const uint16_t* code;
  // ---- composite (multi-level) levels only: amr != 0 ----
  // Bricks carry their own octree level; `lut` holds one dense table per
  // octree level (offset lut_off[L], lnb[L] bricks per axis, -1 = no leaf);
  // bit f of `code` couples to the same-level neighbour only, coarse-fine
  // couplings are the CSR list cf_off/cf_nbr/cf_coef (CODE_HASCF cells).
  int amr;
  int nlev;
  int lut_off[AMR_MAXLEV];
  int lnb[AMR_MAXLEV][3];
  int lcells[AMR_MAXLEV][3];
  double lh2[AMR_MAXLEV][3];
  const int8_t* blevel;
  const double* bweight;  // cell volume / finest cell volume (exact powers of 8)
  const int* cf_off;
  const int* cf_nbr;
  const double* cf_coef;
  // transfer to the next coarser MG level: coarse brick, octant (-1 kept)
  const int* xf_brick;
  const int* xf_oct;
  // ---- per-brick maps for one-round halo staging (fast != 0: every brick is
  // full, i.e. composite levels and uniform levels whose sizes are multiples
  // of 8) ----
  int fast;
  const int* nbr6;   // [nbrick][6] same-level face neighbour brick (periodic wrap) or -1
  const int* par;    // [nbrick] brick of the next coarser level holding this brick's parents
  const int* poct;   // [nbrick] octant bits of this brick in its parent brick, -1 identity
  const int* npar6;  // [nbrick][6] par of nbr6 (-1 where no neighbour)
  const int* npoct6; // [nbrick][6] poct of nbr6
};
constexpr int CODE_DIRICHLET = 6;
constexpr int CODE_TYPE = 12;
constexpr int CODE_HASCF = 14;  // composite levels: the cell has coarse-fine couplings

__host__ __device__ inline int wrapi(int a, int n) { return (a % n + n) % n; }

__device__ __forceinline__ int cell_index(const LevelView& L, int gi, int gj, int gk) {
  const int b = L.lut[((gk >> 3) * L.nby + (gj >> 3)) * L.nbx + (gi >> 3)];
  return b * BR3 + (((gk & 7) << 6) | ((gj & 7) << 3) | (gi & 7));
}

__device__ __forceinline__ void cell_coords(const LevelView& L, int idx, int& gi, int& gj, int& gk) {
  const int b = idx >> 9, l = idx & 511;
  gi = L.bcoord[3 * b] * BR + (l & 7);
  gj = L.bcoord[3 * b + 1] * BR + ((l >> 3) & 7);
  gk = L.bcoord[3 * b + 2] * BR + (l >> 6);
}

// kind 0 = no coupling (Neumann wall/inlet or solid neighbour), 1 = neighbour
// `n`, 2 = Dirichlet outlet. Follows resolveFace (core/src/flow/poisson.cpp:18-52).
__device__ __forceinline__ int resolve_face(const LevelView& L, int gi, int gj, int gk, int axis,
                                            int side, int& n) {
  int c[3] = {gi, gj, gk};
  const int dims[3] = {L.nx, L.ny, L.nz};
  c[axis] += side;
  if (c[axis] < 0 || c[axis] >= dims[axis]) {
    const int bt = L.bc[2 * axis + (side > 0 ? 1 : 0)];
    if (bt == NB_BC_PERIODIC) {
      c[axis] = (c[axis] + dims[axis]) % dims[axis];
    } else {
      return bt == NB_BC_OUTLET ? 2 : 0;
    }
  }
  n = cell_index(L, c[0], c[1], c[2]);
  return L.type[n] == CELL_SOLID ? 0 : 1;
}

// ---------------------------------------------------------------------------
// Device scalar slots of one solve (FP64, in device memory).
// ---------------------------------------------------------------------------
constexpr int MAX_LEVELS = 16;  // composite octree levels + the uniform tail
enum Slot : int {
  S_BSUM = 0,   // sum of b over fluid (rhs mean)
  S_BNORM2,     // rhs . rhs
  S_RZ,         // r . z
  S_PAP,        // p . Ap
  S_ALPHA,
  S_BETA,
  S_RNORM2,
  S_RNEWZ,
  S_RZCROSS,
  S_RMEAN,      // mean of rnew (singular)
  S_ZMEAN2,     // second mean removal of z (Minv's removeMean)
  S_XMEAN,      // final removeMean(x)
  S_TRUERES2,   // true residual sum of squares
  S_DIVMAX,
  S_DIV2,
  S_DU2,
  S_FX,
  S_FY,
  S_MASS,
  S_MAXINV,
  S_IRRES2,     // iterative refinement: true residual sum of squares
  S_IRMEAN,     // iterative refinement: fluid mean of the true residual (singular)
  S_LVL_MEAN = 24,  // [MAX_LEVELS][4]: per-level pending means (x ping, x pong, b)
  S_COUNT = S_LVL_MEAN + MAX_LEVELS * 4
};
inline int lvl_slot(int level, int which) { return S_LVL_MEAN + level * 4 + which; }

constexpr int STOP_TIMEOUT = 3;  // a bounded device-side wait gave up
struct SolveFlags {
  int stop;      // 0 running, 1 converged, 2 breakdown (|pAp| < 1e-300), 3 STOP_TIMEOUT
  int iters;     // completed MG-PCG cycles
  int early;     // rhs already below tolerance
  int nan;       // NaN seen in a reduction
  int restarts;  // iterative-refinement restarts of this solve (mixed form)
  int checked;   // the true residual met the tolerance: no further refinement checks
};

// Reduction scratch: per-block partials + a ticket counter (last-block
// finalisation, deterministic fixed-order tree over the partials).
struct RedBuf {
  double* partials = nullptr;   // [K_MAX][max_blocks]
  unsigned* counter = nullptr;  // single ticket counter
  int max_blocks = 0;
};
constexpr int RED_KMAX = 8;

// ---------------------------------------------------------------------------
// Host-side level description (built once per grid, cached by signature).
// ---------------------------------------------------------------------------
struct HostLevel {
  int nx, ny, nz, nbx, nby, nbz, nbrick;
  int fx = 1, fy = 1, fz = 1;  // coarsening factor from the next-finer level
  double dx, dy, dz;
  std::vector<int> lut, bcoord;
  std::vector<uint8_t> type;   // brick layout
  std::vector<uint16_t> code;  // brick layout, see LevelView::code
  std::vector<uint8_t> solid;  // lexicographic (for hierarchy construction)
  uint64_t nfluid = 0;
};

// Fills L.code from the cell types and the domain BCs (the face resolution of
// core/src/flow/poisson.cpp:18-52, precomputed once per level).
void build_codes(HostLevel& L, const int bc[6]);

// Builds the brick layout of an nx*ny*nz grid with the given lexicographic
// solid mask (NULL = none).
void build_level(HostLevel& L, int nx, int ny, int nz, double dx, double dy, double dz,
                 const uint8_t* solid);
// Builds the MG hierarchy exactly as MgPoisson::solve does (multigrid.cpp:211-266):
// halve every axis of >= 4 cells until the coarse level has <= coarsest_max
// cells (the reference's 2048) or 8 levels exist.
std::vector<HostLevel> build_hierarchy(const nb_grid_desc& g, size_t coarsest_max = 2048);
uint64_t grid_signature(const nb_grid_desc& g);  // multigrid.cpp:43-61 (+ spacing)

// Brackets the launches of one kernel family with CUDA events on the
// launching stream and accumulates their algorithmic bytes (measurement only).
struct Profiler {
  std::string family;  // empty: off
  std::vector<cudaEvent_t> ev;  // pairs (start, stop)
  size_t used = 0;
  uint64_t launches = 0;
  double bytes = 0.0;
  bool on(const char* f) const { return !family.empty() && family == f; }
  void begin(cudaStream_t s) {
    if (ev.size() < 2 * (used + 1)) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      ev.push_back(a);
      ev.push_back(b);
    }
    cudaEventRecord(ev[2 * used], s);
  }
  void end(cudaStream_t s, double nbytes) {
    cudaEventRecord(ev[2 * used + 1], s);
    ++used;
    ++launches;
    bytes += nbytes;
  }
  // Sum of event intervals (ms); resets the counters.
  double drain(uint64_t* nl, double* nb) {
    double ms = 0.0;
    for (size_t i = 0; i < used; ++i) {
      cudaEventSynchronize(ev[2 * i + 1]);
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
      ms += t;
    }
    if (nl) *nl = launches;
    if (nb) *nb = bytes;
    used = 0;
    launches = 0;
    bytes = 0.0;
    return ms;
  }
  ~Profiler() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};

// Launch accounting shared by every launch site of a context.
struct LaunchCounter {
  std::atomic<uint64_t>* count = nullptr;
  Profiler* prof = nullptr;
  void add(uint64_t n = 1) {
    if (count) count->fetch_add(n, std::memory_order_relaxed);
  }
};

// Runs `launch` (one kernel launch statement); brackets it with events when
// family `fam` is being profiled.
#define NB_LAUNCH(lc, fam, stream, nbytes, launch)              \
  do {                                                          \
    const bool nb_prof_on_ = (lc).prof && (lc).prof->on(fam);   \
    if (nb_prof_on_) (lc).prof->begin(stream);                  \
    launch;                                                     \
    if (nb_prof_on_) (lc).prof->end(stream, static_cast<double>(nbytes)); \
    (lc).add();                                                 \
  } while (0)

// CUDA error helpers
#define NB_CUDA(call)                                                                \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) throw nb::CudaError(e_, #call, __FILE__, __LINE__);       \
  } while (0)

struct CudaError {
  cudaError_t err;
  std::string what;
  CudaError(cudaError_t e, const char* call, const char* file, int line);
};
struct ApiError {
  nb_status status;
  std::string what;
};

// ---------------------------------------------------------------------------
// Programmatic dependent launch. A kernel launched with launch_pdl may be
// scheduled while its stream predecessor is still running (hiding the launch
// latency of the long chains of small multigrid kernels); it calls pdl_wait()
// before its first access to global memory, which returns once the
// predecessor grid has completed and its writes are visible. pdl_wait() first
// lets this grid's own successor be scheduled. In a kernel launched without
// the attribute both instructions return at once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// `pdl` false launches without the attribute (a tuning choice).
template <typename... KArgs, typename... Args>
inline void launch_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  NB_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

}  // namespace nb
