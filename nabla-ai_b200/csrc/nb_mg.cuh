// nb_mg.cuh — MG-PCG pressure solver on brick levels (host interface).
//
// Device restatement of MgPoisson (core/src/flow/multigrid.cpp:22-355) and its
// coarsest-level CgPoisson (core/src/flow/poisson.cpp:136-252):
//   * V(2,2) cycle, damped Jacobi (omega 0.8), restriction = average of fluid
//     children, piecewise-constant prolongation, removeMean after every sweep
//     on singular systems (applied lazily by the next kernel that reads the
//     vector, so it costs no extra pass);
//   * coarsest level: Jacobi-PCG to 1e-6 / 500 in one CTA (shared memory);
//   * flexible (Polak-Ribiere) PCG outer loop, FP64 in both forms.
#pragma once
#include <memory>
#include <vector>

#include "nb_amr_level.h"
#include "nb_internal.h"

namespace nb {

struct DevLevel {
  HostLevel h;
  LevelView v{};
  int* d_lut = nullptr;
  int* d_bcoord = nullptr;
  uint8_t* d_type = nullptr;
  uint16_t* d_code = nullptr;
  int* d_xfb = nullptr;  // composite levels: transfer maps to the next level
  int* d_xfo = nullptr;
  // host copies for the one-round halo maps (built once all levels exist)
  std::vector<int> h_nbr6, h_par, h_poct;
  double wfluid = 0.0;   // fluid volume in cell-weight units (= fluid cells on uniform levels)
  double ncell = 0.0;    // cells of the level (for algorithmic byte counts)
  // V-cycle vectors in the level's arithmetic type (double or float):
  // b (restricted residual), x ping, x pong.
  void* b = nullptr;
  void* x0 = nullptr;
  void* x1 = nullptr;
  bool b16 = false;  // b stored as BF16 (mixed form, nb_tuning.coarse_bf16)
};

// Cluster-resident V-cycle tail: one launch runs the V-cycle from level
// `tail_lvl` down (sweeps, residual + restriction, coarsest solve), phase by
// phase, on one thread-block cluster.
constexpr int MAX_TAIL_LEV = 8;
constexpr int MAX_TAIL_PH = 64;
enum TailOp : int { TAIL_SMOOTH = 0, TAIL_RESID = 1, TAIL_DIRECT = 2, TAIL_CG = 3 };
// A level vector as the launch path's fetch reads it (pending mean and
// prolongation); clvl is the tail-relative coarse level, -1 none.
struct TailFetch {
  const void* x;
  const double* xmean;
  const void* ec;
  const double* ecmean;
  int clvl, fx, fy, fz;
  const int* xfb;
  const int* xfo;
};
struct TailPhase {
  int op, lvl, clvl, prev_mode;  // lvl / clvl: tail-relative level and its coarser level
  const void* b;
  const double* bmean;
  TailFetch X, P;
  void* out;          // smoothed x, restricted residual, or coarsest x
  double* mean_out;   // pending mean of `out` (nullptr: none)
  double inv_nf;
  double c2, c1;
  int fx, fy, fz, pad;
};
// Vector pointers in the phases are arena encodings (byte offset in every
// CTA's shared-memory arena + 128), not device addresses.
struct TailProg {
  int nlev, nphase, singular, nf;
  int lcs;            // log2 of the cluster size
  int nbrick;         // bricks of the tail level
  size_t arena_bytes;  // per CTA
  void* b_in;         // tail level's rhs (global), loaded into arena array b_enc
  uintptr_t b_enc;
  void* x_out;        // tail level's result (global), stored from arena array x_enc
  uintptr_t x_enc;
  const double* inv;  // exact coarsest solve (TAIL_DIRECT)
  const int* fmap;
  const int* lexpos;
  const int* lexcell;
  double* xs;  // [nf] scratch
  LevelView lv[MAX_TAIL_LEV];
  TailPhase ph[MAX_TAIL_PH];
};

// Grid-resident V-cycle: one cooperative launch runs the whole V-cycle (every
// level, the coarsest solve included) as a list of phases over all CTAs, with
// a bounded grid barrier between phases. Vectors stay in global memory (L2);
// the phases are the launch path's own per-brick code.
constexpr int MAX_GRID_LEV = 12;
constexpr int MAX_GRID_PH = 160;
struct GridProg {
  int nlev, nphase, singular, nf;
  const double* inv;  // exact coarsest solve (TAIL_DIRECT)
  const int* fmap;
  const int* lexpos;
  const int* lexcell;
  double* xs;          // [nf] scratch of the exact coarsest solve
  unsigned* sync;      // [0] barrier arrivals (zeroed before every launch), [1] abort flag
  double* partials;    // [grid] per-CTA partial sums of a phase's pending mean
  SolveFlags* flags;   // stop = STOP_TIMEOUT when a barrier gives up
  LevelView lv[MAX_GRID_LEV];
  TailPhase ph[MAX_GRID_PH];
};

// Initial guess of a solve (instead of x = 0): x0 = alpha * (*dt) * guess on
// the fluid cells of level 0 (brick layout), e.g. the last projection's
// pressure scaled to this projection's potential.
struct WarmStart {
  const double* guess;
  const double* dt;  // device scalar
  double alpha;
  // History forms (h1, h2, h3 and nhist set): once *nhist >= 2 the guess is
  // instead dt * (h1 + k2 h2 + k3 h3); before that the form above.
  const double* h1 = nullptr;
  const double* h2 = nullptr;
  const double* h3 = nullptr;
  double k2 = 0.0, k3 = 0.0;
  const int* nhist = nullptr;
};

class MgSolver {
 public:
  // `tune` sets launch shapes, halo staging, mixed-form sweeps, the exact
  // coarse-solve threshold and PDL (nb_tuning; nullptr = defaults).
  MgSolver(const nb_grid_desc& g, int precision, LaunchCounter lc, const nb_tuning* tune = nullptr);
  // Composite (octree-AMR) operator on the leaves of `fine` (types and codes
  // already built), with the composite-then-uniform MG hierarchy.
  MgSolver(const AmrLevelHost& fine, int precision, LaunchCounter lc, const nb_tuning* tune = nullptr);
  ~MgSolver();
  MgSolver(const MgSolver&) = delete;
  MgSolver& operator=(const MgSolver&) = delete;

  // Solve A x = b for device vector b (fluid rhs, brick layout). The solution
  // (mean-removed when singular) is left in phi(). Reads back only the small
  // report (one device->host copy of the flags + 3 scalars).
  void solve(cudaStream_t s, const double* b_dev, double tol, int maxit);
  // Same but leaves the report on the device (no host synchronisation);
  // read it later with fetch_report().
  void solve_async(cudaStream_t s, const double* b_dev, double tol, int maxit,
                   double* report = nullptr, const WarmStart* ws = nullptr);
  nb_poisson_report fetch_report(cudaStream_t s);
  // After fetch_report: a bounded device-side wait of the solve gave up.
  bool timed_out() const;
  // Issues the whole solve into stream `s`, which must be capturing a graph:
  // the cycle loop becomes a conditional WHILE node (no host round trip).
  // `report` (6 doubles, device) receives iterations, stop code, early-exit
  // flag, |rhs|^2, |true residual|^2 and the NaN flag. `body_kernels`
  // receives the kernel count of one loop-body execution.
  void capture_solve(cudaStream_t s, const double* b_dev, double tol, int maxit, double* report,
                     uint64_t* body_kernels, const WarmStart* ws = nullptr);
  static nb_poisson_report report_from(const double* r, double tol);
  // Number of loop-body executions so far (device counter).
  unsigned long long* body_execs() const { return body_execs_; }
  void set_counter(std::atomic<uint64_t>* c) { lc_.count = c; }
  std::atomic<uint64_t>* counter() const { return lc_.count; }

  // out = A x (CgPoisson::applyA on level 0), brick layout.
  void apply_a(cudaStream_t s, const double* x, double* out);

  const double* phi() const { return xfin_; }
  const LevelView& view0() const { return lv_[0].v; }
  const HostLevel& host0() const { return lv_[0].h; }
  bool singular() const { return singular_; }
  uint64_t device_bytes() const { return bytes_; }
  int levels() const { return static_cast<int>(lv_.size()); }
  double* scalars() const { return S_; }
  SolveFlags* flags() const { return flags_; }

  // Scratch reduction buffer shared with the flow kernels of the same stream.
  RedBuf red() const { return rb_; }

 private:
  // With `prog` the launches are recorded as tail phases instead (no stream).
  template <typename T>
  void vcycle(cudaStream_t s, int lvl, const void* b, int bmean_slot, void* xout_final,
              int* out_mean_slot, void** out_x, std::vector<TailPhase>* prog = nullptr, bool first_done = false);
  void build_tail();
  void launch_tail(cudaStream_t s);
  void build_grid();
  void mark_bf16();
  void launch_grid(cudaStream_t s, const void* b);
  void iterate(cudaStream_t s, double tol, int maxit, int count);
  void setup(cudaStream_t s, const double* b, double tol, int maxit, const WarmStart* ws = nullptr);
  void first_direction(cudaStream_t s);
  void capture_refinement(cudaStream_t s, double tol, int maxit);
  void finish(cudaStream_t s, double* report);
  void upload_uniform(DevLevel& D, const int bcs[6]);
  void upload_amr(DevLevel& D, const AmrLevelHost& A, const int bcs[6]);
  void build_halo_maps();
  bool build_dense_coarse();
  void common_alloc();
  void* alloc(size_t bytes);
  void set_tuning(const nb_tuning* tune);
  int grid_of(int nbrick) const { return nbrick < grid_cap_ ? nbrick : grid_cap_; }
  int grid_cap_ = 0;   // CTAs of the brick kernels
  int tpb_ = 512;      // threads per CTA of the smoother, residual and matvec kernels
  bool pdl_ = true;    // programmatic dependent launch of the chains
  int sweeps_ = 2;     // smoothing sweeps per side of the coarse correction
  int halo_mode_ = 0;  // 0 per-brick neighbour maps, 1 per-cell walk
  int direct_max_ = 256;  // exact coarsest solve up to this many cells
  int tail_bricks_ = 0;   // cluster tail from the first level (>= 1) of at most this many bricks; 0 off
  int tail_lvl_ = -1;     // first level of the tail (-1: no tail)
  int tail_cs_ = 0;       // CTAs of the tail's cluster
  size_t tail_smem_ = 0;  // dynamic shared memory of the tail (coarsest solve)
  TailProg* tail_prog_ = nullptr;  // device
  void* tail_x_ = nullptr;         // tail level's result and its pending-mean slot
  int tail_slot_ = -1;
  double tail_bytes_ = 0.0;        // algorithmic bytes of one tail launch
  bool vgrid_ = false;          // tuning: run each V-cycle as one grid-resident launch
  bool coarse_bf16_ = false;    // tuning: BF16 residuals on the levels between the finest and the tail
  GridProg* grid_prog_ = nullptr;  // device; nullptr: per-sweep launches
  GridProg* grid_prog_alt_ = nullptr;  // FP64: the same program on the other residual buffer
  const void* grid_b_ = nullptr;       // level-0 rhs grid_prog_ reads
  int grid_ctas_ = 0;
  size_t grid_smem_ = 0;
  double grid_bytes_ = 0.0;       // algorithmic bytes of one grid V-cycle
  void* grid_x_ = nullptr;        // level-0 result of the grid V-cycle and its pending-mean slot
  int grid_slot_ = -1;
  unsigned* grid_sync_ = nullptr;
  bool cheb_ = false;     // mixed form: Chebyshev smoothing instead of damped Jacobi
  double cheb_c2_[4] = {0.8, 0.8, 0.8, 0.8};  // residual weight per sweep of a phase
  double cheb_c1_[4] = {0.0, 0.0, 0.0, 0.0};  // weight of the last step per sweep
  // Exact coarsest-level solve (composite hierarchies only): the inverse of the
  // fluid block of the coarsest operator (regularised on the constant mode when
  // singular), host-factored once.
  bool dense_ = false;
  int dense_nf_ = 0;
  double* dense_inv_ = nullptr;   // [nf][nf]
  int* dense_fmap_ = nullptr;     // fluid row q -> level cell (brick layout)
  int* dense_lexpos_ = nullptr;   // level cell m (lexicographic) -> fluid row or -1
  int* dense_lexcell_ = nullptr;  // level cell m (lexicographic) -> brick-layout index
  cudaStream_t side_ = nullptr;               // capture stream of the loop body
  unsigned long long* body_execs_ = nullptr;  // device counter

  std::vector<DevLevel> lv_;
  bool singular_ = false;
  int precision_ = NB_PRECISION_FP64;
  double tol_ = 1e-9;
  int maxit_ = 100;
  size_t n0_ = 0;  // level-0 slots (nbrick * 512)
  // level-0 PCG vectors (FP64)
  double *rhs_ = nullptr, *x_ = nullptr, *r_ = nullptr, *rnew_ = nullptr, *z_ = nullptr,
         *p_ = nullptr, *p2_ = nullptr, *Ap_ = nullptr, *xfin_ = nullptr;  // p_ / p2_: last / next direction
  bool fuse_dots_ = false;  // level 0's last post-sweep also forms z' and the PCG dots (non-singular)
  float* rnew_f_ = nullptr;  // mixed form: FP32 copy of the V-cycle input
  float* z_f_ = nullptr;     // mixed form: FP32 V-cycle output
  double* S_ = nullptr;
  SolveFlags* flags_ = nullptr;
  SolveFlags* h_flags_ = nullptr;  // pinned
  double* h_S_ = nullptr;          // pinned
  RedBuf rb_;
  std::vector<void*> allocs_;
  uint64_t bytes_ = 0;
  LaunchCounter lc_;
};

}  // namespace nb
