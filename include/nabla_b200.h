/*
 * nabla_b200.h — C ABI of the B200 (sm_100a) per-step fluid update.
 *
 * The path: WENO-5 advection inside SSP-RK3 stages, each stage followed by a
 * pressure projection solved with geometric-multigrid-preconditioned CG
 * (MG-PCG), on a MAC grid stored as 8x8x8-cell bricks in Morton order.
 *
 * Every entry point takes plain pointers and sizes; no C++ or torch types
 * cross this boundary. Host arrays use the reference's lexicographic layouts
 * (x fastest): u is (nx+1)*ny*nz, v nx*(ny+1)*nz, w nx*ny*(nz+1), cell arrays
 * nx*ny*nz (core/include/nabla/flow/ns_solver.hpp:94-111).
 *
 * Errors: every call returns an nb_status. NB_OK is 0. A failed call leaves a
 * message retrievable with nb_last_error(ctx). Solver non-convergence is not
 * an error: it is reported in the report structs (as the reference reports
 * PoissonSolver::Report::converged, core/include/nabla/flow/poisson.hpp:24-28).
 */
#ifndef NABLA_B200_H
#define NABLA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum nb_status {
  NB_OK = 0,
  NB_ERR_BAD_ARG = 1,        /* invalid pointer, size or option */
  NB_ERR_OOM = 2,            /* device allocation failed / over budget */
  NB_ERR_NOT_CONVERGED = 3,  /* only returned where a caller asked for strict convergence */
  NB_ERR_NAN = 4,            /* NaN/Inf detected in a solver input or state */
  NB_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait gave up */
  NB_ERR_CUDA = 6,           /* CUDA runtime error */
  NB_ERR_UNSUPPORTED = 7     /* configuration outside what this build implements */
} nb_status;

/* ---- boundary description: mirrors core/include/nabla/flow/grid.hpp:17-26 */
enum { NB_BC_WALL = 0, NB_BC_INLET = 1, NB_BC_OUTLET = 2, NB_BC_PERIODIC = 3 };
enum { NB_PROFILE_UNIFORM = 0, NB_PROFILE_PARABOLIC = 1 };
enum { NB_CONV_CENTRAL = 0, NB_CONV_WENO5 = 1 };
/* Arithmetic forms of the step. PLAIN is FP64 throughout (the drop-in form).
 * MIXED runs WENO/RK stage arithmetic and the V-cycle in FP32 with FP64 PCG
 * dot products, search directions, true residuals, coarsest solve and the
 * final divergence check. */
enum { NB_PRECISION_FP64 = 0, NB_PRECISION_MIXED = 1 };

typedef struct nb_face_bc {
  int32_t type;             /* NB_BC_* (BoundaryType) */
  int32_t profile;          /* NB_PROFILE_* (InletProfile) */
  int32_t inlet_axis;       /* velocity component the inlet drives */
  int32_t reserved;
  double wall_velocity[3];  /* FaceBC::wallVelocity */
  double inlet_speed;       /* FaceBC::inletSpeed */
} nb_face_bc;

/* Uniform Cartesian grid: mirrors UniformGrid (grid.hpp:32-73). Face order
 * 0=-x 1=+x 2=-y 3=+y 4=-z 5=+z. `solid` is nx*ny*nz bytes (1 = obstacle) in
 * lexicographic order, or NULL for no obstacle. */
typedef struct nb_grid_desc {
  int32_t nx, ny, nz, reserved;
  double origin[3];
  double dx, dy, dz;
  nb_face_bc face[6];
  const uint8_t* solid;
} nb_grid_desc;

/* Mirrors FlowConfig (core/include/nabla/flow/ns_solver.hpp:14-32). */
typedef struct nb_flow_config {
  double reynolds, ref_length, velocity_scale, density, cfl;
  double body_force[3];
  int32_t convection;         /* NB_CONV_* */
  int32_t poisson_max_iters;
  double poisson_tol;
  double tol_continuity, tol_mass;
  double ref_area;
} nb_flow_config;

/* Mirrors StepReport (ns_solver.hpp:34-49). */
typedef struct nb_step_report {
  int32_t step;
  int32_t poisson_iters;
  double t, dt, cfl;
  double momentum_residual, continuity_residual, divergence_max, mass_error;
  double poisson_residual, cd, cl;
  uint64_t cell_count;
  int32_t accepted;
  int32_t converged;          /* all three projections converged */
} nb_step_report;

/* Mirrors PoissonSolver::Report (poisson.hpp:24-28). */
typedef struct nb_poisson_report {
  int32_t iterations;
  int32_t converged;
  double residual;
} nb_poisson_report;

typedef struct nb_ctx nb_ctx;
typedef struct nb_case nb_case;

/* ---- context ------------------------------------------------------------ */
/* Binds CUDA device `device`. Fails with NB_ERR_CUDA when no sm_100 device is
 * present: there is no CPU fallback. */
nb_status nb_ctx_create(int device, nb_ctx** out);
/* Releases the caller's handle. Cases and meshes hold the context too, so they
 * may be destroyed after it, in any order: it is freed with the last of them. */
void nb_ctx_destroy(nb_ctx* ctx);
const char* nb_last_error(const nb_ctx* ctx);
const char* nb_status_string(nb_status s);
/* Kernel launches issued by this context since creation (evidence counter). */
uint64_t nb_ctx_launch_count(const nb_ctx* ctx);
/* The context's cudaStream_t (batch graphs launch on it; for caller-side events). */
void* nb_ctx_stream(const nb_ctx* ctx);
nb_status nb_ctx_synchronize(nb_ctx* ctx);

/* ---- cases: one NS problem resident on the device ----------------------- */
/* Replaces NSSolver::NSSolver(UniformGrid, FlowConfig, shared_ptr<PoissonSolver>)
 * (core/src/flow/ns_solver.cpp:46-69) with the MG-PCG default solver
 * (ns_solver.cpp:49-53). The grid, BCs and solid mask are copied. */
nb_status nb_case_create(nb_ctx* ctx, const nb_grid_desc* grid, const nb_flow_config* cfg,
                         int precision, nb_case** out);
void nb_case_destroy(nb_case* c);
/* Replaces NSSolver::initialize (ns_solver.cpp:95-112). */
nb_status nb_case_initialize(nb_case* c);
/* Replaces NSSolver::setState (ns_solver.cpp:826-839): host arrays in the
 * reference's staggered lexicographic layout. */
nb_status nb_case_set_state(nb_case* c, const double* u, const double* v, const double* w,
                            const double* p, int step, double t, double dt_last);
/* Replaces the uFace()/vFace()/wFace()/pressure() accessors (ns_solver.hpp:76-80).
 * Any pointer may be NULL to skip that field. */
nb_status nb_case_get_state(nb_case* c, double* u, double* v, double* w, double* p);
nb_status nb_case_get_clock(nb_case* c, int* step, double* t, double* dt_last);
/* Replaces NSSolver::computeDt (ns_solver.cpp:581-603). */
nb_status nb_case_compute_dt(nb_case* c, double* dt);
/* Replaces NSSolver::step(double dt) (ns_solver.cpp:767-824); dt <= 0 selects
 * NSSolver::step() (ns_solver.cpp:765), i.e. dt from computeDt. `rep` may be NULL. */
nb_status nb_step(nb_case* c, double dt, nb_step_report* rep);
/* Runs `nsteps` fixed-dt steps without reading any report back (resident
 * throughput path); the last step's report is written to `rep` if non-NULL. */
nb_status nb_step_many(nb_case* c, double dt, int nsteps, nb_step_report* rep);
/* Batched stepping of independent cases (uniform or octree, FP64 or mixed)
 * created on `ctx`: each of the `nsteps` steps of all `n` cases is ONE CUDA
 * graph launch whose independent branches are the cases' own steps (their
 * dt from their CFL condition when dt <= 0, else the fixed dt; their
 * device-side MG-PCG loops), so the small kernels of different cases overlap
 * on the GPU. `reports` (n entries, may be NULL) receives each case's last
 * StepReport. The graph is built on first use for a given case list and
 * reused; destroying a case drops the graphs that contain it. No reference
 * counterpart: the reference steps one NSSolver at a time. */
nb_status nb_batch_step(nb_ctx* ctx, nb_case* const* cases, int n, double dt, int nsteps,
                        nb_step_report* reports);
/* Split form of nb_step for continuous batching: nb_step_async launches the
 * case's step graph on its stream and returns; nb_step_wait waits for it and
 * fills `rep` (may be NULL). Steps of different cases launched this way run
 * concurrently. One step in flight per case; not available while profiling. */
nb_status nb_step_async(nb_case* c, double dt);
nb_status nb_step_wait(nb_case* c, nb_step_report* rep);
/* Non-blocking completion test of the step in flight: *ready = 1 once
 * nb_step_wait would return without waiting, else 0. Lets a request loop
 * collect each case as soon as its own step ends, instead of waiting for all
 * of them in lockstep. No reference counterpart (the reference's job runner,
 * backend/app/jobs.py:50-140, runs one case at a time to completion). */
nb_status nb_step_ready(nb_case* c, int* ready);
/* Replaces SolverBackend::sample (core/include/nabla/adaptive/run.hpp:17), as
 * BaselineBackend implements it (core/src/adaptive/run.cpp:49-62), for n points
 * at once: out[q] = component `component` (0 = u, 1 = v, 2 = w: the average of
 * the two faces of the containing cell along that axis, NSSolver::cellU/V/W,
 * ns_solver.cpp:677-688; 3 = the cell's pressure) at point (xyz[3q], xyz[3q+1],
 * xyz[3q+2]). On octree cases the containing cell is the leaf cell. Cell
 * indices are truncated toward zero and clamped into the domain. xyz and out
 * are host arrays; one kernel launch for all points. */
nb_status nb_case_sample(nb_case* c, int component, int64_t n, const double* xyz, double* out);
/* Device bytes held by the case (admission control uses this). */
uint64_t nb_case_device_bytes(const nb_case* c);
/* Leaf cells of the case (Mcell-steps/s numerator). */
uint64_t nb_case_cell_count(const nb_case* c);
/* The cudaStream_t the case's kernels run on (for caller-side CUDA events). */
void* nb_case_stream(const nb_case* c);

/* ---- measurement ---------------------------------------------------------
 * Bracket every launch of one kernel family with CUDA events on its stream
 * (family names: "rhs_rk", "smooth", "resid_restrict", "coarse_cg",
 * "pcg_matvec", "pcg_update", "correct", "div", "diag"; NULL disables).
 * nb_ctx_profile_read returns the summed event time, the launch count and the
 * algorithmic bytes those launches had to move (each array read or written
 * once per cell; halos excluded). Reading resets the counters. */
nb_status nb_ctx_profile(nb_ctx* ctx, const char* family);
nb_status nb_ctx_profile_read(nb_ctx* ctx, double* total_ms, uint64_t* launches, double* bytes);

/* ---- launch tuning and the autotuner ---------------------------------------
 * No counterpart in the reference. A context's tuning applies to the cases,
 * meshes and Poisson hierarchies created after it is set; objects keep the
 * tuning they were created with. Bricks are fixed at 8^3 cells. */
typedef struct nb_tuning {
  int32_t mg_ctas_per_sm;    /* multigrid brick kernels: grid <= this x SMs (1..16) */
  int32_t rhs_ctas_per_sm;   /* momentum kernel: grid <= this x SMs (1..4) */
  int32_t halo_mode;         /* multigrid halo staging: 0 per-brick neighbour maps
                                (one round of independent loads), 1 per-cell walk */
  int32_t sweeps;            /* smoothing sweeps before and after each coarse
                                correction (1..3), mixed form; FP64 keeps 2 */
  int32_t coarse_direct_max; /* below multi-level meshes, solve coarsest levels of
                                up to this many cells exactly (0..512; 0 = CG) */
  int32_t pdl;               /* 1: multigrid chains use programmatic dependent launch */
  int32_t threads_per_brick; /* CTA size of the smoother, residual-restriction and
                                matvec kernels: 512, 256 or 128 (1, 2 or 4 cells
                                per thread; smaller CTAs keep more bricks in flight) */
  int32_t smoother;          /* mixed form: 1 (default) Chebyshev polynomial on
                                [lmax/6, lmax] of D^-1 A (same cost per sweep,
                                stronger smoothing), 0 damped Jacobi (omega 0.8);
                                the FP64 form always uses the reference's Jacobi */
  int32_t tail_bricks;       /* 0: one launch per multigrid sweep on every level;
                                n > 0 (default 8): the V-cycle from the first level
                                below the finest with at most n bricks down to the
                                coarsest solve runs as one thread-block-cluster
                                launch with those levels in shared memory (0..4096) */
  int32_t warm_start;        /* mixed form, the initial guess of each projection's MG-PCG:
                                0 zero; 1 the last pressure scaled to the RK stage;
                                2 the same RK stage's pressure extrapolated linearly in
                                time over the last two steps; 3 (default) that stage's
                                pressure one step ago plus the change of the previous
                                stage's pressure since, scaled to this stage. 2 and 3 are
                                scaled by this step's dt, use form 1 until two steps of
                                history are held, and restart their history on a new
                                state (so a checkpoint restart agrees with the continuous
                                run to the solver tolerance, not bitwise). The FP64 form
                                always starts from zero as the reference does */
  int32_t vgrid;             /* 0 (default): one launch per sweep (and the cluster
                                tail); 1: each V-cycle (all levels and the coarsest
                                solve) is ONE cooperative launch whose CTAs run the
                                sweeps, restrictions and prolongations phase by phase
                                with a grid barrier between phases (a barrier that waits
                                over a second ends the solve with NB_ERR_DEVICE_TIMEOUT) */
  int32_t coarse_bf16;       /* mixed form: 1 stores the restricted residual of the
                                multigrid levels between the finest and the cluster tail
                                in BF16 (rounded to nearest; BF16 keeps FP32's exponent
                                range, so no per-brick scale is needed), 0 (default)
                                FP32; arithmetic stays FP32 and the PCG FP64 */
  int32_t ghost_map;         /* octree cases: 1 (default) the momentum kernel replays a
                                per-case map of the ghost rules' recorded forms for the
                                halo points that are not same-level cells (built when the
                                case is created, about 60 B per leaf cell); 0 walks the
                                ghost rules for those points at every stage (no map) */
} nb_tuning;

typedef struct nb_tune_report {
  nb_tuning best;
  double best_ms;            /* per step, fastest candidate */
  double default_ms;         /* per step, nb_tuning_default */
  int32_t candidates;        /* candidates timed (0 when taken from the cache) */
  int32_t rejected;          /* candidates whose steps did not converge */
  int32_t from_cache;
  char key[128];             /* cache key: GPU, SM count, mesh kind, precision, size class */
} nb_tune_report;

void nb_tuning_default(nb_tuning* t);
nb_status nb_ctx_set_tuning(nb_ctx* ctx, const nb_tuning* t);
nb_status nb_ctx_get_tuning(const nb_ctx* ctx, nb_tuning* t);
/* Picks the tuning for cases like `sample` and sets it on the context:
 * coordinate descent over the fields of nb_tuning from the default, each
 * candidate timed over `steps` fixed-dt steps (CUDA events, after one warm-up
 * step) on a scratch copy of `sample` (same mesh or grid, configuration,
 * precision and current state); a candidate is kept only if it is at least 2%
 * faster and its steps converge with divergence <= 1e-8. With `cache_path`
 * (a text file, one line per key) a cached entry for the key is used without
 * timing, and a new result is written back. `sample` is not modified. */
nb_status nb_autotune(nb_ctx* ctx, nb_case* sample, int steps, const char* cache_path, nb_tune_report* rep);
/* Cache file access (host only): 1 if `key` was found, 0 if not; negative on
 * an unreadable or malformed file. */
int nb_tune_cache_lookup(const char* cache_path, const char* key, nb_tuning* t, double* ms);
nb_status nb_tune_cache_store(const char* cache_path, const char* key, const nb_tuning* t, double ms);

/* ---- pressure Poisson: the PoissonSolver seam ---------------------------- */
/* Replaces MgPoisson::solve (core/src/flow/multigrid.cpp:206-355) behind
 * PoissonSolver::solve(const UniformGrid&, const std::vector<double>& b,
 * std::vector<double>& x) (core/include/nabla/flow/poisson.hpp:31-32).
 * b and x are host arrays of nx*ny*nz doubles. The multigrid hierarchy is
 * cached on the context keyed by the grid (multigrid.cpp:43-61, :211-266). */
nb_status nb_poisson_solve(nb_ctx* ctx, const nb_grid_desc* grid, const double* b, double* x,
                           double tol, int max_cycles, int precision, nb_poisson_report* rep);
/* Replaces CgPoisson::applyA (core/src/flow/poisson.cpp:102-134). */
nb_status nb_apply_laplacian(nb_ctx* ctx, const nb_grid_desc* grid, const double* x, double* out);

/* ---- octree-AMR brick meshes ------------------------------------------------
 * A mesh is a set of leaf bricks of 8x8x8 cells at octree levels 0..lmax over
 * a base grid of nb0 bricks per axis at level 0 (cell size h0 / 2^level),
 * 2:1 balanced across faces, edges and corners. A leaf is 4 int32 values:
 * (level, bx, by, bz) in level-`level` brick coordinates. Cell arrays over a
 * mesh are nleaf*512 doubles: leaves in the mesh's rank order (Morton order
 * of the leaf anchors on the finest level, the key of
 * core/include/nabla/mesh/morton.hpp:19-48), cells x-fastest inside a brick.
 * Replaces the reference's leaves-only linear Octree (core/src/mesh/octree.cpp)
 * for the flow path; its face rule follows OctreePoisson
 * (core/src/flow/octree_poisson.cpp:24-105). */
typedef struct nb_amr_geom {
  int32_t nb0[3];
  int32_t lmax;
  double h0[3];
  double origin[3];
  nb_face_bc face[6];
} nb_amr_geom;

typedef struct nb_amr_mesh nb_amr_mesh;

/* Splits the flagged leaves (flags[i] != 0) and restores 2:1 balance
 * (Octree::refineByMorton's balance, core/src/mesh/octree.cpp:325-356, at
 * brick granularity and over all 26 neighbours). `out` receives the new leaf
 * list (4 int32 each, any order) when `cap` is large enough; `n_out` always
 * receives the required count (NB_ERR_BAD_ARG if cap is too small). */
nb_status nb_amr_refine(const nb_amr_geom* g, const int32_t* leaves, int64_t n, const uint8_t* flags,
                        int32_t* out, int64_t cap, int64_t* n_out);
/* Builds a mesh from a leaf list (validated: coverage, no overlap, balance).
 * `solid` (optional) holds 512 bytes per leaf in the INPUT order. */
nb_status nb_amr_mesh_create(nb_ctx* ctx, const nb_amr_geom* g, const int32_t* leaves, int64_t n,
                             const uint8_t* solid, nb_amr_mesh** out);
void nb_amr_mesh_destroy(nb_amr_mesh* m);
int64_t nb_amr_mesh_leaf_count(const nb_amr_mesh* m);
/* Leaves in rank order (4 int32 each). */
nb_status nb_amr_mesh_leaves(const nb_amr_mesh* m, int32_t* out);
/* Composite -Laplacian per unit volume, (A x)_i = (1/V_i) sum_f area_f/dist_f
 * (x_i - x_n): OctreePoisson::applyA (core/src/flow/octree_poisson.cpp:64-85)
 * divided by the cell volume, plus the uniform operator's outlet (Dirichlet)
 * and periodic closures (core/src/flow/poisson.cpp:18-52). Solid rows identity. */
nb_status nb_amr_apply_laplacian(nb_ctx* ctx, nb_amr_mesh* m, const double* x, double* out);
/* MG-PCG on the composite operator (volume-weighted inner products and means;
 * composite V-cycle merging the finest octree level per MG level, then the
 * uniform coarsening of core/src/flow/multigrid.cpp:211-266). */
nb_status nb_amr_poisson_solve(nb_ctx* ctx, nb_amr_mesh* m, const double* b, double* x, double tol,
                               int max_cycles, int precision, nb_poisson_report* rep);

/* ---- integer maps of octree brick meshes ------------------------------------
 * Keys: the Morton key of a leaf's anchor on the finest level (leaf (L, b)
 * anchors at b << (lmax - L)), with x in the lowest bit of each triple: the
 * key of core/include/nabla/mesh/morton.hpp:19-48 (mortonEncode/Decode), 21
 * bits per axis. Rank order = ascending key.
 * Face-neighbour table: for rank r and face d (0 -x, 1 +x, 2 -y, 3 +y, 4 -z,
 * 5 +z), nnbr[6r+d] neighbours in nbr[24r+4d .. +3] (unused entries -1): the
 * rule of Octree::faceNeighbors (core/src/mesh/octree.cpp:229-283) at brick
 * granularity: the coarser-or-equal leaf holding the brick across the face,
 * else the 2x2 leaves one level finer on the touching side, in the
 * reference's order (k1 over axis (d/2+1)%3 outer, k2 over axis (d/2+2)%3
 * inner); none across a non-periodic domain face; periodic axes wrap. */
uint64_t nb_morton_encode(uint32_t x, uint32_t y, uint32_t z);
void nb_morton_decode(uint64_t key, uint32_t* x, uint32_t* y, uint32_t* z);
/* Builds the rank order and the face-neighbour table of a leaf list (any
 * order, any 2:1 face balance) on the device: keys (n, sorted), order (n:
 * input position of rank r), nbr (24n), nnbr (6n), all host arrays. A leaf
 * outside the geometry or two leaves with one anchor: NB_ERR_BAD_ARG. */
nb_status nb_amr_build_maps(nb_ctx* ctx, const nb_amr_geom* g, const int32_t* leaves, int64_t n, uint64_t* keys,
                            int32_t* order, int32_t* nbr, int32_t* nnbr);
/* The same keys and table of an existing mesh, read from the host tree its
 * kernels' maps are built from (rank order, per-level lookup tables). */
nb_status nb_amr_mesh_maps(const nb_amr_mesh* m, uint64_t* keys, int32_t* nbr, int32_t* nnbr);
/* Host only (no device, no context): the tree nb_amr_mesh_create would build
 * from this leaf list (coverage and 26-neighbour balance validated,
 * NB_ERR_BAD_ARG otherwise), its keys, its leaves in rank order (ranked: 4n)
 * and its face-neighbour table. */
nb_status nb_amr_tree_maps(const nb_amr_geom* g, const int32_t* leaves, int64_t n, uint64_t* keys, int32_t* ranked,
                           int32_t* nbr, int32_t* nnbr);
/* The coarse-fine couplings of the mesh's composite operator: CSR over the
 * mesh's cells (off: cells+1 entries), each coupling a neighbour cell index
 * (rank * 512 + local cell) and its per-unit-volume coefficient (the face
 * rule of OctreePoisson::faceCoeff, core/src/flow/octree_poisson.cpp:24-32,
 * over the cell volume). *count always receives the number of couplings;
 * pass NULL arrays to query it, else cap >= *count. */
nb_status nb_amr_mesh_couplings(const nb_amr_mesh* m, int64_t* count, int32_t* off, int32_t* nbr, double* coef,
                                int64_t cap);

/* The same refinement as nb_amr_refine (split the flagged leaves below lmax,
 * then restore 26-neighbour 2:1 balance), computed on the device: leaves are
 * ranked by a device sort of their keys, every split leaf marks the touching
 * leaves two or more levels coarser than its children through binary searches
 * in the sorted keys, round by round until nothing changes (at most lmax + 1
 * rounds), and the new leaves are emitted and ranked on the device. `out`
 * receives them in rank order; same error and capacity convention as
 * nb_amr_refine. Replaces Octree::refineByMorton with its balance
 * (core/src/mesh/octree.cpp:325-356) at brick granularity. */
nb_status nb_amr_refine_device(nb_ctx* ctx, const nb_amr_geom* g, const int32_t* leaves, int64_t n,
                               const uint8_t* flags, int32_t* out, int64_t cap, int64_t* n_out);

/* ---- MAC step on an octree-AMR mesh ------------------------------------------
 * NSSolver (core/include/nabla/flow/ns_solver.hpp:58-96) on the composite
 * mesh: the same SSP-RK3 / WENO-5 / MG-PCG step, with the octree face rule of
 * OctreePoisson (core/src/flow/octree_poisson.cpp:24-32) at 2:1 interfaces.
 * The returned case is driven by nb_case_initialize, nb_case_compute_dt,
 * nb_step, nb_step_many, nb_case_destroy; the mesh must outlive it. BCs come
 * from the mesh geometry's faces.
 * Face storage of component a (0 u, 1 v, 2 w): nbrick*512 + nslab*64 doubles.
 * Slot r*512 + l is the low a-face of cell l of leaf r; slab s holds the 64
 * high a-faces (local index a-th coordinate 8, the other two x-fastest) of
 * leaf slabs[s] (nb_amr_case_slabs). A leaf has an a-slab iff its +a
 * neighbour is not a same-level leaf. On periodic axes the domain high face
 * is the low face of the first cell (no second copy). At a 2:1 interface the
 * fine side's four sub-faces are the state; the coarse face is their average
 * (overwritten on every update). Pressure: nbrick*512 cell values. */
nb_status nb_amr_case_create(nb_ctx* ctx, nb_amr_mesh* m, const nb_flow_config* cfg, int precision,
                             nb_case** out);
/* Merges each complete octet of sibling leaves whose eight members are all
 * flagged into its parent (Octree::coarsen, core/src/mesh/octree.cpp:393-473,
 * at brick granularity: all eight children must be leaves, and the merge is
 * refused where the parent would sit next to a leaf two levels finer, here over
 * all 26 neighbours with periodic wrap since these meshes are balanced across
 * edges and corners too). Same output convention as nb_amr_refine. */
nb_status nb_amr_coarsen(const nb_amr_geom* g, const int32_t* leaves, int64_t n, const uint8_t* flags,
                         int32_t* out, int64_t cap, int64_t* n_out);
/* Per-leaf refinement sensors of an octree case, the velocity-gradient
 * sensors of PhysicalSensorEvaluator::evaluate (core/src/adaptive/
 * adaptive_core.cpp:96-113) on brick cells: out[4 r + 0..3] = the maximum over
 * leaf r's fluid cells of |vorticity|, sqrt(2 S:S), Q and |grad p| (cell-centred
 * values, central differences inside the brick, one-sided on its faces). */
nb_status nb_amr_case_sensors(nb_case* c, double* out);
/* Regrid refinement on the device: the case's sensors (as nb_amr_case_sensors,
 * never leaving the device) flag the leaves whose sensor `sensor` exceeds
 * `above` (below lmax), and nb_amr_refine_device's split, balance and ranking
 * run on them. `out` receives the new leaves in rank order (4 int32 each);
 * `n_out` always receives their count (NB_ERR_BAD_ARG if cap is too small).
 * The sensor and split rules of PhysicalSensorEvaluator / Octree::refine
 * (core/src/adaptive/adaptive_core.cpp:96-113, core/src/mesh/octree.cpp:288-356). */
nb_status nb_amr_case_refine(nb_case* c, int sensor, double above, int32_t* out, int64_t cap, int64_t* n_out);
/* Regrid transfer: dst (a fresh case on a mesh from nb_amr_refine or
 * nb_amr_coarsen of src's mesh: same geometry, at most one level apart at every
 * leaf) takes src's state and step clock. Every face dst stores takes src's
 * value at that face: the same face, the average of four finer sub-faces, or
 * the coarse face (or, mid-cell, the mean of the coarse cell's two normal
 * faces), so a divergence-free field stays divergence-free; pressure is copied,
 * injected from the coarser cell or averaged over the eight finer cells. */
nb_status nb_amr_case_transfer(nb_case* dst, nb_case* src);
/* sizes[0..2] = face storage lengths of u, v, w; sizes[3] = cells. */
nb_status nb_amr_case_sizes(const nb_case* c, int64_t sizes[4]);
/* Leaf rank of every a-slab, in slab order ((sizes[a] - cells) / 64 values). */
nb_status nb_amr_case_slabs(const nb_case* c, int axis, int32_t* bricks);
nb_status nb_amr_case_set_state(nb_case* c, const double* u, const double* v, const double* w, const double* p);
/* Any pointer may be NULL to skip that field. */
nb_status nb_amr_case_get_state(nb_case* c, double* u, double* v, double* w, double* p);

/* ---- checkpoints ------------------------------------------------------------
 * Replace writeCheckpoint / readCheckpoint (core/src/flow/case.cpp:244-319).
 * Uniform cases use the reference's NBFCK01 layout: 8 magic bytes "NBFCK01\0",
 * int32 nx, ny, nz, int32 step, FP64 t, FP64 dt, then u, v, w, p each as a
 * uint64 count and that many FP64 values in the reference's lexicographic MAC
 * layout, host byte order; a file moves between the reference and this library
 * in either direction. Octree cases (no reference counterpart) use NBFAMR1:
 * magic, int32 leaf count, the leaves (4 int32 each, rank order), int32 step,
 * FP64 t, FP64 dt, then the u, v, w face arrays in storage order and p, each
 * count-prefixed. Reading checks the magic, the grid dimensions or leaf list
 * and every array size (NB_ERR_BAD_ARG otherwise) and restores the step clock:
 * a restart continues bit for bit. */
nb_status nb_case_write_checkpoint(nb_case* c, const char* path);
nb_status nb_case_read_checkpoint(nb_case* c, const char* path);
/* Host only: header of a checkpoint file. kind 0 = NBFCK01 (dims set),
 * 1 = NBFAMR1 (nleaf set). Returns 0, or -1 for an unreadable or foreign file. */
int nb_checkpoint_info(const char* path, int32_t* kind, int32_t dims[3], int64_t* nleaf, int32_t* step,
                       double* t, double* dt);

/* ---- field output -------------------------------------------------------------
 * Replaces writeGridVtu (core/src/flow/case.cpp:175-241): a VTK XML
 * unstructured grid, one hexahedron per cell (8 corners in VTK order), ASCII
 * values at 8 significant digits, cell data u, v, w (cell-centred, NSSolver::
 * cellVelocity), p, speed and solid. Uniform cases list cells in the
 * reference's lexicographic order; octree cases list every leaf cell (leaves in
 * rank order, cells x-fastest) and add an Int32 `level` array, as the octree
 * writer does (core/src/io/vtu_writer.cpp:8-80). */
nb_status nb_case_write_vtu(nb_case* c, const char* path);

/* ---- case run loop ------------------------------------------------------------
 * Replaces runCase (core/src/flow/case.cpp:349-401), the loop behind
 * `nabla_solve run`: create and initialize the case, optionally restart from
 * a checkpoint, then step (dt from computeDt) up to max_steps times, appending
 * one diagnostics.jsonl record per step in the reference's schema and number
 * formatting (a provenance line first in a fresh file), writing
 * checkpoint_<step>.ckpt every checkpoint_every steps, snapshot_<step>.vtu
 * every snapshot_every steps, final.vtu and final.ckpt at the end (files as
 * nb_case_write_vtu / nb_case_write_checkpoint write them), stopping at
 * stop_time or when the momentum residual falls below steady_tol after step 20. */
typedef struct nb_run_options {
  const char* run_dir;        /* RunOptions::runDir (created if missing) */
  int32_t max_steps;          /* RunOptions::maxSteps */
  int32_t checkpoint_every;   /* RunOptions::checkpointEvery (0: final only) */
  double stop_time;           /* RunOptions::stopTime (0: ignore) */
  double steady_tol;          /* RunOptions::steadyTol (0: ignore) */
  const char* restart_from;   /* RunOptions::restartFrom (NULL or "": fresh run) */
  int32_t precision;          /* NB_PRECISION_* */
  int32_t snapshot_every;     /* RunOptions::snapshotEvery: snapshot_<step>.vtu (0: final.vtu only) */
} nb_run_options;

typedef struct nb_run_summary {  /* mirrors RunSummary (case.hpp:29-40) */
  int32_t steps;
  int32_t steady;
  double time, momentum_residual, continuity_residual, mass_error, cd, cl;
  uint64_t cells;
} nb_run_summary;

nb_status nb_run_case(nb_ctx* ctx, const nb_grid_desc* grid, const nb_flow_config* cfg, const nb_run_options* opt,
                      nb_run_summary* out);

/* ---- allocation-free operator ---------------------------------------------
 * No counterpart in the reference. The same -Laplacian as nb_apply_laplacian,
 * for callers that cannot call cudaMalloc: hosts that own all device memory
 * through their own arena or admission budget, and loops that must not stall
 * on the allocator's implicit synchronisation. `x` and `out` are the caller's DEVICE arrays of
 * nx*ny*nz doubles in lexicographic order; `stream` is a cudaStream_t (NULL =
 * legacy default stream) on the current device. No context is needed and
 * nothing is allocated: the solid mask (grid->solid, host memory, or NULL) is
 * staged into a static device array of NB_NOALLOC_MAX_CELLS bytes that every
 * GPU loading this library holds until exit. Grids with more cells are
 * rejected with NB_ERR_UNSUPPORTED. The first call on a device looks up that
 * array's device address; make it before any stream capture. All calls share
 * the array: calls that overlap on the GPU race and must be serialised. */
#define NB_NOALLOC_MAX_CELLS (16u * 1024u * 1024u)
nb_status nb_apply_laplacian_noalloc(const nb_grid_desc* grid, const double* x, double* out,
                                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NABLA_B200_H */
