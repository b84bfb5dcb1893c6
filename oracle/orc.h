/* orc.h — TEST INFRASTRUCTURE ONLY.
 *
 * The oracle: a plain-C CPU restatement of the reference's per-step fluid
 * update, used only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the checker. Nothing in the product links or calls it.
 *
 * Uniform path (restate.c) follows core/src/flow/{ns_solver,poisson,multigrid}.cpp.
 * Octree maps + octree operator (restate_octree.c) follow core/src/mesh/octree.cpp,
 * core/include/nabla/mesh/morton.hpp and core/src/flow/octree_poisson.cpp.
 * Multi-level MAC step (restate_amr.c) has no reference counterpart; it is
 * pinned to the uniform restatement on single-level meshes.
 */
#ifndef ORC_H
#define ORC_H
#include <stdint.h>

#include "nabla_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- uniform Poisson (core/src/flow/poisson.cpp, multigrid.cpp) ---- */
void orc_apply_a(const nb_grid_desc* g, const double* x, double* out);
void orc_build_diagonal(const nb_grid_desc* g, double* diag);
int orc_cg_solve(const nb_grid_desc* g, const double* b, double* x, double tol, int maxit,
                 nb_poisson_report* rep);
int orc_mg_solve(const nb_grid_desc* g, const double* b, double* x, double tol, int maxit,
                 nb_poisson_report* rep);

/* ---- uniform NS step (core/src/flow/ns_solver.cpp) ---- */
typedef struct orc_ns orc_ns;
orc_ns* orc_ns_create(const nb_grid_desc* g, const nb_flow_config* cfg);
void orc_ns_destroy(orc_ns* s);
void orc_ns_initialize(orc_ns* s);
void orc_ns_set_state(orc_ns* s, const double* u, const double* v, const double* w,
                      const double* p, int step, double t, double dt_last);
void orc_ns_get_state(const orc_ns* s, double* u, double* v, double* w, double* p);
double orc_ns_compute_dt(const orc_ns* s);
void orc_ns_step(orc_ns* s, double dt, nb_step_report* rep);

/* ---- MAC step on an octree mesh of 8^3 leaf bricks (restate_amr.c) ----
 * No reference counterpart; restates the rules of the brick path on dense
 * per-level arrays. Leaves: 4 int32 each (level, bx, by, bz); solid: 512
 * bytes per leaf in the same order (or NULL). Faces are addressed by (level,
 * i, j, k) in level-level face indices, comp 3 addresses cells. */
typedef struct orc_amr orc_amr;
orc_amr* orc_amr_create(const nb_amr_geom* g, const int32_t* leaves, int64_t n, const uint8_t* solid,
                        const nb_flow_config* cfg);
void orc_amr_destroy(orc_amr* A);
void orc_amr_set(orc_amr* A, int comp, int64_t n, const int32_t* lev, const int32_t* i, const int32_t* j,
                 const int32_t* k, const double* val);
void orc_amr_get(orc_amr* A, int comp, int64_t n, const int32_t* lev, const int32_t* i, const int32_t* j,
                 const int32_t* k, double* val);
double orc_amr_step(orc_amr* A, double dt, double tol, int* cg_iters);

/* ---- Morton + linear octree (core/include/nabla/mesh/morton.hpp, core/src/mesh/octree.cpp) ---- */
uint64_t orc_morton_encode(uint32_t x, uint32_t y, uint32_t z);
void orc_morton_decode(uint64_t code, uint32_t* x, uint32_t* y, uint32_t* z);

#ifdef __cplusplus
}
#endif
#endif
