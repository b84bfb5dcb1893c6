/* restate.c — TEST INFRASTRUCTURE ONLY: the oracle's CPU restatement of the
 * reference's uniform MAC step and pressure solvers, in plain C (FP64).
 *
 * Each function names the reference lines (paths within the reference
 * project) whose arithmetic it restates. Loop orders and the association of
 * every floating-point expression follow the reference so that results agree
 * to rounding; the file is compiled with -ffp-contract=off.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc.h"

/* ------------------------------------------------------------------------ */
/* grid helpers: core/include/nabla/flow/grid.hpp:37-72                      */
/* ------------------------------------------------------------------------ */
static size_t cidx(const nb_grid_desc* g, int i, int j, int k) {
  return (size_t)i + (size_t)g->nx * ((size_t)j + (size_t)g->ny * (size_t)k);
}
static size_t ncell(const nb_grid_desc* g) { return (size_t)g->nx * g->ny * g->nz; }
static int is_solid(const nb_grid_desc* g, int i, int j, int k) {
  if (i < 0 || i >= g->nx || j < 0 || j >= g->ny || k < 0 || k >= g->nz) return 0;
  return g->solid != NULL && g->solid[cidx(g, i, j, k)] != 0;
}
static int periodic(const nb_grid_desc* g, int axis) {
  return g->face[2 * axis].type == NB_BC_PERIODIC;
}
static int has_dirichlet(const nb_grid_desc* g) { /* poisson.cpp:93-100 */
  for (int f = 0; f < 6; ++f)
    if (g->face[f].type == NB_BC_OUTLET) return 1;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* -Laplacian: core/src/flow/poisson.cpp:18-134                              */
/* ------------------------------------------------------------------------ */
/* kind 0 = no coupling, 1 = interior neighbour n, 2 = Dirichlet (poisson.cpp:18-52) */
static int resolve_face(const nb_grid_desc* g, int i, int j, int k, int axis, int side,
                        size_t* n) {
  int c[3] = {i, j, k};
  const int dims[3] = {g->nx, g->ny, g->nz};
  c[axis] += side;
  if (c[axis] >= 0 && c[axis] < dims[axis]) {
    if (is_solid(g, c[0], c[1], c[2])) return 0;
    *n = cidx(g, c[0], c[1], c[2]);
    return 1;
  }
  const int face = 2 * axis + (side > 0 ? 1 : 0);
  const int bt = g->face[face].type;
  if (bt == NB_BC_PERIODIC) {
    c[axis] = (c[axis] + dims[axis]) % dims[axis];
    if (is_solid(g, c[0], c[1], c[2])) return 0;
    *n = cidx(g, c[0], c[1], c[2]);
    return 1;
  }
  if (bt == NB_BC_OUTLET) return 2;
  return 0;
}

static double diag_of(const nb_grid_desc* g, int i, int j, int k) { /* poisson.cpp:54-74 */
  const double h2[3] = {1.0 / (g->dx * g->dx), 1.0 / (g->dy * g->dy), 1.0 / (g->dz * g->dz)};
  double d = 0.0;
  for (int axis = 0; axis < 3; ++axis) {
    if (axis == 2 && g->nz == 1) continue;
    for (int side = -1; side <= 1; side += 2) {
      size_t n = 0;
      const int kind = resolve_face(g, i, j, k, axis, side, &n);
      if (kind == 1) d += h2[axis];
      else if (kind == 2) d += 2.0 * h2[axis];
    }
  }
  return d;
}

void orc_build_diagonal(const nb_grid_desc* g, double* diag) { /* poisson.cpp:78-91 */
  for (size_t c = 0; c < ncell(g); ++c) diag[c] = 1.0;
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        if (is_solid(g, i, j, k)) continue;
        const double d = diag_of(g, i, j, k);
        diag[cidx(g, i, j, k)] = (d > 0.0) ? d : 1.0;
      }
}

void orc_apply_a(const nb_grid_desc* g, const double* x, double* out) { /* poisson.cpp:102-134 */
  const double h2[3] = {1.0 / (g->dx * g->dx), 1.0 / (g->dy * g->dy), 1.0 / (g->dz * g->dz)};
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const size_t c = cidx(g, i, j, k);
        if (is_solid(g, i, j, k)) {
          out[c] = x[c];
          continue;
        }
        double diag = 0.0, off = 0.0;
        for (int axis = 0; axis < 3; ++axis) {
          if (axis == 2 && g->nz == 1) continue;
          for (int side = -1; side <= 1; side += 2) {
            size_t n = 0;
            const int kind = resolve_face(g, i, j, k, axis, side, &n);
            if (kind == 1) {
              diag += h2[axis];
              off += h2[axis] * x[n];
            } else if (kind == 2) {
              diag += 2.0 * h2[axis];
            }
          }
        }
        out[c] = diag * x[c] - off;
      }
}

static double dot(const double* a, const double* b, size_t n) {
  double s = 0.0;
  for (size_t m = 0; m < n; ++m) s += a[m] * b[m];
  return s;
}

/* Jacobi-PCG: core/src/flow/poisson.cpp:136-252 */
int orc_cg_solve(const nb_grid_desc* g, const double* b, double* x, double tol, int maxit,
                 nb_poisson_report* rep) {
  const size_t N = ncell(g);
  double* diag = malloc(N * 8);
  uint8_t* fluid = calloc(N, 1);
  double* rhs = malloc(N * 8);
  double* r = malloc(N * 8);
  double* z = malloc(N * 8);
  double* p = malloc(N * 8);
  double* Ap = malloc(N * 8);
  size_t nFluid = 0;
  for (size_t c = 0; c < N; ++c) {
    x[c] = 0.0;
    diag[c] = 1.0;
  }
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const size_t c = cidx(g, i, j, k);
        if (is_solid(g, i, j, k)) continue;
        fluid[c] = 1;
        ++nFluid;
        const double d = diag_of(g, i, j, k);
        diag[c] = (d > 0.0) ? d : 1.0;
      }
  memcpy(rhs, b, N * 8);
  const int singular = !has_dirichlet(g);
  if (singular && nFluid > 0) {
    double mean = 0.0;
    for (size_t c = 0; c < N; ++c)
      if (fluid[c]) mean += rhs[c];
    mean /= (double)nFluid;
    for (size_t c = 0; c < N; ++c) {
      if (fluid[c]) rhs[c] -= mean;
      else rhs[c] = 0.0;
    }
  }
  memcpy(r, rhs, N * 8);
  for (size_t m = 0; m < N; ++m) z[m] = r[m] / diag[m];
  memcpy(p, z, N * 8);
  double rz = dot(r, z, N);
  const double bnorm = sqrt(dot(rhs, rhs, N)) + 1e-300;
  int converged = 0, it = 0;
  for (; it < maxit; ++it) {
    orc_apply_a(g, p, Ap);
    const double pAp = dot(p, Ap, N);
    if (fabs(pAp) < 1e-300) break;
    const double alpha = rz / pAp;
    for (size_t m = 0; m < N; ++m) {
      x[m] += alpha * p[m];
      r[m] -= alpha * Ap[m];
    }
    const double rnorm = sqrt(dot(r, r, N));
    if (rnorm <= tol * bnorm) {
      ++it;
      converged = 1;
      break;
    }
    for (size_t m = 0; m < N; ++m) z[m] = r[m] / diag[m];
    const double rzNew = dot(r, z, N);
    const double beta = rzNew / rz;
    for (size_t m = 0; m < N; ++m) p[m] = z[m] + beta * p[m];
    rz = rzNew;
  }
  if (singular && nFluid > 0) {
    double mean = 0.0;
    for (size_t c = 0; c < N; ++c)
      if (fluid[c]) mean += x[c];
    mean /= (double)nFluid;
    for (size_t c = 0; c < N; ++c)
      if (fluid[c]) x[c] -= mean;
  }
  orc_apply_a(g, x, Ap);
  double rr = 0.0;
  for (size_t m = 0; m < N; ++m) {
    const double e = rhs[m] - Ap[m];
    rr += e * e;
  }
  rep->iterations = it;
  rep->residual = sqrt(rr) / bnorm;
  rep->converged = (converged || rep->residual <= 1e-6) ? 1 : 0;
  free(diag);
  free(fluid);
  free(rhs);
  free(r);
  free(z);
  free(p);
  free(Ap);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Geometric multigrid: core/src/flow/multigrid.cpp:22-355                   */
/* ------------------------------------------------------------------------ */
#define ORC_OMEGA 0.8         /* multigrid.cpp:38 */
#define ORC_MAX_LEVELS 8      /* multigrid.cpp:39 */
#define ORC_COARSEST_MAX 2048 /* multigrid.cpp:40 */
#define ORC_MIN_COARSEN 4     /* multigrid.cpp:41 */

typedef struct {
  nb_grid_desc g;
  uint8_t* solid;
  double* diag;
  uint8_t* fluid;
  size_t nFluid;
  int fx, fy, fz;
} mg_level;

typedef struct {
  mg_level lv[ORC_MAX_LEVELS];
  int nlev;
  int singular;
} mg_hier;

static void fill_level_meta(mg_level* L) { /* multigrid.cpp:63-79 */
  const size_t n = ncell(&L->g);
  L->diag = malloc(n * 8);
  orc_build_diagonal(&L->g, L->diag);
  L->fluid = calloc(n, 1);
  L->nFluid = 0;
  for (int k = 0; k < L->g.nz; ++k)
    for (int j = 0; j < L->g.ny; ++j)
      for (int i = 0; i < L->g.nx; ++i)
        if (!is_solid(&L->g, i, j, k)) {
          L->fluid[cidx(&L->g, i, j, k)] = 1;
          ++L->nFluid;
        }
}

static void build_hier(const nb_grid_desc* grid, mg_hier* H) { /* multigrid.cpp:211-266 */
  memset(H, 0, sizeof(*H));
  H->singular = !has_dirichlet(grid);
  mg_level* F = &H->lv[0];
  F->g = *grid;
  F->solid = calloc(ncell(grid), 1);
  if (grid->solid) memcpy(F->solid, grid->solid, ncell(grid));
  F->g.solid = F->solid;
  F->fx = F->fy = F->fz = 1;
  fill_level_meta(F);
  H->nlev = 1;
  while (H->nlev < ORC_MAX_LEVELS) {
    const nb_grid_desc* f = &H->lv[H->nlev - 1].g;
    const int fx = (f->nx >= ORC_MIN_COARSEN) ? 2 : 1;
    const int fy = (f->ny >= ORC_MIN_COARSEN) ? 2 : 1;
    const int fz = (f->nz >= ORC_MIN_COARSEN) ? 2 : 1;
    if (fx == 1 && fy == 1 && fz == 1) break;
    mg_level* C = &H->lv[H->nlev];
    C->fx = fx;
    C->fy = fy;
    C->fz = fz;
    C->g = *f;
    C->g.nx = (f->nx + fx - 1) / fx;
    C->g.ny = (f->ny + fy - 1) / fy;
    C->g.nz = (f->nz + fz - 1) / fz;
    C->g.dx = f->dx * (double)f->nx / (double)C->g.nx;
    C->g.dy = f->dy * (double)f->ny / (double)C->g.ny;
    C->g.dz = f->dz * (double)f->nz / (double)C->g.nz;
    const size_t nc = ncell(&C->g);
    C->solid = malloc(nc);
    uint8_t* saw = calloc(nc, 1);
    const mg_level* FL = &H->lv[H->nlev - 1];
    for (int k = 0; k < f->nz; ++k)
      for (int j = 0; j < f->ny; ++j)
        for (int i = 0; i < f->nx; ++i)
          if (FL->fluid[cidx(f, i, j, k)]) saw[cidx(&C->g, i / fx, j / fy, k / fz)] = 1;
    for (size_t cc = 0; cc < nc; ++cc) C->solid[cc] = saw[cc] ? 0 : 1;
    free(saw);
    C->g.solid = C->solid;
    fill_level_meta(C);
    H->nlev++;
    if (nc <= ORC_COARSEST_MAX) break;
  }
}

static void free_hier(mg_hier* H) {
  for (int l = 0; l < H->nlev; ++l) {
    free(H->lv[l].solid);
    free(H->lv[l].diag);
    free(H->lv[l].fluid);
  }
}

static void remove_mean(const mg_level* L, double* x) { /* multigrid.cpp:81-99 */
  if (L->nFluid == 0) return;
  const size_t n = ncell(&L->g);
  double mean = 0.0;
  for (size_t c = 0; c < n; ++c) {
    if (L->fluid[c]) mean += x[c];
    else x[c] = 0.0;
  }
  mean /= (double)L->nFluid;
  for (size_t c = 0; c < n; ++c)
    if (L->fluid[c]) x[c] -= mean;
}

static void smooth(const mg_level* L, const double* b, double* x, int sweeps, int singular) {
  /* multigrid.cpp:102-114 */
  const size_t n = ncell(&L->g);
  double* Ax = malloc(n * 8);
  for (int s = 0; s < sweeps; ++s) {
    orc_apply_a(&L->g, x, Ax);
    for (size_t c = 0; c < n; ++c)
      x[c] = L->fluid[c] ? x[c] + ORC_OMEGA * (b[c] - Ax[c]) / L->diag[c] : 0.0;
    if (singular) remove_mean(L, x);
  }
  free(Ax);
}

static void vcycle(mg_hier* H, int lvl, const double* b, double* x, int pre, int post) {
  /* multigrid.cpp:175-194 */
  const mg_level* L = &H->lv[lvl];
  if (lvl + 1 >= H->nlev) {
    nb_poisson_report rep;
    orc_cg_solve(&L->g, b, x, 1e-6, 500, &rep);
    return;
  }
  smooth(L, b, x, pre, H->singular);
  const size_t n = ncell(&L->g);
  const mg_level* C = &H->lv[lvl + 1];
  const size_t nc = ncell(&C->g);
  double* r = malloc(n * 8);
  orc_apply_a(&L->g, x, r); /* residual, multigrid.cpp:116-122 */
  for (size_t c = 0; c < n; ++c) r[c] = L->fluid[c] ? b[c] - r[c] : 0.0;
  double* rc = calloc(nc, 8); /* restrictResidual, multigrid.cpp:127-154 */
  int* count = calloc(nc, sizeof(int));
  for (int k = 0; k < L->g.nz; ++k)
    for (int j = 0; j < L->g.ny; ++j)
      for (int i = 0; i < L->g.nx; ++i) {
        const size_t f = cidx(&L->g, i, j, k);
        if (!L->fluid[f]) continue;
        const size_t Cc = cidx(&C->g, i / C->fx, j / C->fy, k / C->fz);
        rc[Cc] += r[f];
        ++count[Cc];
      }
  for (size_t Cc = 0; Cc < nc; ++Cc)
    if (count[Cc] > 0) rc[Cc] /= (double)count[Cc];
  if (H->singular) remove_mean(C, rc);
  double* ec = calloc(nc, 8);
  vcycle(H, lvl + 1, rc, ec, pre, post);
  for (int k = 0; k < L->g.nz; ++k) /* prolongAdd, multigrid.cpp:158-173 */
    for (int j = 0; j < L->g.ny; ++j)
      for (int i = 0; i < L->g.nx; ++i) {
        const size_t f = cidx(&L->g, i, j, k);
        if (!L->fluid[f]) continue;
        x[f] += ec[cidx(&C->g, i / C->fx, j / C->fy, k / C->fz)];
      }
  smooth(L, b, x, post, H->singular);
  free(r);
  free(rc);
  free(count);
  free(ec);
}

/* MG-PCG (flexible, Polak-Ribiere): core/src/flow/multigrid.cpp:206-355 */
int orc_mg_solve(const nb_grid_desc* grid, const double* b, double* x, double tol, int maxit,
                 nb_poisson_report* rep) {
  mg_hier H;
  build_hier(grid, &H);
  const int pre = 2, post = 2;
  const size_t N = ncell(grid);
  const mg_level* L0 = &H.lv[0];
  double* rhs = malloc(N * 8);
  double* r = malloc(N * 8);
  double* z = malloc(N * 8);
  double* p = malloc(N * 8);
  double* Ap = malloc(N * 8);
  double* rnew = malloc(N * 8);
  double* znew = malloc(N * 8);
  for (size_t c = 0; c < N; ++c) x[c] = 0.0;
  memcpy(rhs, b, N * 8);
  for (size_t c = 0; c < N; ++c)
    if (!L0->fluid[c]) rhs[c] = 0.0;
  if (H.singular) remove_mean(L0, rhs);
  const double bnorm = sqrt(dot(rhs, rhs, N)) + 1e-300;
  memcpy(r, rhs, N * 8);
  int it = 0, converged = 0;
  if (sqrt(dot(r, r, N)) <= tol * bnorm) {
    rep->iterations = 0;
    rep->residual = sqrt(dot(r, r, N)) / bnorm;
    rep->converged = 1;
    goto done;
  }
  memset(z, 0, N * 8);
  vcycle(&H, 0, r, z, pre, post);
  if (H.singular) remove_mean(L0, z);
  memcpy(p, z, N * 8);
  double rz = dot(r, z, N);
  for (; it < maxit; ++it) {
    orc_apply_a(grid, p, Ap);
    const double pAp = dot(p, Ap, N);
    if (fabs(pAp) < 1e-300) break;
    const double alpha = rz / pAp;
    for (size_t c = 0; c < N; ++c) {
      x[c] += alpha * p[c];
      rnew[c] = r[c] - alpha * Ap[c];
    }
    if (H.singular) remove_mean(L0, rnew);
    if (sqrt(dot(rnew, rnew, N)) <= tol * bnorm) {
      ++it;
      memcpy(r, rnew, N * 8);
      converged = 1;
      break;
    }
    memset(znew, 0, N * 8);
    vcycle(&H, 0, rnew, znew, pre, post);
    if (H.singular) remove_mean(L0, znew);
    double rnewz = 0.0, rz_cross = 0.0;
    for (size_t c = 0; c < N; ++c) {
      rnewz += znew[c] * rnew[c];
      rz_cross += znew[c] * r[c];
    }
    const double beta = (rnewz - rz_cross) / rz;
    for (size_t c = 0; c < N; ++c) p[c] = znew[c] + beta * p[c];
    rz = rnewz;
    memcpy(r, rnew, N * 8);
  }
  if (H.singular) remove_mean(L0, x);
  orc_apply_a(grid, x, Ap);
  {
    double rr = 0.0;
    for (size_t c = 0; c < N; ++c) {
      const double e = rhs[c] - Ap[c];
      rr += e * e;
    }
    rep->iterations = it;
    rep->residual = sqrt(rr) / bnorm;
    rep->converged = (converged || rep->residual <= tol) ? 1 : 0;
  }
done:
  free(rhs);
  free(r);
  free(z);
  free(p);
  free(Ap);
  free(rnew);
  free(znew);
  free_hier(&H);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* NS step: core/src/flow/ns_solver.cpp                                     */
/* ------------------------------------------------------------------------ */
struct orc_ns {
  nb_grid_desc g;
  uint8_t* solid;
  nb_flow_config cfg;
  double nu;
  double *u, *v, *w, *p;
  size_t nu_, nv_, nw_, np_;
  int hasSolid;
  int step;
  double t, dtLast;
};

static size_t UI(const orc_ns* s, int i, int j, int k) { /* ns_solver.hpp:94-99 */
  return (size_t)i + (size_t)(s->g.nx + 1) * ((size_t)j + (size_t)s->g.ny * (size_t)k);
}
static size_t VI(const orc_ns* s, int i, int j, int k) { /* ns_solver.hpp:100-105 */
  return (size_t)i + (size_t)s->g.nx * ((size_t)j + (size_t)(s->g.ny + 1) * (size_t)k);
}
static size_t WI(const orc_ns* s, int i, int j, int k) { /* ns_solver.hpp:106-111 */
  return (size_t)i + (size_t)s->g.nx * ((size_t)j + (size_t)s->g.ny * (size_t)k);
}
static size_t CI(const orc_ns* s, int i, int j, int k) { return cidx(&s->g, i, j, k); }
static int wrap(int a, int n) { return (a % n + n) % n; }
static int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }

orc_ns* orc_ns_create(const nb_grid_desc* g, const nb_flow_config* cfg) { /* ns_solver.cpp:46-69 */
  orc_ns* s = calloc(1, sizeof(orc_ns));
  s->g = *g;
  s->solid = calloc(ncell(g), 1);
  if (g->solid) memcpy(s->solid, g->solid, ncell(g));
  s->g.solid = s->solid;
  s->cfg = *cfg;
  s->nu = cfg->velocity_scale * cfg->ref_length / cfg->reynolds;
  s->nu_ = (size_t)(g->nx + 1) * g->ny * g->nz;
  s->nv_ = (size_t)g->nx * (g->ny + 1) * g->nz;
  s->nw_ = (size_t)g->nx * g->ny * (g->nz + 1);
  s->np_ = ncell(g);
  s->u = calloc(s->nu_, 8);
  s->v = calloc(s->nv_, 8);
  s->w = calloc(s->nw_, 8);
  s->p = calloc(s->np_, 8);
  for (size_t c = 0; c < s->np_; ++c)
    if (s->solid[c]) {
      s->hasSolid = 1;
      break;
    }
  return s;
}

void orc_ns_destroy(orc_ns* s) {
  if (!s) return;
  free(s->solid);
  free(s->u);
  free(s->v);
  free(s->w);
  free(s->p);
  free(s);
}

static void inlet_velocity_at(const orc_ns* s, int face, int j, int k, double vel[3]) {
  /* ns_solver.cpp:71-93 */
  const nb_face_bc* fb = &s->g.face[face];
  double mag = fb->inlet_speed;
  (void)k;
  if (fb->profile == NB_PROFILE_PARABOLIC) {
    const double H = s->g.ny * s->g.dy;
    const double yc = s->g.origin[1] + 0.5 * H;
    const double y = s->g.origin[1] + (j + 0.5) * s->g.dy;
    const double r = (y - yc) / (0.5 * H);
    mag = 1.5 * fb->inlet_speed * (1.0 - r * r);
  }
  vel[0] = vel[1] = vel[2] = 0.0;
  if (fb->inlet_axis == 0) vel[0] = mag;
  else if (fb->inlet_axis == 1) vel[1] = mag;
  else vel[2] = mag;
}

/* BC-aware staggered accessors: ns_solver.cpp:116-219 */
static double U_(const orc_ns* s, const double* u, int i, int j, int k) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  if (k < 0 || k >= nz) {
    if (periodic(&s->g, 2)) return U_(s, u, i, j, wrap(k, nz));
    const int km = (k < 0) ? (-1 - k) : (2 * nz - 1 - k);
    const int face = (k < 0) ? 4 : 5;
    return 2.0 * s->g.face[face].wall_velocity[0] - U_(s, u, i, j, km);
  }
  if (j < 0 || j >= ny) {
    if (periodic(&s->g, 1)) return U_(s, u, i, wrap(j, ny), k);
    const int jm = (j < 0) ? (-1 - j) : (2 * ny - 1 - j);
    const int face = (j < 0) ? 2 : 3;
    return 2.0 * s->g.face[face].wall_velocity[0] - U_(s, u, i, jm, k);
  }
  if (i < 0 || i > nx) {
    if (periodic(&s->g, 0)) return U_(s, u, wrap(i, nx), j, k);
    const int ib = (i < 0) ? 0 : nx;
    const int ir = 2 * ib - i;
    const int face = (i < 0) ? 0 : 1;
    if (s->g.face[face].type == NB_BC_OUTLET) return u[UI(s, clampi(ib, 0, nx), j, k)];
    return 2.0 * u[UI(s, ib, j, k)] - U_(s, u, ir, j, k);
  }
  return u[UI(s, i, j, k)];
}

static double V_(const orc_ns* s, const double* v, int i, int j, int k) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  if (k < 0 || k >= nz) {
    if (periodic(&s->g, 2)) return V_(s, v, i, j, wrap(k, nz));
    const int km = (k < 0) ? (-1 - k) : (2 * nz - 1 - k);
    const int face = (k < 0) ? 4 : 5;
    return 2.0 * s->g.face[face].wall_velocity[1] - V_(s, v, i, j, km);
  }
  if (i < 0 || i >= nx) {
    if (periodic(&s->g, 0)) return V_(s, v, wrap(i, nx), j, k);
    const int im = (i < 0) ? (-1 - i) : (2 * nx - 1 - i);
    const int face = (i < 0) ? 0 : 1;
    if (s->g.face[face].type == NB_BC_INLET) {
      double vel[3];
      inlet_velocity_at(s, face, j, k, vel);
      return 2.0 * vel[1] - V_(s, v, im, j, k);
    }
    if (s->g.face[face].type == NB_BC_OUTLET) return v[VI(s, clampi(i, 0, nx - 1), j, k)];
    return 2.0 * s->g.face[face].wall_velocity[1] - V_(s, v, im, j, k);
  }
  if (j < 0 || j > ny) {
    if (periodic(&s->g, 1)) return V_(s, v, i, wrap(j, ny), k);
    const int jb = (j < 0) ? 0 : ny;
    const int jr = 2 * jb - j;
    const int face = (j < 0) ? 2 : 3;
    if (s->g.face[face].type == NB_BC_OUTLET) return v[VI(s, i, clampi(jb, 0, ny), k)];
    return 2.0 * v[VI(s, i, jb, k)] - V_(s, v, i, jr, k);
  }
  return v[VI(s, i, j, k)];
}

static double W_(const orc_ns* s, const double* w, int i, int j, int k) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  if (j < 0 || j >= ny) {
    if (periodic(&s->g, 1)) return W_(s, w, i, wrap(j, ny), k);
    const int jm = (j < 0) ? (-1 - j) : (2 * ny - 1 - j);
    const int face = (j < 0) ? 2 : 3;
    return 2.0 * s->g.face[face].wall_velocity[2] - W_(s, w, i, jm, k);
  }
  if (i < 0 || i >= nx) {
    if (periodic(&s->g, 0)) return W_(s, w, wrap(i, nx), j, k);
    const int im = (i < 0) ? (-1 - i) : (2 * nx - 1 - i);
    const int face = (i < 0) ? 0 : 1;
    if (s->g.face[face].type == NB_BC_OUTLET) return w[WI(s, clampi(i, 0, nx - 1), j, k)];
    return 2.0 * s->g.face[face].wall_velocity[2] - W_(s, w, im, j, k);
  }
  if (k < 0 || k > nz) {
    if (periodic(&s->g, 2)) return W_(s, w, i, j, wrap(k, nz));
    const int kb = (k < 0) ? 0 : nz;
    const int kr = 2 * kb - k;
    return 2.0 * w[WI(s, i, j, kb)] - W_(s, w, i, j, kr);
  }
  return w[WI(s, i, j, k)];
}

/* Jiang-Shu WENO-5: ns_solver.cpp:15-31 */
static double weno5(double v0, double v1, double v2, double v3, double v4) {
  const double eps = 1e-12;
  const double b0 = 13.0 / 12.0 * (v0 - 2 * v1 + v2) * (v0 - 2 * v1 + v2) +
                    0.25 * (v0 - 4 * v1 + 3 * v2) * (v0 - 4 * v1 + 3 * v2);
  const double b1 = 13.0 / 12.0 * (v1 - 2 * v2 + v3) * (v1 - 2 * v2 + v3) +
                    0.25 * (v1 - v3) * (v1 - v3);
  const double b2 = 13.0 / 12.0 * (v2 - 2 * v3 + v4) * (v2 - 2 * v3 + v4) +
                    0.25 * (3 * v2 - 4 * v3 + v4) * (3 * v2 - 4 * v3 + v4);
  const double a0 = 0.1 / ((eps + b0) * (eps + b0));
  const double a1 = 0.6 / ((eps + b1) * (eps + b1));
  const double a2 = 0.3 / ((eps + b2) * (eps + b2));
  const double sum = a0 + a1 + a2;
  const double p0 = (2 * v0 - 7 * v1 + 11 * v2) / 6.0;
  const double p1 = (-v1 + 5 * v2 + 2 * v3) / 6.0;
  const double p2 = (2 * v2 + 5 * v3 - v4) / 6.0;
  return (a0 * p0 + a1 * p1 + a2 * p2) / sum;
}

/* ns_solver.cpp:35-42: q[0..5] = cells i-2..i+3 around the face between i and i+1 */
static double recon(int weno, double adv, double qm2, double qm1, double q0, double qp1,
                    double qp2, double qp3) {
  if (!weno) return 0.5 * (q0 + qp1);
  return (adv >= 0.0) ? weno5(qm2, qm1, q0, qp1, qp2) : weno5(qp3, qp2, qp1, q0, qm1);
}

/* ns_solver.cpp:221-309 */
static void apply_velocity_bc(const orc_ns* s, double* u, double* v, double* w, int outflow) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  double vel[3];
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int side = 0; side < 2; ++side) {
        const int face = side, i = side == 0 ? 0 : nx;
        switch (s->g.face[face].type) {
          case NB_BC_WALL: u[UI(s, i, j, k)] = 0.0; break;
          case NB_BC_INLET:
            inlet_velocity_at(s, face, j, k, vel);
            u[UI(s, i, j, k)] = vel[0];
            break;
          case NB_BC_OUTLET:
            if (outflow) u[UI(s, i, j, k)] = u[UI(s, side == 0 ? 1 : nx - 1, j, k)];
            break;
          default: break;
        }
      }
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i)
      for (int side = 0; side < 2; ++side) {
        const int face = 2 + side, j = side == 0 ? 0 : ny;
        switch (s->g.face[face].type) {
          case NB_BC_WALL: v[VI(s, i, j, k)] = 0.0; break;
          case NB_BC_INLET:
            inlet_velocity_at(s, face, i, k, vel);
            v[VI(s, i, j, k)] = vel[1];
            break;
          case NB_BC_OUTLET:
            if (outflow) v[VI(s, i, j, k)] = v[VI(s, i, side == 0 ? 1 : ny - 1, k)];
            break;
          default: break;
        }
      }
  if (nz > 1)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        for (int side = 0; side < 2; ++side) {
          const int face = 4 + side, k = side == 0 ? 0 : nz;
          switch (s->g.face[face].type) {
            case NB_BC_WALL: w[WI(s, i, j, k)] = 0.0; break;
            case NB_BC_INLET:
              inlet_velocity_at(s, face, i, j, vel);
              w[WI(s, i, j, k)] = vel[2];
              break;
            case NB_BC_OUTLET:
              if (outflow) w[WI(s, i, j, k)] = w[WI(s, i, j, side == 0 ? 1 : nz - 1)];
              break;
            default: break;
          }
        }
  if (s->hasSolid) {
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i)
          if (is_solid(&s->g, i - 1, j, k) || is_solid(&s->g, i, j, k)) u[UI(s, i, j, k)] = 0.0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i)
          if (is_solid(&s->g, i, j - 1, k) || is_solid(&s->g, i, j, k)) v[VI(s, i, j, k)] = 0.0;
    if (nz > 1)
      for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i)
            if (is_solid(&s->g, i, j, k - 1) || is_solid(&s->g, i, j, k)) w[WI(s, i, j, k)] = 0.0;
  }
}

/* ns_solver.cpp:311-473 */
static void compute_rhs(const orc_ns* s, const double* u, const double* v, const double* w,
                        double* ru, double* rv, double* rw) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  const double dx = s->g.dx, dy = s->g.dy, dz = s->g.dz;
  const int twoD = (nz == 1);
  const int sc = s->cfg.convection == NB_CONV_WENO5;
  const double nu = s->nu;
  memset(ru, 0, s->nu_ * 8);
  memset(rv, 0, s->nv_ * 8);
  memset(rw, 0, s->nw_ * 8);
#define Uq(a, b, c) U_(s, u, (a), (b), (c))
#define Vq(a, b, c) V_(s, v, (a), (b), (c))
#define Wq(a, b, c) W_(s, w, (a), (b), (c))
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 1; i < nx; ++i) {
        if (is_solid(&s->g, i - 1, j, k) || is_solid(&s->g, i, j, k)) continue;
        const double ucL = 0.5 * (Uq(i - 1, j, k) + Uq(i, j, k));
        const double ucR = 0.5 * (Uq(i, j, k) + Uq(i + 1, j, k));
        const double uxL = recon(sc, ucL, Uq(i - 3, j, k), Uq(i - 2, j, k), Uq(i - 1, j, k),
                                 Uq(i, j, k), Uq(i + 1, j, k), Uq(i + 2, j, k));
        const double uxR = recon(sc, ucR, Uq(i - 2, j, k), Uq(i - 1, j, k), Uq(i, j, k),
                                 Uq(i + 1, j, k), Uq(i + 2, j, k), Uq(i + 3, j, k));
        const double dFx = (ucR * uxR - ucL * uxL) / dx;
        const double vT = 0.5 * (Vq(i - 1, j + 1, k) + Vq(i, j + 1, k));
        const double vB = 0.5 * (Vq(i - 1, j, k) + Vq(i, j, k));
        const double uyT = recon(sc, vT, Uq(i, j - 2, k), Uq(i, j - 1, k), Uq(i, j, k),
                                 Uq(i, j + 1, k), Uq(i, j + 2, k), Uq(i, j + 3, k));
        const double uyB = recon(sc, vB, Uq(i, j - 3, k), Uq(i, j - 2, k), Uq(i, j - 1, k),
                                 Uq(i, j, k), Uq(i, j + 1, k), Uq(i, j + 2, k));
        const double dFy = (vT * uyT - vB * uyB) / dy;
        double dFz = 0.0;
        if (!twoD) {
          const double wT = 0.5 * (Wq(i - 1, j, k + 1) + Wq(i, j, k + 1));
          const double wB = 0.5 * (Wq(i - 1, j, k) + Wq(i, j, k));
          const double uzT = recon(sc, wT, Uq(i, j, k - 2), Uq(i, j, k - 1), Uq(i, j, k),
                                   Uq(i, j, k + 1), Uq(i, j, k + 2), Uq(i, j, k + 3));
          const double uzB = recon(sc, wB, Uq(i, j, k - 3), Uq(i, j, k - 2), Uq(i, j, k - 1),
                                   Uq(i, j, k), Uq(i, j, k + 1), Uq(i, j, k + 2));
          dFz = (wT * uzT - wB * uzB) / dz;
        }
        double lap = (Uq(i + 1, j, k) - 2 * Uq(i, j, k) + Uq(i - 1, j, k)) / (dx * dx) +
                     (Uq(i, j + 1, k) - 2 * Uq(i, j, k) + Uq(i, j - 1, k)) / (dy * dy);
        if (!twoD) lap += (Uq(i, j, k + 1) - 2 * Uq(i, j, k) + Uq(i, j, k - 1)) / (dz * dz);
        ru[UI(s, i, j, k)] = -(dFx + dFy + dFz) + nu * lap + s->cfg.body_force[0];
      }
  for (int k = 0; k < nz; ++k)
    for (int j = 1; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (is_solid(&s->g, i, j - 1, k) || is_solid(&s->g, i, j, k)) continue;
        const double vcB = 0.5 * (Vq(i, j - 1, k) + Vq(i, j, k));
        const double vcT = 0.5 * (Vq(i, j, k) + Vq(i, j + 1, k));
        const double vyB = recon(sc, vcB, Vq(i, j - 3, k), Vq(i, j - 2, k), Vq(i, j - 1, k),
                                 Vq(i, j, k), Vq(i, j + 1, k), Vq(i, j + 2, k));
        const double vyT = recon(sc, vcT, Vq(i, j - 2, k), Vq(i, j - 1, k), Vq(i, j, k),
                                 Vq(i, j + 1, k), Vq(i, j + 2, k), Vq(i, j + 3, k));
        const double dFy = (vcT * vyT - vcB * vyB) / dy;
        const double uR = 0.5 * (Uq(i + 1, j - 1, k) + Uq(i + 1, j, k));
        const double uL = 0.5 * (Uq(i, j - 1, k) + Uq(i, j, k));
        const double vxR = recon(sc, uR, Vq(i - 2, j, k), Vq(i - 1, j, k), Vq(i, j, k),
                                 Vq(i + 1, j, k), Vq(i + 2, j, k), Vq(i + 3, j, k));
        const double vxL = recon(sc, uL, Vq(i - 3, j, k), Vq(i - 2, j, k), Vq(i - 1, j, k),
                                 Vq(i, j, k), Vq(i + 1, j, k), Vq(i + 2, j, k));
        const double dFx = (uR * vxR - uL * vxL) / dx;
        double dFz = 0.0;
        if (!twoD) {
          const double wR = 0.5 * (Wq(i, j - 1, k + 1) + Wq(i, j, k + 1));
          const double wL = 0.5 * (Wq(i, j - 1, k) + Wq(i, j, k));
          const double vzR = recon(sc, wR, Vq(i, j, k - 2), Vq(i, j, k - 1), Vq(i, j, k),
                                   Vq(i, j, k + 1), Vq(i, j, k + 2), Vq(i, j, k + 3));
          const double vzL = recon(sc, wL, Vq(i, j, k - 3), Vq(i, j, k - 2), Vq(i, j, k - 1),
                                   Vq(i, j, k), Vq(i, j, k + 1), Vq(i, j, k + 2));
          dFz = (wR * vzR - wL * vzL) / dz;
        }
        double lap = (Vq(i + 1, j, k) - 2 * Vq(i, j, k) + Vq(i - 1, j, k)) / (dx * dx) +
                     (Vq(i, j + 1, k) - 2 * Vq(i, j, k) + Vq(i, j - 1, k)) / (dy * dy);
        if (!twoD) lap += (Vq(i, j, k + 1) - 2 * Vq(i, j, k) + Vq(i, j, k - 1)) / (dz * dz);
        rv[VI(s, i, j, k)] = -(dFx + dFy + dFz) + nu * lap + s->cfg.body_force[1];
      }
  if (!twoD)
    for (int k = 1; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (is_solid(&s->g, i, j, k - 1) || is_solid(&s->g, i, j, k)) continue;
          const double wcB = 0.5 * (Wq(i, j, k - 1) + Wq(i, j, k));
          const double wcT = 0.5 * (Wq(i, j, k) + Wq(i, j, k + 1));
          const double wzB = recon(sc, wcB, Wq(i, j, k - 3), Wq(i, j, k - 2), Wq(i, j, k - 1),
                                   Wq(i, j, k), Wq(i, j, k + 1), Wq(i, j, k + 2));
          const double wzT = recon(sc, wcT, Wq(i, j, k - 2), Wq(i, j, k - 1), Wq(i, j, k),
                                   Wq(i, j, k + 1), Wq(i, j, k + 2), Wq(i, j, k + 3));
          const double dFz = (wcT * wzT - wcB * wzB) / dz;
          const double uR = 0.5 * (Uq(i + 1, j, k - 1) + Uq(i + 1, j, k));
          const double uL = 0.5 * (Uq(i, j, k - 1) + Uq(i, j, k));
          const double wxR = recon(sc, uR, Wq(i - 2, j, k), Wq(i - 1, j, k), Wq(i, j, k),
                                   Wq(i + 1, j, k), Wq(i + 2, j, k), Wq(i + 3, j, k));
          const double wxL = recon(sc, uL, Wq(i - 3, j, k), Wq(i - 2, j, k), Wq(i - 1, j, k),
                                   Wq(i, j, k), Wq(i + 1, j, k), Wq(i + 2, j, k));
          const double dFx = (uR * wxR - uL * wxL) / dx;
          const double vR = 0.5 * (Vq(i, j + 1, k - 1) + Vq(i, j + 1, k));
          const double vL = 0.5 * (Vq(i, j, k - 1) + Vq(i, j, k));
          const double wyR = recon(sc, vR, Wq(i, j - 2, k), Wq(i, j - 1, k), Wq(i, j, k),
                                   Wq(i, j + 1, k), Wq(i, j + 2, k), Wq(i, j + 3, k));
          const double wyL = recon(sc, vL, Wq(i, j - 3, k), Wq(i, j - 2, k), Wq(i, j - 1, k),
                                   Wq(i, j, k), Wq(i, j + 1, k), Wq(i, j + 2, k));
          const double dFy = (vR * wyR - vL * wyL) / dy;
          const double lap =
              (Wq(i + 1, j, k) - 2 * Wq(i, j, k) + Wq(i - 1, j, k)) / (dx * dx) +
              (Wq(i, j + 1, k) - 2 * Wq(i, j, k) + Wq(i, j - 1, k)) / (dy * dy) +
              (Wq(i, j, k + 1) - 2 * Wq(i, j, k) + Wq(i, j, k - 1)) / (dz * dz);
          rw[WI(s, i, j, k)] = -(dFx + dFy + dFz) + nu * lap + s->cfg.body_force[2];
        }
#undef Uq
#undef Vq
#undef Wq
}

static double div_at(const orc_ns* s, const double* u, const double* v, const double* w, int i,
                     int j, int k) {
  double d = (u[UI(s, i + 1, j, k)] - u[UI(s, i, j, k)]) / s->g.dx +
             (v[VI(s, i, j + 1, k)] - v[VI(s, i, j, k)]) / s->g.dy;
  if (s->g.nz > 1) d += (w[WI(s, i, j, k + 1)] - w[WI(s, i, j, k)]) / s->g.dz;
  return d;
}

static double phi_at(const orc_ns* s, const double* phi, int i, int j, int k) {
  /* ns_solver.cpp:508-526 */
  int c[3] = {i, j, k};
  const int n[3] = {s->g.nx, s->g.ny, s->g.nz};
  double sgn = 1.0;
  for (int a = 0; a < 3; ++a) {
    double f = 1.0;
    if (!(c[a] >= 0 && c[a] < n[a])) {
      if (periodic(&s->g, a)) {
        c[a] = wrap(c[a], n[a]);
      } else {
        const int faceId = 2 * a + (c[a] < 0 ? 0 : 1);
        c[a] = clampi(c[a], 0, n[a] - 1);
        f = s->g.face[faceId].type == NB_BC_OUTLET ? -1.0 : 1.0;
      }
    }
    sgn *= f;
  }
  return sgn * phi[CI(s, c[0], c[1], c[2])];
}

/* ns_solver.cpp:475-579 */
static void project(orc_ns* s, double* u, double* v, double* w, double dt, int* iters,
                    double* res, int* conv) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  apply_velocity_bc(s, u, v, w, 1);
  double* b = calloc(s->np_, 8);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (is_solid(&s->g, i, j, k)) continue;
        b[CI(s, i, j, k)] = -div_at(s, u, v, w, i, j, k);
      }
  double* phi = malloc(s->np_ * 8);
  nb_poisson_report rep;
  orc_mg_solve(&s->g, b, phi, s->cfg.poisson_tol, s->cfg.poisson_max_iters, &rep);
  *iters = rep.iterations;
  *res = rep.residual;
  *conv = rep.converged;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        if (is_solid(&s->g, i - 1, j, k) || is_solid(&s->g, i, j, k)) continue;
        u[UI(s, i, j, k)] -= (phi_at(s, phi, i, j, k) - phi_at(s, phi, i - 1, j, k)) / s->g.dx;
      }
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (is_solid(&s->g, i, j - 1, k) || is_solid(&s->g, i, j, k)) continue;
        v[VI(s, i, j, k)] -= (phi_at(s, phi, i, j, k) - phi_at(s, phi, i, j - 1, k)) / s->g.dy;
      }
  if (nz > 1)
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (is_solid(&s->g, i, j, k - 1) || is_solid(&s->g, i, j, k)) continue;
          w[WI(s, i, j, k)] -= (phi_at(s, phi, i, j, k) - phi_at(s, phi, i, j, k - 1)) / s->g.dz;
        }
  apply_velocity_bc(s, u, v, w, 0);
  for (size_t c = 0; c < s->np_; ++c) s->p[c] = phi[c] / dt;
  free(b);
  free(phi);
}

double orc_ns_compute_dt(const orc_ns* s) { /* ns_solver.cpp:581-603 */
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  const int twoD = (nz == 1);
  const double visc =
      2.0 * s->nu *
      (1.0 / (s->g.dx * s->g.dx) + 1.0 / (s->g.dy * s->g.dy) + (twoD ? 0.0 : 1.0 / (s->g.dz * s->g.dz)));
  double maxInv = visc + 1e-300;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (is_solid(&s->g, i, j, k)) continue;
        const double uc = fabs(0.5 * (s->u[UI(s, i, j, k)] + s->u[UI(s, i + 1, j, k)]));
        const double vc = fabs(0.5 * (s->v[VI(s, i, j, k)] + s->v[VI(s, i, j + 1, k)]));
        const double wc = twoD ? 0.0 : fabs(0.5 * (s->w[WI(s, i, j, k)] + s->w[WI(s, i, j, k + 1)]));
        const double inv = uc / s->g.dx + vc / s->g.dy + (twoD ? 0.0 : wc / s->g.dz) + visc;
        if (inv > maxInv) maxInv = inv;
      }
  return s->cfg.cfl / maxInv;
}

void orc_ns_initialize(orc_ns* s) { /* ns_solver.cpp:95-112 */
  memset(s->u, 0, s->nu_ * 8);
  memset(s->v, 0, s->nv_ * 8);
  memset(s->w, 0, s->nw_ * 8);
  memset(s->p, 0, s->np_ * 8);
  for (int f = 0; f < 6; ++f)
    if (s->g.face[f].type == NB_BC_INLET && s->g.face[f].inlet_axis == 0) {
      for (size_t m = 0; m < s->nu_; ++m) s->u[m] = s->g.face[f].inlet_speed;
      break;
    }
  apply_velocity_bc(s, s->u, s->v, s->w, 1);
  s->step = 0;
  s->t = 0.0;
  s->dtLast = 0.0;
}

void orc_ns_set_state(orc_ns* s, const double* u, const double* v, const double* w,
                      const double* p, int step, double t, double dt_last) {
  memcpy(s->u, u, s->nu_ * 8);
  memcpy(s->v, v, s->nv_ * 8);
  memcpy(s->w, w, s->nw_ * 8);
  memcpy(s->p, p, s->np_ * 8);
  s->step = step;
  s->t = t;
  s->dtLast = dt_last;
}

void orc_ns_get_state(const orc_ns* s, double* u, double* v, double* w, double* p) {
  if (u) memcpy(u, s->u, s->nu_ * 8);
  if (v) memcpy(v, s->v, s->nv_ * 8);
  if (w) memcpy(w, s->w, s->nw_ * 8);
  if (p) memcpy(p, s->p, s->np_ * 8);
}

/* ns_solver.cpp:767-824 */
void orc_ns_step(orc_ns* s, double dt, nb_step_report* rep) {
  const int nx = s->g.nx, ny = s->g.ny, nz = s->g.nz;
  if (dt <= 0.0) dt = orc_ns_compute_dt(s);
  double* u0 = malloc(s->nu_ * 8);
  double* v0 = malloc(s->nv_ * 8);
  double* w0 = malloc(s->nw_ * 8);
  double* ru = malloc(s->nu_ * 8);
  double* rv = malloc(s->nv_ * 8);
  double* rw = malloc(s->nw_ * 8);
  memcpy(u0, s->u, s->nu_ * 8);
  memcpy(v0, s->v, s->nv_ * 8);
  memcpy(w0, s->w, s->nw_ * 8);
  int it[3] = {0, 0, 0}, cv[3] = {1, 1, 1};
  double pr[3] = {0, 0, 0};
  apply_velocity_bc(s, s->u, s->v, s->w, 1);
  compute_rhs(s, s->u, s->v, s->w, ru, rv, rw);
  for (size_t m = 0; m < s->nu_; ++m) s->u[m] = u0[m] + dt * ru[m];
  for (size_t m = 0; m < s->nv_; ++m) s->v[m] = v0[m] + dt * rv[m];
  for (size_t m = 0; m < s->nw_; ++m) s->w[m] = w0[m] + dt * rw[m];
  project(s, s->u, s->v, s->w, dt, &it[0], &pr[0], &cv[0]);
  compute_rhs(s, s->u, s->v, s->w, ru, rv, rw);
  for (size_t m = 0; m < s->nu_; ++m) s->u[m] = 0.75 * u0[m] + 0.25 * (s->u[m] + dt * ru[m]);
  for (size_t m = 0; m < s->nv_; ++m) s->v[m] = 0.75 * v0[m] + 0.25 * (s->v[m] + dt * rv[m]);
  for (size_t m = 0; m < s->nw_; ++m) s->w[m] = 0.75 * w0[m] + 0.25 * (s->w[m] + dt * rw[m]);
  project(s, s->u, s->v, s->w, dt, &it[1], &pr[1], &cv[1]);
  compute_rhs(s, s->u, s->v, s->w, ru, rv, rw);
  const double c1 = 1.0 / 3.0, c2 = 2.0 / 3.0;
  for (size_t m = 0; m < s->nu_; ++m) s->u[m] = c1 * u0[m] + c2 * (s->u[m] + dt * ru[m]);
  for (size_t m = 0; m < s->nv_; ++m) s->v[m] = c1 * v0[m] + c2 * (s->v[m] + dt * rv[m]);
  for (size_t m = 0; m < s->nw_; ++m) s->w[m] = c1 * w0[m] + c2 * (s->w[m] + dt * rw[m]);
  project(s, s->u, s->v, s->w, dt, &it[2], &pr[2], &cv[2]);

  double du = 0.0;
  size_t n = 0;
  for (size_t m = 0; m < s->nu_; ++m) { du += (s->u[m] - u0[m]) * (s->u[m] - u0[m]); ++n; }
  for (size_t m = 0; m < s->nv_; ++m) { du += (s->v[m] - v0[m]) * (s->v[m] - v0[m]); ++n; }
  for (size_t m = 0; m < s->nw_; ++m) { du += (s->w[m] - w0[m]) * (s->w[m] - w0[m]); ++n; }
  const double momRes = sqrt(du / (double)(n ? n : 1)) / (dt * s->cfg.velocity_scale + 1e-300);

  s->step += 1;
  s->t += dt;
  s->dtLast = dt;
  memset(rep, 0, sizeof(*rep));
  rep->step = s->step;
  rep->t = s->t;
  rep->dt = dt;
  rep->cfl = s->cfg.cfl;
  rep->momentum_residual = momRes;
  /* divergenceL2 / divergenceMax: ns_solver.cpp:605-649 */
  double s2 = 0.0, mx = 0.0;
  size_t nd = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (is_solid(&s->g, i, j, k)) continue;
        const double d = div_at(s, s->u, s->v, s->w, i, j, k);
        s2 += d * d;
        ++nd;
        if (fabs(d) > mx) mx = fabs(d);
      }
  rep->continuity_residual = nd ? sqrt(s2 / (double)nd) : 0.0;
  rep->divergence_max = mx;
  /* massFluxError: ns_solver.cpp:651-675 */
  {
    const double ax = s->g.dy * s->g.dz, ay = s->g.dx * s->g.dz, az = s->g.dx * s->g.dy;
    double net = 0.0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) net += (s->u[UI(s, 0, j, k)] - s->u[UI(s, nx, j, k)]) * ax;
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nx; ++i) net += (s->v[VI(s, i, 0, k)] - s->v[VI(s, i, ny, k)]) * ay;
    if (nz > 1)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) net += (s->w[WI(s, i, j, 0)] - s->w[WI(s, i, j, nz)]) * az;
    const double scale = s->cfg.velocity_scale * (ny * ay) + 1e-300;
    rep->mass_error = fabs(net) / scale;
  }
  rep->poisson_iters = it[0] + it[1] + it[2];
  rep->poisson_residual = fmax(pr[0], fmax(pr[1], pr[2]));
  rep->converged = cv[0] && cv[1] && cv[2];
  /* computeForces: ns_solver.cpp:703-763 */
  rep->cd = 0.0;
  rep->cl = 0.0;
  if (s->hasSolid) {
    const double areaX = s->g.dy * s->g.dz, areaY = s->g.dx * s->g.dz, areaZ = s->g.dx * s->g.dy;
    const double mu = s->nu * s->cfg.density;
    double fx = 0.0, fy = 0.0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const int nb[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k},
                                {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
          const double nox[6] = {1.0, -1.0, 0.0, 0.0, 0.0, 0.0};
          const double noy[6] = {0.0, 0.0, 1.0, -1.0, 0.0, 0.0};
          const double area[6] = {areaX, areaX, areaY, areaY, areaZ, areaZ};
          const double dn[6] = {s->g.dx, s->g.dx, s->g.dy, s->g.dy, s->g.dz, s->g.dz};
          const int nd6 = nz > 1 ? 6 : 4;
          for (int d = 0; d < nd6; ++d) {
            const int axis = d / 2;
            if (!is_solid(&s->g, nb[d][0], nb[d][1], nb[d][2]) || is_solid(&s->g, i, j, k)) continue;
            const double pf = s->p[CI(s, i, j, k)];
            fx += -pf * nox[d] * area[d];
            fy += -pf * noy[d] * area[d];
            const double uc = 0.5 * (s->u[UI(s, i, j, k)] + s->u[UI(s, i + 1, j, k)]);
            const double vc = 0.5 * (s->v[VI(s, i, j, k)] + s->v[VI(s, i, j + 1, k)]);
            if (axis != 0) fx += mu * uc / (0.5 * dn[d]) * area[d];
            if (axis != 1) fy += mu * vc / (0.5 * dn[d]) * area[d];
          }
        }
    double aref = s->cfg.ref_area;
    if (aref <= 0.0) aref = s->cfg.ref_length * s->cfg.ref_length;
    const double q = 0.5 * s->cfg.density * s->cfg.velocity_scale * s->cfg.velocity_scale * aref + 1e-300;
    rep->cd = fx / q;
    rep->cl = fy / q;
  }
  rep->cell_count = s->np_;
  rep->accepted = (rep->continuity_residual < s->cfg.tol_continuity &&
                   rep->mass_error < s->cfg.tol_mass) ? 1 : 0;
  free(u0);
  free(v0);
  free(w0);
  free(ru);
  free(rv);
  free(rw);
}
