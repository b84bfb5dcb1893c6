/* restate_amr.c — TEST INFRASTRUCTURE ONLY: the oracle's CPU restatement of the
 * MAC step on an octree mesh of 8^3-cell leaf bricks (FP64, plain C).
 *
 * The reference has no octree MAC step; this restates the rules the library
 * implements, written independently of it and on a different data layout
 * (dense arrays per octree level instead of bricks):
 *   - the uniform step of core/src/flow/ns_solver.cpp evaluated at each
 *     leaf's own level: ghost accessors U/Vv/W (:116-219) with the reference's
 *     recursion, WENO-5 (:15-42), computeRhs (:311-473) with R = 0 on domain
 *     faces and faces touching a solid, SSP-RK3 (:773-795), applyVelocityBC
 *     (:221-309) on every level's boundary faces, project (:475-579);
 *   - at a 2:1 interface the four fine sub-faces are the state and the coarse
 *     face is their average (recomputed after every update); a face read at
 *     level L inside a coarser leaf is the coarse face (even index) or the
 *     mean of the coarse cell's two faces (odd index), over finer leaves the
 *     mean of the four sub-faces;
 *   - the pressure operator is the conservative octree rule of
 *     core/src/flow/octree_poisson.cpp:24-32 per unit volume (same level
 *     1/h^2, fine to coarse 1/(1.5 h^2), coarse to each of 4 fine 1/(3 H^2)),
 *     with the uniform operator's Dirichlet outlet and periodic closures
 *     (core/src/flow/poisson.cpp:18-52), solved by volume-weighted Jacobi-CG
 *     to a tight tolerance; the correction uses the same centre distances.
 * A level-L cell covered by a finer leaf reports the first child's solid flag.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc.h"

#define ML 8

struct orc_amr {
  nb_amr_geom g;
  nb_flow_config cfg;
  double nu;
  int per[3];
  int nl;                 /* levels present 0..nl-1 */
  int n[ML][3];           /* cells per axis */
  double h[ML][3];
  int fine[3];            /* cells per axis at level nl-1 */
  int* leaf;              /* finest cell -> level of its leaf */
  uint8_t* solid[ML];     /* dense per level (leaf cells of that level) */
  double* f[3][ML];       /* faces, dims n + e_a */
  double* f0[3][ML];      /* RK stage start */
  double* p[ML];          /* cells */
  double* phi[ML];
  double divmax;
  int cg_iters;
  /* Leaf cells in (L, k, j, i) order and the operator's rows, built once on
   * the first solve (the mesh never changes): the CG loops walk this list
   * instead of scanning the dense per-level arrays. Same cells, same order,
   * same arithmetic, so the results are those of the dense scan bit for bit. */
  size_t nlc;
  int* lc_L;
  size_t* lc_ci;
  double* lc_vol;     /* h0 * h1 * h2 of the cell's level */
  size_t* op_off;     /* [nlc + 1] row offsets; a solid row has no entries */
  int* op_L;
  size_t* op_ci;
  double* op_coef;
  double* op_diag;    /* diagonal in face order; 1 for solid rows */
};

/* ------------------------------------------------------------------ maps -- */
static size_t cidx(const orc_amr* A, int L, int i, int j, int k) {
  return (size_t)i + (size_t)A->n[L][0] * ((size_t)j + (size_t)A->n[L][1] * (size_t)k);
}
static size_t fidx(const orc_amr* A, int a, int L, int i, int j, int k) {
  const size_t ex = A->n[L][0] + (a == 0), ey = A->n[L][1] + (a == 1);
  return (size_t)i + ex * ((size_t)j + ey * (size_t)k);
}
static size_t fsize(const orc_amr* A, int a, int L) {
  return (size_t)(A->n[L][0] + (a == 0)) * (A->n[L][1] + (a == 1)) * (A->n[L][2] + (a == 2));
}
static int wrapi(int x, int n) { return ((x % n) + n) % n; }

/* Wraps periodic axes; 0 if the cell is outside the domain. */
static int in_domain(const orc_amr* A, int L, int c[3]) {
  for (int a = 0; a < 3; ++a)
    if (c[a] < 0 || c[a] >= A->n[L][a]) {
      if (!A->per[a]) return 0;
      c[a] = wrapi(c[a], A->n[L][a]);
    }
  return 1;
}

/* Level of the leaf covering in-domain level-L cell c. */
static int leaf_level(const orc_amr* A, int L, const int c[3]) {
  const int s = A->nl - 1 - L;
  if (s >= 0) {
    const size_t q = (size_t)(c[0] << s) + (size_t)A->fine[0] * ((size_t)(c[1] << s) + (size_t)A->fine[1] * (size_t)(c[2] << s));
    return A->leaf[q];
  }
  return -1;
}

static int cell_solid(const orc_amr* A, int L, const int c0[3]) {
  int c[3] = {c0[0], c0[1], c0[2]};
  if (!in_domain(A, L, c)) return 0;
  const int lev = leaf_level(A, L, c);
  int q[3];
  for (int a = 0; a < 3; ++a) q[a] = lev <= L ? c[a] >> (L - lev) : c[a] << (lev - L);
  return A->solid[lev][cidx(A, lev, q[0], q[1], q[2])] != 0;
}

/* Is the level-L a-face at p stored at level L (an adjacent cell is a leaf cell of level L)? */
static int stored(const orc_amr* A, int a, int L, const int p[3], int* lev_minus, int* lev_plus) {
  int m[3] = {p[0], p[1], p[2]}, q[3] = {p[0], p[1], p[2]};
  m[a] -= 1;
  *lev_minus = in_domain(A, L, m) ? leaf_level(A, L, m) : -1;
  *lev_plus = in_domain(A, L, q) ? leaf_level(A, L, q) : -1;
  return *lev_minus == L || *lev_plus == L;
}

/* Storage position of a stored level-L face (periodic high faces are the low ones). */
static double* fslot(orc_amr* A, int a, int L, const int p0[3]) {
  int p[3] = {p0[0], p0[1], p0[2]};
  if (A->per[a] && p[a] == A->n[L][a]) p[a] = 0;
  return &A->f[a][L][fidx(A, a, L, p[0], p[1], p[2])];
}

/* a-face value at level L, position p (p[a] in [0, N], others in range). */
static double face_get(orc_amr* A, int a, int L, const int p0[3]) {
  int p[3] = {p0[0], p0[1], p0[2]};
  if (A->per[a] && p[a] == A->n[L][a]) p[a] = 0;
  int lm, lp;
  if (stored(A, a, L, p, &lm, &lp)) return *fslot(A, a, L, p);
  const int lev = lp >= 0 ? lp : lm;
  const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
  if (lev > L) { /* finer on both sides: mean of the four sub-faces */
    double s = 0.0;
    for (int d2 = 0; d2 < 2; ++d2)
      for (int d1 = 0; d1 < 2; ++d1) {
        int c[3];
        c[a] = 2 * p[a];
        c[t1] = 2 * p[t1] + d1;
        c[t2] = 2 * p[t2] + d2;
        s += face_get(A, a, L + 1, c);
      }
    return 0.25 * s;
  }
  /* inside a coarser leaf */
  int c[3] = {p[0] >> 1, p[1] >> 1, p[2] >> 1};
  if ((p[a] & 1) == 0) {
    c[a] = p[a] / 2;
    return face_get(A, a, L - 1, c);
  }
  const double lo = face_get(A, a, L - 1, c);
  c[a] += 1;
  const double hi = face_get(A, a, L - 1, c);
  return 0.5 * (lo + hi);
}

/* ------------------------------------------------------- ghost accessors -- */
static double inlet_at(const orc_amr* A, int face, int L, int j, int comp) {
  const nb_face_bc* fb = &A->g.face[face];
  double mag = fb->inlet_speed;
  if (fb->profile == NB_PROFILE_PARABOLIC) {
    const double dy = A->h[L][1];
    const double H = A->n[L][1] * dy;
    const double yc = A->g.origin[1] + 0.5 * H;
    const double y = A->g.origin[1] + (j + 0.5) * dy;
    const double r = (y - yc) / (0.5 * H);
    mag = 1.5 * fb->inlet_speed * (1.0 - r * r);
  }
  return fb->inlet_axis == comp ? mag : 0.0;
}

static double U_(orc_amr* A, int L, int i, int j, int k) {
  const int nx = A->n[L][0], ny = A->n[L][1], nz = A->n[L][2];
  if (k < 0 || k >= nz) {
    if (A->per[2]) return U_(A, L, i, j, wrapi(k, nz));
    const int face = k < 0 ? 4 : 5;
    return 2.0 * A->g.face[face].wall_velocity[0] - U_(A, L, i, j, k < 0 ? -1 - k : 2 * nz - 1 - k);
  }
  if (j < 0 || j >= ny) {
    if (A->per[1]) return U_(A, L, i, wrapi(j, ny), k);
    const int face = j < 0 ? 2 : 3;
    return 2.0 * A->g.face[face].wall_velocity[0] - U_(A, L, i, j < 0 ? -1 - j : 2 * ny - 1 - j, k);
  }
  if (i < 0 || i > nx) {
    if (A->per[0]) return U_(A, L, wrapi(i, nx), j, k);
    const int ib = i < 0 ? 0 : nx, face = i < 0 ? 0 : 1;
    const int pb[3] = {ib, j, k};
    if (A->g.face[face].type == NB_BC_OUTLET) return face_get(A, 0, L, pb);
    return 2.0 * face_get(A, 0, L, pb) - U_(A, L, 2 * ib - i, j, k);
  }
  const int pp[3] = {i, j, k};
  return face_get(A, 0, L, pp);
}

static double V_(orc_amr* A, int L, int i, int j, int k) {
  const int nx = A->n[L][0], ny = A->n[L][1], nz = A->n[L][2];
  if (k < 0 || k >= nz) {
    if (A->per[2]) return V_(A, L, i, j, wrapi(k, nz));
    const int face = k < 0 ? 4 : 5;
    return 2.0 * A->g.face[face].wall_velocity[1] - V_(A, L, i, j, k < 0 ? -1 - k : 2 * nz - 1 - k);
  }
  if (i < 0 || i >= nx) {
    if (A->per[0]) return V_(A, L, wrapi(i, nx), j, k);
    const int im = i < 0 ? -1 - i : 2 * nx - 1 - i, face = i < 0 ? 0 : 1;
    if (A->g.face[face].type == NB_BC_INLET) return 2.0 * inlet_at(A, face, L, j, 1) - V_(A, L, im, j, k);
    if (A->g.face[face].type == NB_BC_OUTLET) {
      const int pb[3] = {i < 0 ? 0 : nx - 1, j < 0 ? 0 : (j > ny ? ny : j), k};
      return face_get(A, 1, L, pb);
    }
    return 2.0 * A->g.face[face].wall_velocity[1] - V_(A, L, im, j, k);
  }
  if (j < 0 || j > ny) {
    if (A->per[1]) return V_(A, L, i, wrapi(j, ny), k);
    const int jb = j < 0 ? 0 : ny, face = j < 0 ? 2 : 3;
    const int pb[3] = {i, jb, k};
    if (A->g.face[face].type == NB_BC_OUTLET) return face_get(A, 1, L, pb);
    return 2.0 * face_get(A, 1, L, pb) - V_(A, L, i, 2 * jb - j, k);
  }
  const int pp[3] = {i, j, k};
  return face_get(A, 1, L, pp);
}

static double W_(orc_amr* A, int L, int i, int j, int k) {
  const int nx = A->n[L][0], ny = A->n[L][1], nz = A->n[L][2];
  if (j < 0 || j >= ny) {
    if (A->per[1]) return W_(A, L, i, wrapi(j, ny), k);
    const int face = j < 0 ? 2 : 3;
    return 2.0 * A->g.face[face].wall_velocity[2] - W_(A, L, i, j < 0 ? -1 - j : 2 * ny - 1 - j, k);
  }
  if (i < 0 || i >= nx) {
    if (A->per[0]) return W_(A, L, wrapi(i, nx), j, k);
    const int im = i < 0 ? -1 - i : 2 * nx - 1 - i, face = i < 0 ? 0 : 1;
    if (A->g.face[face].type == NB_BC_OUTLET) {
      const int pb[3] = {i < 0 ? 0 : nx - 1, j, k < 0 ? 0 : (k > nz ? nz : k)};
      return face_get(A, 2, L, pb);
    }
    return 2.0 * A->g.face[face].wall_velocity[2] - W_(A, L, im, j, k);
  }
  if (k < 0 || k > nz) {
    if (A->per[2]) return W_(A, L, i, j, wrapi(k, nz));
    const int kb = k < 0 ? 0 : nz;
    const int pb[3] = {i, j, kb};
    return 2.0 * face_get(A, 2, L, pb) - W_(A, L, i, j, 2 * kb - k);
  }
  const int pp[3] = {i, j, k};
  return face_get(A, 2, L, pp);
}

static double weno5(double v0, double v1, double v2, double v3, double v4) {
  const double eps = 1e-12;
  const double b0 = 13.0 / 12.0 * (v0 - 2 * v1 + v2) * (v0 - 2 * v1 + v2) +
                    0.25 * (v0 - 4 * v1 + 3 * v2) * (v0 - 4 * v1 + 3 * v2);
  const double b1 = 13.0 / 12.0 * (v1 - 2 * v2 + v3) * (v1 - 2 * v2 + v3) + 0.25 * (v1 - v3) * (v1 - v3);
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
static double recon(int weno, double adv, double qm2, double qm1, double q0, double qp1, double qp2, double qp3) {
  if (!weno) return 0.5 * (q0 + qp1);
  return adv >= 0.0 ? weno5(qm2, qm1, q0, qp1, qp2) : weno5(qp3, qp2, qp1, q0, qm1);
}

/* computeRhs at one a-face of level L (i, j, k): ns_solver.cpp:322-472. */
static double rhs_at(orc_amr* A, int a, int L, int i, int j, int k) {
  const double dx = A->h[L][0], dy = A->h[L][1], dz = A->h[L][2];
  const int sc = A->cfg.convection == NB_CONV_WENO5;
  const double nu = A->nu;
#define Uq(x, y, z) U_(A, L, (x), (y), (z))
#define Vq(x, y, z) V_(A, L, (x), (y), (z))
#define Wq(x, y, z) W_(A, L, (x), (y), (z))
  if (a == 0) {
    const double ucL = 0.5 * (Uq(i - 1, j, k) + Uq(i, j, k));
    const double ucR = 0.5 * (Uq(i, j, k) + Uq(i + 1, j, k));
    const double uxL = recon(sc, ucL, Uq(i - 3, j, k), Uq(i - 2, j, k), Uq(i - 1, j, k), Uq(i, j, k), Uq(i + 1, j, k), Uq(i + 2, j, k));
    const double uxR = recon(sc, ucR, Uq(i - 2, j, k), Uq(i - 1, j, k), Uq(i, j, k), Uq(i + 1, j, k), Uq(i + 2, j, k), Uq(i + 3, j, k));
    const double dFx = (ucR * uxR - ucL * uxL) / dx;
    const double vT = 0.5 * (Vq(i - 1, j + 1, k) + Vq(i, j + 1, k));
    const double vB = 0.5 * (Vq(i - 1, j, k) + Vq(i, j, k));
    const double uyT = recon(sc, vT, Uq(i, j - 2, k), Uq(i, j - 1, k), Uq(i, j, k), Uq(i, j + 1, k), Uq(i, j + 2, k), Uq(i, j + 3, k));
    const double uyB = recon(sc, vB, Uq(i, j - 3, k), Uq(i, j - 2, k), Uq(i, j - 1, k), Uq(i, j, k), Uq(i, j + 1, k), Uq(i, j + 2, k));
    const double dFy = (vT * uyT - vB * uyB) / dy;
    const double wT = 0.5 * (Wq(i - 1, j, k + 1) + Wq(i, j, k + 1));
    const double wB = 0.5 * (Wq(i - 1, j, k) + Wq(i, j, k));
    const double uzT = recon(sc, wT, Uq(i, j, k - 2), Uq(i, j, k - 1), Uq(i, j, k), Uq(i, j, k + 1), Uq(i, j, k + 2), Uq(i, j, k + 3));
    const double uzB = recon(sc, wB, Uq(i, j, k - 3), Uq(i, j, k - 2), Uq(i, j, k - 1), Uq(i, j, k), Uq(i, j, k + 1), Uq(i, j, k + 2));
    const double dFz = (wT * uzT - wB * uzB) / dz;
    double lap = (Uq(i + 1, j, k) - 2 * Uq(i, j, k) + Uq(i - 1, j, k)) / (dx * dx) +
                 (Uq(i, j + 1, k) - 2 * Uq(i, j, k) + Uq(i, j - 1, k)) / (dy * dy);
    lap += (Uq(i, j, k + 1) - 2 * Uq(i, j, k) + Uq(i, j, k - 1)) / (dz * dz);
    return -(dFx + dFy + dFz) + nu * lap + A->cfg.body_force[0];
  }
  if (a == 1) {
    const double vcB = 0.5 * (Vq(i, j - 1, k) + Vq(i, j, k));
    const double vcT = 0.5 * (Vq(i, j, k) + Vq(i, j + 1, k));
    const double vyB = recon(sc, vcB, Vq(i, j - 3, k), Vq(i, j - 2, k), Vq(i, j - 1, k), Vq(i, j, k), Vq(i, j + 1, k), Vq(i, j + 2, k));
    const double vyT = recon(sc, vcT, Vq(i, j - 2, k), Vq(i, j - 1, k), Vq(i, j, k), Vq(i, j + 1, k), Vq(i, j + 2, k), Vq(i, j + 3, k));
    const double dFy = (vcT * vyT - vcB * vyB) / dy;
    const double uR = 0.5 * (Uq(i + 1, j - 1, k) + Uq(i + 1, j, k));
    const double uL = 0.5 * (Uq(i, j - 1, k) + Uq(i, j, k));
    const double vxR = recon(sc, uR, Vq(i - 2, j, k), Vq(i - 1, j, k), Vq(i, j, k), Vq(i + 1, j, k), Vq(i + 2, j, k), Vq(i + 3, j, k));
    const double vxL = recon(sc, uL, Vq(i - 3, j, k), Vq(i - 2, j, k), Vq(i - 1, j, k), Vq(i, j, k), Vq(i + 1, j, k), Vq(i + 2, j, k));
    const double dFx = (uR * vxR - uL * vxL) / dx;
    const double wR = 0.5 * (Wq(i, j - 1, k + 1) + Wq(i, j, k + 1));
    const double wL = 0.5 * (Wq(i, j - 1, k) + Wq(i, j, k));
    const double vzR = recon(sc, wR, Vq(i, j, k - 2), Vq(i, j, k - 1), Vq(i, j, k), Vq(i, j, k + 1), Vq(i, j, k + 2), Vq(i, j, k + 3));
    const double vzL = recon(sc, wL, Vq(i, j, k - 3), Vq(i, j, k - 2), Vq(i, j, k - 1), Vq(i, j, k), Vq(i, j, k + 1), Vq(i, j, k + 2));
    const double dFz = (wR * vzR - wL * vzL) / dz;
    double lap = (Vq(i + 1, j, k) - 2 * Vq(i, j, k) + Vq(i - 1, j, k)) / (dx * dx) +
                 (Vq(i, j + 1, k) - 2 * Vq(i, j, k) + Vq(i, j - 1, k)) / (dy * dy);
    lap += (Vq(i, j, k + 1) - 2 * Vq(i, j, k) + Vq(i, j, k - 1)) / (dz * dz);
    return -(dFx + dFy + dFz) + nu * lap + A->cfg.body_force[1];
  }
  const double wcB = 0.5 * (Wq(i, j, k - 1) + Wq(i, j, k));
  const double wcT = 0.5 * (Wq(i, j, k) + Wq(i, j, k + 1));
  const double wzB = recon(sc, wcB, Wq(i, j, k - 3), Wq(i, j, k - 2), Wq(i, j, k - 1), Wq(i, j, k), Wq(i, j, k + 1), Wq(i, j, k + 2));
  const double wzT = recon(sc, wcT, Wq(i, j, k - 2), Wq(i, j, k - 1), Wq(i, j, k), Wq(i, j, k + 1), Wq(i, j, k + 2), Wq(i, j, k + 3));
  const double dFz = (wcT * wzT - wcB * wzB) / dz;
  const double uR = 0.5 * (Uq(i + 1, j, k - 1) + Uq(i + 1, j, k));
  const double uL = 0.5 * (Uq(i, j, k - 1) + Uq(i, j, k));
  const double wxR = recon(sc, uR, Wq(i - 2, j, k), Wq(i - 1, j, k), Wq(i, j, k), Wq(i + 1, j, k), Wq(i + 2, j, k), Wq(i + 3, j, k));
  const double wxL = recon(sc, uL, Wq(i - 3, j, k), Wq(i - 2, j, k), Wq(i - 1, j, k), Wq(i, j, k), Wq(i + 1, j, k), Wq(i + 2, j, k));
  const double dFx = (uR * wxR - uL * wxL) / dx;
  const double vR = 0.5 * (Vq(i, j + 1, k - 1) + Vq(i, j + 1, k));
  const double vL = 0.5 * (Vq(i, j, k - 1) + Vq(i, j, k));
  const double wyR = recon(sc, vR, Wq(i, j - 2, k), Wq(i, j - 1, k), Wq(i, j, k), Wq(i, j + 1, k), Wq(i, j + 2, k), Wq(i, j + 3, k));
  const double wyL = recon(sc, vL, Wq(i, j - 3, k), Wq(i, j - 2, k), Wq(i, j - 1, k), Wq(i, j, k), Wq(i, j + 1, k), Wq(i, j + 2, k));
  const double dFy = (vR * wyR - vL * wyL) / dy;
  const double lap = (Wq(i + 1, j, k) - 2 * Wq(i, j, k) + Wq(i - 1, j, k)) / (dx * dx) +
                     (Wq(i, j + 1, k) - 2 * Wq(i, j, k) + Wq(i, j - 1, k)) / (dy * dy) +
                     (Wq(i, j, k + 1) - 2 * Wq(i, j, k) + Wq(i, j, k - 1)) / (dz * dz);
  return -(dFx + dFy + dFz) + nu * lap + A->cfg.body_force[2];
#undef Uq
#undef Vq
#undef Wq
}

/* ------------------------------------------------------ face enumeration -- */
/* Calls fn(a, L, p, kind) for every stored face: kind 1 owned, 2 derived
 * (one side a leaf cell of level L, the other finer). Periodic high faces are
 * visited once, at index 0. */
typedef void (*face_fn)(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx);
static void for_faces(orc_amr* A, face_fn fn, void* ctx) {
  for (int L = 0; L < A->nl; ++L)
    for (int a = 0; a < 3; ++a) {
      const int ex = A->n[L][0] + (a == 0), ey = A->n[L][1] + (a == 1), ez = A->n[L][2] + (a == 2);
      for (int k = 0; k < ez; ++k)
        for (int j = 0; j < ey; ++j)
          for (int i = 0; i < ex; ++i) {
            const int p[3] = {i, j, k};
            if (A->per[a] && p[a] == A->n[L][a]) continue;
            int lm, lp;
            if (!stored(A, a, L, p, &lm, &lp)) continue;
            const int kind = (lm > L || lp > L) ? 2 : 1;
            fn(A, a, L, p, kind, ctx);
          }
    }
}

static void sync_fn(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx) {
  (void)ctx;
  if (kind != 2) return;
  const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
  double s = 0.0;
  for (int d2 = 0; d2 < 2; ++d2)
    for (int d1 = 0; d1 < 2; ++d1) {
      int c[3];
      c[a] = 2 * p[a];
      c[t1] = 2 * p[t1] + d1;
      c[t2] = 2 * p[t2] + d2;
      s += *fslot(A, a, L + 1, c);
    }
  *fslot(A, a, L, p) = 0.25 * s;
}
static void sync_derived(orc_amr* A) { for_faces(A, sync_fn, NULL); }

/* applyVelocityBC on boundary faces of every level, then solids (owned faces). */
static void bc_fn(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx) {
  const int outflow = *(const int*)ctx;
  if (kind != 1 || A->per[a]) return;
  const int N = A->n[L][a];
  if (p[a] != 0 && p[a] != N) return;
  const int side = p[a] == N, face = 2 * a + side;
  const int bt = A->g.face[face].type;
  double* d = fslot(A, a, L, p);
  if (bt == NB_BC_WALL) *d = 0.0;
  else if (bt == NB_BC_INLET) *d = inlet_at(A, face, L, a == 0 ? p[1] : p[0], a);
  else if (bt == NB_BC_OUTLET && outflow) {
    int q[3] = {p[0], p[1], p[2]};
    q[a] = side ? N - 1 : 1;
    *d = *fslot(A, a, L, q);
  }
}
static void solid_fn(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx) {
  (void)ctx;
  if (kind != 1) return;
  int m[3] = {p[0], p[1], p[2]};
  m[a] -= 1;
  if (cell_solid(A, L, m) || cell_solid(A, L, p)) *fslot(A, a, L, p) = 0.0;
}
static void apply_bc(orc_amr* A, int outflow) {
  for_faces(A, bc_fn, &outflow);
  for_faces(A, solid_fn, NULL);
  sync_derived(A);
}

/* --------------------------------------------------------------- RK stage -- */
typedef struct {
  double dt;
  int stage;
  double** rhs;  /* [3*ML] scratch per stored face */
} stage_ctx;
static void rhs_fn(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx) {
  stage_ctx* S = (stage_ctx*)ctx;
  if (kind != 1) return;
  double r = 0.0;
  const int N = A->n[L][a];
  int m[3] = {p[0], p[1], p[2]};
  m[a] -= 1;
  if (p[a] != 0 && p[a] != N && !cell_solid(A, L, m) && !cell_solid(A, L, p)) r = rhs_at(A, a, L, p[0], p[1], p[2]);
  S->rhs[a * ML + L][fidx(A, a, L, p[0], p[1], p[2])] = r;
}
static void comb_fn(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx) {
  stage_ctx* S = (stage_ctx*)ctx;
  if (kind != 1) return;
  const size_t q = fidx(A, a, L, p[0], p[1], p[2]);
  const double r = S->rhs[a * ML + L][q], a0 = A->f0[a][L][q], cur = A->f[a][L][q], dt = S->dt;
  double v;
  if (S->stage == 1) v = a0 + dt * r;
  else if (S->stage == 2) v = 0.75 * a0 + 0.25 * (cur + dt * r);
  else v = (1.0 / 3.0) * a0 + (2.0 / 3.0) * (cur + dt * r);
  A->f[a][L][q] = v;
}

/* -------------------------------------------------------------- pressure -- */
typedef struct {
  int L, c[3];
} cell_ref;

/* Visits the leaf cells of every level in (L, k, j, i) order. */
#define FOR_LEAF_CELLS(A, L, i, j, k)                                           \
  for (int L = 0; L < (A)->nl; ++L)                                             \
    for (int k = 0; k < (A)->n[L][2]; ++k)                                      \
      for (int j = 0; j < (A)->n[L][1]; ++j)                                    \
        for (int i = 0; i < (A)->n[L][0]; ++i)                                  \
          if (leaf_level((A), L, (const int[3]){i, j, k}) == L)

/* The leaf-cell list and the rows of the per-unit-volume composite operator
 * (out = A x on leaf cells): faces in order -x, +x, -y, +y, -z, +z; a same-level
 * neighbour 1/h^2, a coarser one 1/(1.5 h^2), each of four finer ones
 * 1/(3 h^2); a solid neighbour is skipped; an outlet face adds 2/h^2 to the
 * diagonal; solid rows are identity. */
static void build_rows(orc_amr* A) {
  if (A->lc_L) return;
  size_t n = 0;
  FOR_LEAF_CELLS(A, L, i, j, k) { ++n; }
  A->nlc = n;
  A->lc_L = malloc(n * sizeof(int));
  A->lc_ci = malloc(n * sizeof(size_t));
  A->lc_vol = malloc(n * sizeof(double));
  A->op_off = malloc((n + 1) * sizeof(size_t));
  A->op_diag = malloc(n * sizeof(double));
  size_t cap = 8 * n + 16, ne = 0;
  A->op_L = malloc(cap * sizeof(int));
  A->op_ci = malloc(cap * sizeof(size_t));
  A->op_coef = malloc(cap * sizeof(double));
  size_t q = 0;
#define PUSH(LL, CC, CO)                                              \
  do {                                                                \
    if (ne == cap) {                                                  \
      cap *= 2;                                                       \
      A->op_L = realloc(A->op_L, cap * sizeof(int));                  \
      A->op_ci = realloc(A->op_ci, cap * sizeof(size_t));             \
      A->op_coef = realloc(A->op_coef, cap * sizeof(double));         \
    }                                                                 \
    A->op_L[ne] = (LL);                                               \
    A->op_ci[ne] = (CC);                                              \
    A->op_coef[ne] = (CO);                                            \
    ++ne;                                                             \
  } while (0)
  FOR_LEAF_CELLS(A, L, i, j, k) {
    const size_t ci = cidx(A, L, i, j, k);
    const int c[3] = {i, j, k};
    A->lc_L[q] = L;
    A->lc_ci[q] = ci;
    A->lc_vol[q] = A->h[L][0] * A->h[L][1] * A->h[L][2];
    A->op_off[q] = ne;
    if (A->solid[L][ci]) {
      A->op_diag[q++] = 1.0;
      continue;
    }
    double diag = 0.0;
    for (int f = 0; f < 6; ++f) {
      const int a = f >> 1, s = (f & 1) ? 1 : -1;
      const double ih2 = 1.0 / (A->h[L][a] * A->h[L][a]);
      int qq[3] = {c[0], c[1], c[2]};
      qq[a] += s;
      if (!in_domain(A, L, qq)) {
        if (A->g.face[2 * a + (s > 0)].type == NB_BC_OUTLET) diag += 2.0 * ih2;
        continue;
      }
      const int lev = leaf_level(A, L, qq);
      if (lev == L) {
        if (A->solid[L][cidx(A, L, qq[0], qq[1], qq[2])]) continue;
        diag += ih2;
        PUSH(L, cidx(A, L, qq[0], qq[1], qq[2]), ih2);
      } else if (lev == L - 1) {
        const size_t cc = cidx(A, L - 1, qq[0] >> 1, qq[1] >> 1, qq[2] >> 1);
        if (A->solid[L - 1][cc]) continue;
        const double coef = ih2 / 1.5;
        diag += coef;
        PUSH(L - 1, cc, coef);
      } else {
        const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
        for (int d2 = 0; d2 < 2; ++d2)
          for (int d1 = 0; d1 < 2; ++d1) {
            int fq[3];
            fq[a] = s > 0 ? 2 * qq[a] : 2 * qq[a] + 1;
            fq[t1] = 2 * c[t1] + d1;
            fq[t2] = 2 * c[t2] + d2;
            const size_t fc = cidx(A, L + 1, fq[0], fq[1], fq[2]);
            if (A->solid[L + 1][fc]) continue;
            const double coef = ih2 / 3.0;
            diag += coef;
            PUSH(L + 1, fc, coef);
          }
      }
    }
    A->op_diag[q++] = diag;
  }
#undef PUSH
  A->op_off[n] = ne;
}

/* out = A x from the recorded rows. */
static void apply_rows(orc_amr* A, double* const* x, double* const* out) {
  /* rows are independent: threads change nothing in any row's arithmetic */
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < A->nlc; ++q) {
    const int L = A->lc_L[q];
    const size_t ci = A->lc_ci[q];
    if (A->solid[L][ci]) {
      out[L][ci] = x[L][ci];
      continue;
    }
    double off = 0.0;
    for (size_t e = A->op_off[q]; e < A->op_off[q + 1]; ++e) off += A->op_coef[e] * x[A->op_L[e]][A->op_ci[e]];
    out[L][ci] = A->op_diag[q] * x[L][ci] - off;
  }
}

static double vdot(orc_amr* A, double* const* x, double* const* y) {
  double s = 0.0;
  for (size_t q = 0; q < A->nlc; ++q) {
    const int L = A->lc_L[q];
    const size_t ci = A->lc_ci[q];
    s += A->lc_vol[q] * x[L][ci] * y[L][ci];
  }
  return s;
}

static int has_outlet(const orc_amr* A) {
  for (int f = 0; f < 6; ++f)
    if (A->g.face[f].type == NB_BC_OUTLET) return 1;
  return 0;
}

static void remove_fluid_mean(orc_amr* A, double* const* x) {
  double s = 0.0, v = 0.0;
  for (size_t q = 0; q < A->nlc; ++q) {
    const int L = A->lc_L[q];
    const size_t ci = A->lc_ci[q];
    if (A->solid[L][ci]) continue;
    const double vol = A->lc_vol[q];
    s += vol * x[L][ci];
    v += vol;
  }
  const double m = v > 0.0 ? s / v : 0.0;
  for (size_t q = 0; q < A->nlc; ++q) {
    const int L = A->lc_L[q];
    const size_t ci = A->lc_ci[q];
    if (!A->solid[L][ci]) x[L][ci] -= m;
  }
}

/* Volume-weighted Jacobi-CG on the composite operator; b is overwritten. */
static int solve_pressure(orc_amr* A, double* const* b, double* const* x, double tol) {
  build_rows(A);
  double *r[ML], *z[ML], *pp[ML], *Ap[ML];
  for (int L = 0; L < A->nl; ++L) {
    const size_t n = (size_t)A->n[L][0] * A->n[L][1] * A->n[L][2];
    r[L] = calloc(n, 8);
    z[L] = calloc(n, 8);
    pp[L] = calloc(n, 8);
    Ap[L] = calloc(n, 8);
    memset(x[L], 0, n * 8);
  }
  const int sing = !has_outlet(A);
  if (sing) remove_fluid_mean(A, b);
  /* Jacobi diagonal: diag > 0 ? diag : 1 (1 on solid rows) */
  double* dg = malloc(A->nlc * sizeof(double));
  for (size_t q = 0; q < A->nlc; ++q) dg[q] = A->op_diag[q] > 0.0 ? A->op_diag[q] : 1.0;
  for (size_t q = 0; q < A->nlc; ++q) {
    const int L = A->lc_L[q];
    const size_t ci = A->lc_ci[q];
    r[L][ci] = A->solid[L][ci] ? 0.0 : b[L][ci];
    z[L][ci] = r[L][ci] / dg[q];
    pp[L][ci] = z[L][ci];
  }
  const double bnorm = sqrt(vdot(A, r, r)) + 1e-300;
  double rz = vdot(A, r, z);
  int it = 0;
  for (; it < 20000; ++it) {
    if (sqrt(vdot(A, r, r)) <= tol * bnorm) break;
    apply_rows(A, pp, Ap);
    const double pap = vdot(A, pp, Ap);
    if (fabs(pap) < 1e-300) break;
    const double alpha = rz / pap;
    for (size_t q = 0; q < A->nlc; ++q) {
      const int L = A->lc_L[q];
      const size_t ci = A->lc_ci[q];
      x[L][ci] += alpha * pp[L][ci];
      r[L][ci] -= alpha * Ap[L][ci];
    }
    if (sing) remove_fluid_mean(A, r);
    for (size_t q = 0; q < A->nlc; ++q) {
      const int L = A->lc_L[q];
      const size_t ci = A->lc_ci[q];
      z[L][ci] = r[L][ci] / dg[q];
    }
    const double rzn = vdot(A, r, z);
    const double beta = rzn / rz;
    rz = rzn;
    for (size_t q = 0; q < A->nlc; ++q) {
      const int L = A->lc_L[q];
      const size_t ci = A->lc_ci[q];
      pp[L][ci] = z[L][ci] + beta * pp[L][ci];
    }
  }
  if (sing) remove_fluid_mean(A, x);
  free(dg);
  for (int L = 0; L < A->nl; ++L) {
    free(r[L]);
    free(z[L]);
    free(pp[L]);
    free(Ap[L]);
  }
  return it;
}

/* phi and level of the cell on one side of a face; 0 outside the domain. */
static int side_phi(orc_amr* A, int L, const int c0[3], double* phi, int* lev, int* solid) {
  int c[3] = {c0[0], c0[1], c0[2]};
  if (!in_domain(A, L, c)) return 0;
  *lev = leaf_level(A, L, c);
  int q[3];
  for (int a = 0; a < 3; ++a) q[a] = *lev <= L ? c[a] >> (L - *lev) : c[a] << (*lev - L);
  const size_t ci = cidx(A, *lev, q[0], q[1], q[2]);
  *phi = A->phi[*lev][ci];
  *solid = A->solid[*lev][ci] != 0;
  return 1;
}

static void correct_fn(orc_amr* A, int a, int L, const int p[3], int kind, void* ctx) {
  (void)ctx;
  if (kind != 1) return;
  int m[3] = {p[0], p[1], p[2]};
  m[a] -= 1;
  double phm = 0, php = 0;
  int lm = -1, lp = -1, sm = 0, sp = 0;
  const int hm = side_phi(A, L, m, &phm, &lm, &sm);
  const int hp = side_phi(A, L, p, &php, &lp, &sp);
  if (sm || sp) return;
  const double h = A->h[L][a];
  if (!hm) { /* low domain face: ghost from the inside cell */
    const int bt = A->g.face[2 * a].type;
    phm = bt == NB_BC_OUTLET ? -php : php;
    lm = lp;
  }
  if (!hp) {
    const int bt = A->g.face[2 * a + 1].type;
    php = bt == NB_BC_OUTLET ? -phm : phm;
    lp = lm;
  }
  const double d = (lm == L && lp == L) ? h : 1.5 * h;
  *fslot(A, a, L, p) -= (php - phm) / d;
}

static double cell_div(orc_amr* A, int L, int i, int j, int k) {
  const int c[3] = {i, j, k};
  double d = 0.0;
  double parts[3];
  for (int a = 0; a < 3; ++a) {
    int q[3] = {c[0], c[1], c[2]};
    const double lo = face_get(A, a, L, q);
    q[a] += 1;
    const double hi = face_get(A, a, L, q);
    parts[a] = (hi - lo) / A->h[L][a];
  }
  d = parts[0] + parts[1];
  d += parts[2];
  return d;
}

static void project(orc_amr* A, double dt, double tol) {
  apply_bc(A, 1);
  double* b[ML];
  for (int L = 0; L < A->nl; ++L) b[L] = calloc((size_t)A->n[L][0] * A->n[L][1] * A->n[L][2], 8);
  FOR_LEAF_CELLS(A, L, i, j, k) {
    const size_t ci = cidx(A, L, i, j, k);
    b[L][ci] = A->solid[L][ci] ? 0.0 : -cell_div(A, L, i, j, k);
  }
  A->cg_iters += solve_pressure(A, b, A->phi, tol);
  for_faces(A, correct_fn, NULL);
  FOR_LEAF_CELLS(A, L, i, j, k) {
    const size_t ci = cidx(A, L, i, j, k);
    A->p[L][ci] = A->phi[L][ci] / dt;
  }
  sync_derived(A);
  apply_bc(A, 0);
  for (int L = 0; L < A->nl; ++L) free(b[L]);
}

/* -------------------------------------------------------------------- API -- */
orc_amr* orc_amr_create(const nb_amr_geom* g, const int32_t* leaves, int64_t n, const uint8_t* solid,
                        const nb_flow_config* cfg) {
  orc_amr* A = calloc(1, sizeof(orc_amr));
  A->g = *g;
  A->cfg = *cfg;
  A->nu = cfg->velocity_scale * cfg->ref_length / cfg->reynolds;
  for (int a = 0; a < 3; ++a) A->per[a] = g->face[2 * a].type == NB_BC_PERIODIC;
  int lmax = 0;
  for (int64_t q = 0; q < n; ++q)
    if (leaves[4 * q] > lmax) lmax = leaves[4 * q];
  A->nl = lmax + 1;
  for (int L = 0; L < A->nl; ++L)
    for (int a = 0; a < 3; ++a) {
      A->n[L][a] = (g->nb0[a] * 8) << L;
      A->h[L][a] = g->h0[a] / (double)(1 << L);
    }
  for (int a = 0; a < 3; ++a) A->fine[a] = A->n[lmax][a];
  A->leaf = malloc((size_t)A->fine[0] * A->fine[1] * A->fine[2] * sizeof(int));
  for (int L = 0; L < A->nl; ++L) {
    const size_t nc = (size_t)A->n[L][0] * A->n[L][1] * A->n[L][2];
    A->solid[L] = calloc(nc, 1);
    A->p[L] = calloc(nc, 8);
    A->phi[L] = calloc(nc, 8);
    for (int a = 0; a < 3; ++a) {
      A->f[a][L] = calloc(fsize(A, a, L), 8);
      A->f0[a][L] = calloc(fsize(A, a, L), 8);
    }
  }
  for (int64_t q = 0; q < n; ++q) {
    const int L = leaves[4 * q], s = lmax - L;
    const int b[3] = {leaves[4 * q + 1], leaves[4 * q + 2], leaves[4 * q + 3]};
    const int span = 8 << s;
    for (int k = 0; k < span; ++k)
      for (int j = 0; j < span; ++j)
        for (int i = 0; i < span; ++i) {
          const size_t fq = (size_t)(b[0] * span + i) +
                            (size_t)A->fine[0] * ((size_t)(b[1] * span + j) + (size_t)A->fine[1] * (size_t)(b[2] * span + k));
          A->leaf[fq] = L;
        }
    if (solid)
      for (int l = 0; l < 512; ++l) {
        const int i = b[0] * 8 + (l & 7), j = b[1] * 8 + ((l >> 3) & 7), k = b[2] * 8 + (l >> 6);
        A->solid[L][cidx(A, L, i, j, k)] = solid[q * 512 + l];
      }
  }
  return A;
}

void orc_amr_destroy(orc_amr* A) {
  if (!A) return;
  free(A->leaf);
  free(A->lc_L);
  free(A->lc_ci);
  free(A->lc_vol);
  free(A->op_off);
  free(A->op_L);
  free(A->op_ci);
  free(A->op_coef);
  free(A->op_diag);
  for (int L = 0; L < A->nl; ++L) {
    free(A->solid[L]);
    free(A->p[L]);
    free(A->phi[L]);
    for (int a = 0; a < 3; ++a) {
      free(A->f[a][L]);
      free(A->f0[a][L]);
    }
  }
  free(A);
}

/* comp 0..2: faces at (lev, i, j, k); comp 3: cells. */
void orc_amr_set(orc_amr* A, int comp, int64_t n, const int32_t* lev, const int32_t* i, const int32_t* j,
                 const int32_t* k, const double* val) {
  for (int64_t q = 0; q < n; ++q) {
    const int p[3] = {i[q], j[q], k[q]};
    if (comp < 3) *fslot(A, comp, lev[q], p) = val[q];
    else A->p[lev[q]][cidx(A, lev[q], i[q], j[q], k[q])] = val[q];
  }
}

void orc_amr_get(orc_amr* A, int comp, int64_t n, const int32_t* lev, const int32_t* i, const int32_t* j,
                 const int32_t* k, double* val) {
  for (int64_t q = 0; q < n; ++q) {
    const int p[3] = {i[q], j[q], k[q]};
    val[q] = comp < 3 ? *fslot(A, comp, lev[q], p) : A->p[lev[q]][cidx(A, lev[q], i[q], j[q], k[q])];
  }
}

/* One SSP-RK3 step with fixed dt; Poisson solves to relative residual tol.
 * Returns the post-projection max |div| over fluid leaf cells. */
double orc_amr_step(orc_amr* A, double dt, double tol, int* cg_iters) {
  sync_derived(A);
  for (int L = 0; L < A->nl; ++L)
    for (int a = 0; a < 3; ++a) memcpy(A->f0[a][L], A->f[a][L], fsize(A, a, L) * 8);
  apply_bc(A, 1);
  double* rhs[3 * ML];
  for (int L = 0; L < A->nl; ++L)
    for (int a = 0; a < 3; ++a) rhs[a * ML + L] = calloc(fsize(A, a, L), 8);
  A->cg_iters = 0;
  for (int stage = 1; stage <= 3; ++stage) {
    stage_ctx S = {dt, stage, rhs};
    for_faces(A, rhs_fn, &S);
    for_faces(A, comb_fn, &S);
    sync_derived(A);
    project(A, dt, tol);
  }
  for (int L = 0; L < A->nl; ++L)
    for (int a = 0; a < 3; ++a) free(rhs[a * ML + L]);
  double dmax = 0.0;
  FOR_LEAF_CELLS(A, L, i, j, k) {
    if (A->solid[L][cidx(A, L, i, j, k)]) continue;
    const double d = fabs(cell_div(A, L, i, j, k));
    if (d > dmax) dmax = d;
  }
  if (cg_iters) *cg_iters = A->cg_iters;
  return dmax;
}
