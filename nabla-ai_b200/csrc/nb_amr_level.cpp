// nb_amr_level.cpp — per-level operator maps of composite (multi-level) grids.
//
// The pressure operator on a composite grid is the conservative finite-volume
// -Laplacian per unit volume:
//   (A p)_i = (1/V_i) sum_f (area_f / dist_f) (p_i - p_n)
// with area_f the finer cell's face area and dist_f the true centre distance
// (core/src/flow/octree_poisson.cpp:24-32, :64-85, divided by V_i). Same-level
// faces reduce to 1/h^2 exactly (the uniform operator of
// core/src/flow/poisson.cpp:102-134); a fine cell sees its coarse neighbour
// with 1/(1.5 h^2); a coarse cell sees each of its 4 fine neighbours with
// 1/(3 H^2). Solid neighbours are Neumann, outlets Dirichlet (+2/h^2).
#include "nb_amr_level.h"

#include <algorithm>

namespace nb {

void amr_level_geometry(AmrLevelHost& A) {
  const AmrTree& t = A.tree;
  const size_t nb = t.leaves.size();
  A.bcoord.assign(3 * nb, 0);
  A.blevel.assign(nb, 0);
  A.bweight.assign(nb, 1.0);
  for (size_t r = 0; r < nb; ++r) {
    const AmrLeaf& f = t.leaves[r];
    for (int a = 0; a < 3; ++a) A.bcoord[3 * r + a] = f.b[a];
    A.blevel[r] = static_cast<int8_t>(f.level);
    A.bweight[r] = static_cast<double>(1ull << (3 * (A.wlmax - f.level)));  // exact powers of 8
  }
}

void amr_level_types_from(AmrLevelHost& A, const std::function<bool(int, int, int, int)>& solid) {
  const AmrTree& t = A.tree;
  A.type.assign(t.leaves.size() * BR3, CELL_FLUID);
  for (size_t r = 0; r < t.leaves.size(); ++r) {
    const AmrLeaf& f = t.leaves[r];
    for (int l = 0; l < BR3; ++l) {
      const int i = f.b[0] * BR + (l & 7), j = f.b[1] * BR + ((l >> 3) & 7), k = f.b[2] * BR + (l >> 6);
      A.type[r * BR3 + l] = solid(f.level, i, j, k) ? CELL_SOLID : CELL_FLUID;
    }
  }
}

void amr_level_types_coarsened(AmrLevelHost& C, const AmrLevelHost& F) {
  C.type.assign(C.tree.leaves.size() * BR3, CELL_SOLID);
  for (size_t r = 0; r < F.tree.leaves.size(); ++r) {
    const int cb = F.xf_brick[r], oct = F.xf_oct[r];
    for (int l = 0; l < BR3; ++l) {
      const bool fluid = F.type[r * BR3 + l] == CELL_FLUID;
      size_t cidx;
      if (oct < 0) {
        cidx = static_cast<size_t>(cb) * BR3 + l;
        C.type[cidx] = fluid ? CELL_FLUID : CELL_SOLID;
      } else {
        const int ci = (oct & 1) * 4 + ((l & 7) >> 1), cj = ((oct >> 1) & 1) * 4 + (((l >> 3) & 7) >> 1),
                  ck = (oct >> 2) * 4 + ((l >> 6) >> 1);
        cidx = static_cast<size_t>(cb) * BR3 + ((ck << 6) | (cj << 3) | ci);
        if (fluid) C.type[cidx] = CELL_FLUID;  // a coarse cell is fluid if any child is
      }
    }
  }
}

void amr_level_codes(AmrLevelHost& A) {
  const AmrTree& t = A.tree;
  const AmrGeom& g = t.geom;
  const size_t ncell = t.leaves.size() * BR3;
  A.code.assign(ncell, 0);
  A.cf_off.assign(ncell + 1, 0);
  A.cf_nbr.clear();
  A.cf_coef.clear();
  A.wfluid = 0.0;
  A.nfluid = 0;
  for (size_t r = 0; r < t.leaves.size(); ++r) {
    const AmrLeaf& f = t.leaves[r];
    const int L = f.level;
    const int dims[3] = {t.cells(L, 0), t.cells(L, 1), t.cells(L, 2)};
    for (int l = 0; l < BR3; ++l) {
      const size_t c = r * BR3 + l;
      A.cf_off[c] = static_cast<int>(A.cf_nbr.size());
      const uint8_t ty = A.type[c];
      uint32_t code = static_cast<uint32_t>(ty) << CODE_TYPE;
      if (ty != CELL_FLUID) {
        A.code[c] = static_cast<uint16_t>(code);
        continue;
      }
      A.wfluid += A.bweight[r];
      A.nfluid += 1;
      const int p[3] = {f.b[0] * BR + (l & 7), f.b[1] * BR + ((l >> 3) & 7), f.b[2] * BR + (l >> 6)};
      int ncf = 0;
      for (int fc = 0; fc < 6; ++fc) {
        const int a = fc >> 1, side = fc & 1;
        int n[3] = {p[0], p[1], p[2]};
        n[a] += side ? 1 : -1;
        if (n[a] < 0 || n[a] >= dims[a]) {
          const int bt = g.bc[fc];
          if (bt == NB_BC_OUTLET) {
            code |= 1u << (CODE_DIRICHLET + fc);
            continue;
          }
          if (bt != NB_BC_PERIODIC) continue;
          n[a] = (n[a] + dims[a]) % dims[a];
        }
        int lev = -1;
        const int nr = t.leaf_of_cell(L, n[0], n[1], n[2], lev);
        if (nr < 0) continue;
        const AmrLeaf& nf = t.leaves[nr];
        const double ha = t.h(L, a);
        if (lev == L) {
          const int nl = ((n[2] & 7) << 6) | ((n[1] & 7) << 3) | (n[0] & 7);
          if (A.type[static_cast<size_t>(nr) * BR3 + nl] == CELL_FLUID) code |= 1u << fc;
        } else if (lev == L - 1) {
          const int q[3] = {n[0] >> 1, n[1] >> 1, n[2] >> 1};
          const int nl = ((q[2] - nf.b[2] * BR) << 6) | ((q[1] - nf.b[1] * BR) << 3) | (q[0] - nf.b[0] * BR);
          const size_t nc = static_cast<size_t>(nr) * BR3 + nl;
          if (A.type[nc] == CELL_FLUID) {
            A.cf_nbr.push_back(static_cast<int>(nc));
            A.cf_coef.push_back(1.0 / (1.5 * ha * ha));
            ++ncf;
          }
        } else {  // finer: the 4 level-(L+1) cells touching the face
          const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
          for (int d1 = 0; d1 < 2; ++d1)
            for (int d2 = 0; d2 < 2; ++d2) {
              int q[3];
              q[a] = 2 * n[a] + (side ? 0 : 1);
              q[t1] = 2 * n[t1] + d1;
              q[t2] = 2 * n[t2] + d2;
              int lv2 = -1;
              const int fr = t.leaf_of_cell(L + 1, q[0], q[1], q[2], lv2);
              if (fr < 0 || lv2 != L + 1) continue;
              const AmrLeaf& ff = t.leaves[fr];
              const int nl = ((q[2] - ff.b[2] * BR) << 6) | ((q[1] - ff.b[1] * BR) << 3) | (q[0] - ff.b[0] * BR);
              const size_t nc = static_cast<size_t>(fr) * BR3 + nl;
              if (A.type[nc] == CELL_FLUID) {
                A.cf_nbr.push_back(static_cast<int>(nc));
                A.cf_coef.push_back(1.0 / (3.0 * ha * ha));
                ++ncf;
              }
            }
        }
      }
      if (ncf) code |= 1u << CODE_HASCF;
      A.code[c] = static_cast<uint16_t>(code);
    }
  }
  A.cf_off[ncell] = static_cast<int>(A.cf_nbr.size());
}

}  // namespace nb
