// nb_amr_faces.cpp — MAC face ownership, slabs, coarse-face sync lists and
// boundary-condition op lists of an octree-AMR brick mesh.
#include "nb_amr_faces.h"

#include <cstring>
#include <string>

namespace nb {

namespace {

// Slab-local index of a face: the brick-local cell index with axis a dropped.
inline int slab_local(int a, int li, int lj, int lk) {
  return a == 0 ? lj + 8 * lk : (a == 1 ? li + 8 * lk : li + 8 * lj);
}

// Relation of the region next to brick r on axis a, side s (+1 / -1); `same`
// receives the same-level neighbour brick (periodic wrap applied) or -1.
int8_t relation(const AmrTree& t, int r, int a, int s, int& same) {
  const AmrLeaf& f = t.leaves[r];
  const int L = f.level;
  int c[3] = {f.b[0], f.b[1], f.b[2]};
  c[a] += s;
  const int n = t.lnb(L, a);
  same = -1;
  if (c[a] < 0 || c[a] >= n) {
    if (t.geom.bc[2 * a] != NB_BC_PERIODIC) return REL_BOUNDARY;
    c[a] = (c[a] + n) % n;
  }
  const int q = t.find(L, c[0], c[1], c[2]);
  if (q >= 0) {
    same = q;
    return REL_SAME;
  }
  if (L >= 1 && t.find(L - 1, c[0] >> 1, c[1] >> 1, c[2] >> 1) >= 0) return REL_COARSER;
  return REL_FINER;
}

// Wraps level-L cell coordinate p on periodic axes; false if outside the domain.
bool wrap_cell(const AmrTree& t, int L, int p[3]) {
  for (int a = 0; a < 3; ++a) {
    const int n = t.cells(L, a);
    if (p[a] < 0 || p[a] >= n) {
      if (t.geom.bc[2 * a] != NB_BC_PERIODIC) return false;
      p[a] = (p[a] % n + n) % n;
    }
  }
  return true;
}

bool cell_solid(const AmrTree& t, const std::vector<uint8_t>& type, int L, const int p0[3]) {
  int p[3] = {p0[0], p0[1], p0[2]};
  if (!wrap_cell(t, L, p)) return false;
  int lev = -1;
  const int r = t.leaf_of_cell(L, p[0], p[1], p[2], lev);
  if (r < 0) return false;
  int q[3] = {p[0], p[1], p[2]};
  if (lev == L - 1)
    for (int a = 0; a < 3; ++a) q[a] >>= 1;
  if (lev == L + 1)
    for (int a = 0; a < 3; ++a) q[a] <<= 1;
  return type[face_lo_index(r, q)] == CELL_SOLID;
}

// inletVelocityAt(face, first transverse index, ...) at level L
// (core/src/flow/ns_solver.cpp:71-93).
double inlet_value(const AmrTree& t, const nb_amr_geom& g, int face, int L, int jidx, int comp) {
  const nb_face_bc& fb = g.face[face];
  double mag = fb.inlet_speed;
  if (fb.profile == NB_PROFILE_PARABOLIC) {
    const double dy = t.h(L, 1);
    const double H = t.cells(L, 1) * dy;
    const double yc = g.origin[1] + 0.5 * H;
    const double y = g.origin[1] + (jidx + 0.5) * dy;
    const double r = (y - yc) / (0.5 * H);
    mag = 1.5 * fb.inlet_speed * (1.0 - r * r);
  }
  return fb.inlet_axis == comp ? mag : 0.0;
}

[[noreturn]] void map_error(const char* what) {
  throw ApiError{NB_ERR_BAD_ARG, std::string("AMR face maps: ") + what};
}

}  // namespace

void build_face_maps(const AmrTree& t, AmrFaceMaps& M) {
  const int nb = static_cast<int>(t.leaves.size());
  M.nbrick = nb;
  M.rel_lo.assign(3 * nb, REL_SAME);
  M.rel_hi.assign(3 * nb, REL_SAME);
  M.nbr_hi.assign(3 * nb, -1);
  M.nbr_lo.assign(3 * nb, -1);
  M.slab_id.assign(3 * nb, -1);
  for (int a = 0; a < 3; ++a) {
    M.nslab[a] = 0;
    M.slab_brick[a].clear();
    M.sync[a].clear();
  }
  for (int r = 0; r < nb; ++r)
    for (int a = 0; a < 3; ++a) {
      int same = -1;
      M.rel_lo[3 * r + a] = relation(t, r, a, -1, same);
      M.nbr_lo[3 * r + a] = same;
      M.rel_hi[3 * r + a] = relation(t, r, a, +1, same);
      M.nbr_hi[3 * r + a] = same;
      if (M.rel_hi[3 * r + a] != REL_SAME) {
        M.slab_id[3 * r + a] = M.nslab[a]++;
        M.slab_brick[a].push_back(r);
      }
    }
  for (int a = 0; a < 3; ++a) {
    M.store[a] = static_cast<long long>(nb) * BR3 + static_cast<long long>(M.nslab[a]) * 64;
    M.owned[a] = static_cast<long long>(nb) * BR3;
  }
  const long long base = static_cast<long long>(nb) * BR3;
  for (int r = 0; r < nb; ++r) {
    const AmrLeaf& f = t.leaves[r];
    const int L = f.level;
    for (int a = 0; a < 3; ++a) {
      const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
      const bool lo_fine = M.rel_lo[3 * r + a] == REL_FINER;
      const bool hi_fine = M.rel_hi[3 * r + a] == REL_FINER;
      if (M.slab_id[3 * r + a] >= 0 && !hi_fine) M.owned[a] += 64;
      if (lo_fine) M.owned[a] -= 64;
      for (int side = 0; side < 2; ++side) {
        if (side == 0 && !lo_fine) continue;
        if (side == 1 && !hi_fine) continue;
        for (int m2 = 0; m2 < 8; ++m2)
          for (int m1 = 0; m1 < 8; ++m1) {
            int p[3];
            p[a] = BR * f.b[a] + (side ? BR : 0);  // face index at level L
            p[t1] = BR * f.b[t1] + m1;
            p[t2] = BR * f.b[t2] + m2;
            int loc[3] = {0, 0, 0};
            loc[t1] = m1;
            loc[t2] = m2;
            long long dst;
            if (side == 0) {
              loc[a] = 0;
              dst = static_cast<long long>(r) * BR3 + ((loc[2] << 6) | (loc[1] << 3) | loc[0]);
            } else {
              dst = base + static_cast<long long>(M.slab_id[3 * r + a]) * 64 + slab_local(a, loc[0], loc[1], loc[2]);
            }
            M.sync[a].push_back(dst);
            for (int d2 = 0; d2 < 2; ++d2)
              for (int d1 = 0; d1 < 2; ++d1) {
                int q[3];
                q[a] = 2 * p[a];
                q[t1] = 2 * p[t1] + d1;
                q[t2] = 2 * p[t2] + d2;
                long long src;
                if (side == 0) {  // fine cells on the -a side own these as their high (slab) faces
                  int c[3] = {q[0], q[1], q[2]};
                  c[a] -= 1;
                  if (!wrap_cell(t, L + 1, c)) map_error("fine source outside the domain");
                  const int fr = t.find(L + 1, c[0] >> 3, c[1] >> 3, c[2] >> 3);
                  const int sid = fr >= 0 ? M.slab_id[3 * fr + a] : -1;
                  if (sid < 0 || (c[a] & 7) != 7) map_error("fine owner without a slab");
                  src = base + static_cast<long long>(sid) * 64 + slab_local(a, c[0] & 7, c[1] & 7, c[2] & 7);
                } else {  // fine cells on the +a side own these as their low faces
                  int c[3] = {q[0], q[1], q[2]};
                  if (!wrap_cell(t, L + 1, c)) map_error("fine source outside the domain");
                  const int fr = t.find(L + 1, c[0] >> 3, c[1] >> 3, c[2] >> 3);
                  if (fr < 0) map_error("fine owner missing");
                  src = face_lo_index(fr, c);
                }
                M.sync[a].push_back(src);
              }
          }
      }
    }
  }
}

void build_amr_bc(const AmrTree& t, const AmrFaceMaps& M, const std::vector<uint8_t>& type,
                  const nb_amr_geom& g, bool outflow, std::vector<BcOp>& ops, std::vector<BcOp>& solid_ops) {
  const long long base = static_cast<long long>(M.nbrick) * BR3;
  for (int a = 0; a < 3; ++a) {
    const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    for (int r = 0; r < M.nbrick; ++r) {
      const AmrLeaf& f = t.leaves[r];
      const int L = f.level;
      for (int side = 0; side < 2; ++side) {
        const int8_t rel = side ? M.rel_hi[3 * r + a] : M.rel_lo[3 * r + a];
        if (rel != REL_BOUNDARY) continue;
        const int face = 2 * a + side;
        const int bt = g.face[face].type;
        if (bt == NB_BC_PERIODIC || (bt == NB_BC_OUTLET && !outflow)) continue;
        for (int m2 = 0; m2 < 8; ++m2)
          for (int m1 = 0; m1 < 8; ++m1) {
            int loc[3] = {0, 0, 0};
            loc[t1] = m1;
            loc[t2] = m2;
            long long idx, src;
            if (side == 0) {
              loc[a] = 0;
              idx = static_cast<long long>(r) * BR3 + ((loc[2] << 6) | (loc[1] << 3) | loc[0]);
              loc[a] = 1;
              src = static_cast<long long>(r) * BR3 + ((loc[2] << 6) | (loc[1] << 3) | loc[0]);
            } else {
              idx = base + static_cast<long long>(M.slab_id[3 * r + a]) * 64 + slab_local(a, loc[0], loc[1], loc[2]);
              loc[a] = 7;
              src = static_cast<long long>(r) * BR3 + ((loc[2] << 6) | (loc[1] << 3) | loc[0]);
            }
            // first transverse index of the reference's inletVelocityAt call
            const int jidx = a == 0 ? BR * f.b[1] + m1 : BR * f.b[0] + m1;
            if (bt == NB_BC_WALL) ops.push_back(BcOp{a, 0, idx, 0, 0.0});
            else if (bt == NB_BC_INLET) ops.push_back(BcOp{a, 0, idx, 0, inlet_value(t, g, face, L, jidx, a)});
            else ops.push_back(BcOp{a, 1, idx, src, 0.0});
          }
      }
    }
  }
  // every owned face touching a solid cell
  for (int a = 0; a < 3; ++a)
    for (int r = 0; r < M.nbrick; ++r) {
      const AmrLeaf& f = t.leaves[r];
      const int L = f.level;
      for (int l = 0; l < BR3; ++l) {
        const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
        const int p[3] = {BR * f.b[0] + loc[0], BR * f.b[1] + loc[1], BR * f.b[2] + loc[2]};
        const bool own_solid = type[static_cast<size_t>(r) * BR3 + l] == CELL_SOLID;
        if (!(loc[a] == 0 && M.rel_lo[3 * r + a] == REL_FINER)) {  // derived faces are synced
          int q[3] = {p[0], p[1], p[2]};
          q[a] -= 1;
          if (own_solid || cell_solid(t, type, L, q))
            solid_ops.push_back(BcOp{a, 0, static_cast<long long>(r) * BR3 + l, 0, 0.0});
        }
        if (loc[a] == 7 && M.slab_id[3 * r + a] >= 0 && M.rel_hi[3 * r + a] != REL_FINER) {
          int e[3] = {p[0], p[1], p[2]};
          e[a] += 1;
          if (own_solid || cell_solid(t, type, L, e))
            solid_ops.push_back(BcOp{a, 0,
                                     base + static_cast<long long>(M.slab_id[3 * r + a]) * 64 +
                                         slab_local(a, loc[0], loc[1], loc[2]),
                                     0, 0.0});
        }
      }
    }
}

}  // namespace nb
