// nb_amr_faces.h — MAC face maps of an octree-AMR brick mesh (integer maps).
//
// Storage of face component a (u, v, w for a = 0, 1, 2): one array of
// nbrick*512 + nslab[a]*64 doubles. Slot brick*512 + l holds the low
// a-face of cell l; slab s holds the 64 high a-faces (i == 8) of brick
// slab_brick[a][s]. A brick has an a-slab iff its +a neighbour region is not
// a same-level leaf (coarser, finer, or the non-periodic domain boundary).
//
// Ownership at a 2:1 interface: the fine side owns the four sub-faces; the
// coarse face is "derived" = their average and is recomputed by the sync list
// after every update of owned faces. So every stored face is either owned or
// derived, and readers never need to average.
#pragma once
#include <vector>

#include "nb_amr.h"
#include "nb_flow.cuh"

namespace nb {

enum : int8_t { REL_SAME = 0, REL_COARSER = 1, REL_FINER = 2, REL_BOUNDARY = 3 };

struct AmrFaceMaps {
  int nbrick = 0;
  std::vector<int8_t> rel_lo, rel_hi;  // [nbrick][3]
  std::vector<int> nbr_hi;             // [nbrick][3] same-level +a neighbour brick or -1
  std::vector<int> nbr_lo;             // [nbrick][3] same-level -a neighbour brick or -1
  std::vector<int> slab_id;            // [nbrick][3] slab index or -1
  int nslab[3] = {0, 0, 0};
  std::vector<int> slab_brick[3];
  long long store[3] = {0, 0, 0};      // storage length per component
  // derived faces: dst, then 4 sources (storage indices of the same component)
  std::vector<long long> sync[3];      // 5 entries per derived face
  long long owned[3] = {0, 0, 0};      // owned faces per component
};

// Face storage index of the low a-face of cell p (level coordinates) inside brick r.
inline long long face_lo_index(int r, const int p[3]) {
  return static_cast<long long>(r) * BR3 + (((p[2] & 7) << 6) | ((p[1] & 7) << 3) | (p[0] & 7));
}

void build_face_maps(const AmrTree& t, AmrFaceMaps& M);
// applyVelocityBC (core/src/flow/ns_solver.cpp:221-309) on the owned boundary
// faces of every level, then zero every owned face touching a solid cell.
void build_amr_bc(const AmrTree& t, const AmrFaceMaps& M, const std::vector<uint8_t>& type,
                  const nb_amr_geom& g, bool outflow, std::vector<BcOp>& ops, std::vector<BcOp>& solid_ops);

}  // namespace nb
