// nb_amr_level.h — operator maps of one composite (multi-level) MG level.
#pragma once
#include <functional>
#include <vector>

#include "nb_amr.h"

namespace nb {

struct AmrLevelHost {
  AmrTree tree;
  int wlmax = 0;                   // finest level of the whole mesh (weights are 8^(wlmax-L))
  std::vector<int> bcoord;         // [nbrick][3]
  std::vector<int8_t> blevel;      // [nbrick]
  std::vector<double> bweight;     // [nbrick] cell volume / finest cell volume
  std::vector<uint8_t> type;       // [nbrick*512]
  std::vector<uint16_t> code;      // [nbrick*512] (CODE_* bits, CODE_HASCF)
  std::vector<int> cf_off;         // [nbrick*512 + 1] CSR offsets of coarse-fine couplings
  std::vector<int> cf_nbr;         // neighbour cell index
  std::vector<double> cf_coef;     // per-unit-volume coefficient
  double wfluid = 0.0;             // sum of weights over fluid cells
  uint64_t nfluid = 0;
  // Transfer to the next coarser MG level: coarse brick per brick, and the
  // octant of a merged brick inside its parent (-1: the brick is kept).
  std::vector<int> xf_brick, xf_oct;
};

void amr_level_geometry(AmrLevelHost& A);
// Cell types from a predicate solid(level, i, j, k) on level-L cell indices.
void amr_level_types_from(AmrLevelHost& A, const std::function<bool(int, int, int, int)>& solid);
// Cell types of coarse level C from fine level F (fluid if any child is fluid).
void amr_level_types_coarsened(AmrLevelHost& C, const AmrLevelHost& F);
void amr_level_codes(AmrLevelHost& A);

}  // namespace nb
