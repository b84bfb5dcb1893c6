// nb_amr.h — host construction of octree-AMR brick meshes (integer maps).
//
// A mesh is a set of leaf bricks (8x8x8 cells) at octree levels 0..lmax over
// a base grid of nb0 bricks per axis at level 0. A level-L brick at brick
// coordinates (bx,by,bz) covers level-L cells [8bx, 8bx+8) per axis; cells at
// level L have size h0 / 2^L. Leaves are 2:1 balanced across faces, edges and
// corners (every cell of a brick's 3-cell halo lies in a leaf whose level
// differs by at most one). Bricks are ranked by the Morton key of their anchor
// on the finest level (the key of core/include/nabla/mesh/morton.hpp:19-48).
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "nb_internal.h"

namespace nb {

constexpr int AMR_MAXL = AMR_MAXLEV;

struct AmrLeaf {
  int level;
  int b[3];
};

struct AmrGeom {
  int nb0[3];         // level-0 bricks per axis
  double h0[3];       // level-0 cell size
  double origin[3];
  int bc[6];          // NB_BC_* per domain face
  int lmax;           // finest level allowed
};

// A balanced leaf set with its lookup tables.
struct AmrTree {
  AmrGeom geom;
  std::vector<AmrLeaf> leaves;     // ranked (Morton order of finest-level anchors)
  int nlev = 1;                    // levels present: 0..nlev-1
  std::vector<int> lut_off;        // per level offset into lut
  std::vector<int> lut;            // per level dense [bz][by][bx] -> leaf rank or -1
  int lnb(int L, int a) const { return geom.nb0[a] << L; }
  int cells(int L, int a) const { return (geom.nb0[a] * BR) << L; }
  double h(int L, int a) const { return geom.h0[a] / static_cast<double>(1 << L); }
  int find(int L, int bx, int by, int bz) const {
    return lut[lut_off[L] + (bz * lnb(L, 1) + by) * lnb(L, 0) + bx];
  }
  // Leaf containing level-L cell (i,j,k) (in-domain coordinates): returns the
  // leaf rank and its level (L-1, L or L+1 under balance), or -1.
  int leaf_of_cell(int L, int i, int j, int k, int& lev) const;
};

// Builds a balanced tree: every level-0 brick is a leaf; then for L = 0 ..
// lmax-1 the leaves at level L with refine(L, bx, by, bz) true are split, and
// balance is restored after each pass.
AmrTree build_tree(const AmrGeom& g, const std::function<bool(int, int, int, int)>& refine);
// Builds a tree from an explicit leaf list (validates coverage and balance).
AmrTree tree_from_leaves(const AmrGeom& g, const std::vector<AmrLeaf>& leaves, std::string& err);
// The next coarser composite tree: leaves at the finest level merged into parents.
AmrTree coarsen_tree(const AmrTree& t, std::vector<int>& xf_brick, std::vector<int>& xf_oct);
bool tree_balanced(const AmrTree& t);
// Splits leaves[q] where flags[q] != 0 (below lmax), then restores balance.
// Merges every complete octet of sibling leaves whose eight members are all
// flagged into their parent, except where the parent would touch (26
// neighbours, periodic wrap) a leaf two levels finer than itself. The result
// is balanced whenever the input is.
std::vector<AmrLeaf> coarsen_leaves(const AmrGeom& g, const std::vector<AmrLeaf>& leaves,
                                    const std::vector<uint8_t>& flags, std::string& err);
std::vector<AmrLeaf> refine_leaves(const AmrGeom& g, const std::vector<AmrLeaf>& leaves,
                                   const std::vector<uint8_t>& flags, std::string& err);

}  // namespace nb
