// nb_amr.cpp — octree brick trees: refinement, 26-neighbour 2:1 balance,
// Morton ranking, per-level lookup tables, composite coarsening, and the
// merging of flagged sibling octets for regridding.
#include "nb_amr.h"

#include <algorithm>
#include <array>
#include <map>
#include <set>
#include <string>

#include "nb_morton.h"

namespace nb {

namespace {

enum : int8_t { ST_ABSENT = 0, ST_LEAF = 1, ST_REFINED = 2 };

struct States {
  const AmrGeom& g;
  std::vector<std::vector<int8_t>> st;  // per level
  explicit States(const AmrGeom& geom) : g(geom), st(geom.lmax + 1) {
    for (int L = 0; L <= g.lmax; ++L)
      st[L].assign(static_cast<size_t>(g.nb0[0] << L) * (g.nb0[1] << L) * (g.nb0[2] << L), ST_ABSENT);
  }
  int nb(int L, int a) const { return g.nb0[a] << L; }
  size_t idx(int L, int x, int y, int z) const {
    return (static_cast<size_t>(z) * nb(L, 1) + y) * nb(L, 0) + x;
  }
  int8_t& at(int L, int x, int y, int z) { return st[L][idx(L, x, y, z)]; }
  void split(int L, int x, int y, int z) {
    at(L, x, y, z) = ST_REFINED;
    for (int c = 0; c < 8; ++c) at(L + 1, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2)) = ST_LEAF;
  }
  // Level of the leaf containing level-L brick position (x,y,z), or -1 when
  // that region is refined below L (the leaf is finer).
  int leaf_level(int L, int x, int y, int z) const {
    for (int l = L; l >= 0; --l) {
      const int s = L - l;
      const int8_t v = st[l][idx(l, x >> s, y >> s, z >> s)];
      if (v == ST_LEAF) return l;
      if (v == ST_REFINED) return -1;
    }
    return -1;
  }
  // Restores 26-neighbour 2:1 balance by splitting coarse leaves.
  void balance() {
    bool changed = true;
    while (changed) {
      changed = false;
      for (int L = g.lmax; L >= 2; --L) {
        const int nx = nb(L, 0), ny = nb(L, 1), nz = nb(L, 2);
        for (int z = 0; z < nz; ++z)
          for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
              if (st[L][idx(L, x, y, z)] != ST_LEAF) continue;
              for (int d = 0; d < 27; ++d) {
                if (d == 13) continue;
                int c[3] = {x + d % 3 - 1, y + (d / 3) % 3 - 1, z + d / 9 - 1};
                const int n[3] = {nx, ny, nz};
                bool inside = true;
                for (int a = 0; a < 3; ++a)
                  if (c[a] < 0 || c[a] >= n[a]) {
                    if (g.bc[2 * a] == NB_BC_PERIODIC) c[a] = (c[a] + n[a]) % n[a];
                    else inside = false;
                  }
                if (!inside) continue;
                const int lv = leaf_level(L, c[0], c[1], c[2]);
                if (lv >= 0 && L - lv >= 2) {
                  const int s = L - lv;
                  split(lv, c[0] >> s, c[1] >> s, c[2] >> s);
                  changed = true;
                }
              }
            }
      }
    }
  }
};

AmrTree finish(const AmrGeom& g, const States& S) {
  AmrTree t;
  t.geom = g;
  std::vector<std::pair<uint64_t, AmrLeaf>> keyed;
  int maxL = 0;
  for (int L = 0; L <= g.lmax; ++L)
    for (int z = 0; z < S.nb(L, 2); ++z)
      for (int y = 0; y < S.nb(L, 1); ++y)
        for (int x = 0; x < S.nb(L, 0); ++x)
          if (S.st[L][S.idx(L, x, y, z)] == ST_LEAF) {
            const int s = g.lmax - L;
            keyed.push_back({morton_encode(static_cast<uint32_t>(x) << s, static_cast<uint32_t>(y) << s,
                                           static_cast<uint32_t>(z) << s),
                             AmrLeaf{L, {x, y, z}}});
            maxL = std::max(maxL, L);
          }
  std::sort(keyed.begin(), keyed.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  t.nlev = maxL + 1;
  t.leaves.reserve(keyed.size());
  for (auto& k : keyed) t.leaves.push_back(k.second);
  t.lut_off.assign(t.nlev + 1, 0);
  for (int L = 0; L < t.nlev; ++L)
    t.lut_off[L + 1] = t.lut_off[L] + t.lnb(L, 0) * t.lnb(L, 1) * t.lnb(L, 2);
  t.lut.assign(t.lut_off[t.nlev], -1);
  for (size_t r = 0; r < t.leaves.size(); ++r) {
    const AmrLeaf& f = t.leaves[r];
    t.lut[t.lut_off[f.level] + (f.b[2] * t.lnb(f.level, 1) + f.b[1]) * t.lnb(f.level, 0) + f.b[0]] =
        static_cast<int>(r);
  }
  return t;
}

}  // namespace

int AmrTree::leaf_of_cell(int L, int i, int j, int k, int& lev) const {
  if (L < nlev) {
    const int r = find(L, i >> 3, j >> 3, k >> 3);
    if (r >= 0) {
      lev = L;
      return r;
    }
  }
  if (L >= 1 && L - 1 < nlev) {
    const int r = find(L - 1, i >> 4, j >> 4, k >> 4);
    if (r >= 0) {
      lev = L - 1;
      return r;
    }
  }
  if (L + 1 < nlev) {
    const int r = find(L + 1, (2 * i) >> 3, (2 * j) >> 3, (2 * k) >> 3);
    if (r >= 0) {
      lev = L + 1;
      return r;
    }
  }
  lev = -1;
  return -1;
}

AmrTree build_tree(const AmrGeom& g, const std::function<bool(int, int, int, int)>& refine) {
  States S(g);
  std::fill(S.st[0].begin(), S.st[0].end(), ST_LEAF);
  for (int L = 0; L < g.lmax; ++L) {
    std::vector<std::array<int, 3>> todo;
    for (int z = 0; z < S.nb(L, 2); ++z)
      for (int y = 0; y < S.nb(L, 1); ++y)
        for (int x = 0; x < S.nb(L, 0); ++x)
          if (S.st[L][S.idx(L, x, y, z)] == ST_LEAF && refine(L, x, y, z)) todo.push_back({x, y, z});
    for (auto& c : todo) S.split(L, c[0], c[1], c[2]);
    S.balance();
  }
  return finish(g, S);
}

AmrTree tree_from_leaves(const AmrGeom& g, const std::vector<AmrLeaf>& leaves, std::string& err) {
  States S(g);
  for (const AmrLeaf& f : leaves) {
    if (f.level < 0 || f.level > g.lmax) {
      err = "leaf level out of range";
      return AmrTree{};
    }
    for (int a = 0; a < 3; ++a)
      if (f.b[a] < 0 || f.b[a] >= S.nb(f.level, a)) {
        err = "leaf brick coordinate out of range";
        return AmrTree{};
      }
    int8_t& v = S.at(f.level, f.b[0], f.b[1], f.b[2]);
    if (v != ST_ABSENT) {
      err = "duplicate leaf";
      return AmrTree{};
    }
    v = ST_LEAF;
    // mark ancestors refined
    for (int L = f.level - 1, s = 1; L >= 0; --L, ++s) {
      int8_t& a = S.at(L, f.b[0] >> s, f.b[1] >> s, f.b[2] >> s);
      if (a == ST_LEAF) {
        err = "leaves overlap";
        return AmrTree{};
      }
      a = ST_REFINED;
    }
  }
  // coverage: every refined brick has all 8 children present
  for (int L = 0; L < g.lmax; ++L)
    for (int z = 0; z < S.nb(L, 2); ++z)
      for (int y = 0; y < S.nb(L, 1); ++y)
        for (int x = 0; x < S.nb(L, 0); ++x) {
          const int8_t v = S.st[L][S.idx(L, x, y, z)];
          if (L == 0 && v == ST_ABSENT) {
            err = "leaves do not cover the domain";
            return AmrTree{};
          }
          if (v != ST_REFINED) continue;
          for (int c = 0; c < 8; ++c)
            if (S.at(L + 1, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2)) == ST_ABSENT) {
              err = "leaves do not cover the domain";
              return AmrTree{};
            }
        }
  AmrTree t = finish(g, S);
  if (!tree_balanced(t)) err = "leaves are not 2:1 balanced";
  return t;
}

std::vector<AmrLeaf> refine_leaves(const AmrGeom& g, const std::vector<AmrLeaf>& leaves,
                                   const std::vector<uint8_t>& flags, std::string& err) {
  AmrTree t = tree_from_leaves(g, leaves, err);
  if (!err.empty()) return {};
  States S(g);
  for (const AmrLeaf& f : t.leaves) {
    S.at(f.level, f.b[0], f.b[1], f.b[2]) = ST_LEAF;
    for (int L = f.level - 1, s = 1; L >= 0; --L, ++s) S.at(L, f.b[0] >> s, f.b[1] >> s, f.b[2] >> s) = ST_REFINED;
  }
  for (size_t q = 0; q < leaves.size(); ++q) {
    const AmrLeaf& f = leaves[q];
    if (!flags[q]) continue;
    if (f.level >= g.lmax) continue;  // already at the finest allowed level
    S.split(f.level, f.b[0], f.b[1], f.b[2]);
  }
  S.balance();
  return finish(g, S).leaves;
}

std::vector<AmrLeaf> coarsen_leaves(const AmrGeom& g, const std::vector<AmrLeaf>& leaves,
                                    const std::vector<uint8_t>& flags, std::string& err) {
  AmrTree t = tree_from_leaves(g, leaves, err);
  if (!err.empty()) return {};
  // parents whose eight children are all flagged leaves
  std::map<std::array<int, 4>, int> flagged;  // (level, bx, by, bz) of the parent -> flagged children
  for (size_t q = 0; q < leaves.size(); ++q) {
    const AmrLeaf& f = leaves[q];
    if (!flags[q] || f.level == 0) continue;
    ++flagged[{f.level - 1, f.b[0] >> 1, f.b[1] >> 1, f.b[2] >> 1}];
  }
  std::set<std::array<int, 4>> merge;
  for (const auto& [P, n] : flagged) {
    if (n != 8) continue;
    const int Lp = P[0];
    // a leaf two levels finer than the parent inside any neighbour region blocks the merge
    bool ok = true;
    for (int d = 0; d < 27 && ok; ++d) {
      if (d == 13) continue;
      int c[3] = {P[1] + d % 3 - 1, P[2] + (d / 3) % 3 - 1, P[3] + d / 9 - 1};
      bool inside = true;
      for (int a = 0; a < 3; ++a) {
        const int nb = t.lnb(Lp, a);
        if (c[a] < 0 || c[a] >= nb) {
          if (g.bc[2 * a] == NB_BC_PERIODIC) c[a] = (c[a] + nb) % nb;
          else inside = false;
        }
      }
      if (!inside || Lp + 2 >= t.nlev) continue;
      for (int z = 0; z < 4 && ok; ++z)
        for (int y = 0; y < 4 && ok; ++y)
          for (int x = 0; x < 4 && ok; ++x)
            if (t.find(Lp + 2, 4 * c[0] + x, 4 * c[1] + y, 4 * c[2] + z) >= 0) ok = false;
    }
    if (ok) merge.insert(P);
  }
  std::vector<AmrLeaf> out;
  out.reserve(leaves.size());
  for (const AmrLeaf& f : t.leaves) {
    if (f.level > 0 && merge.count({f.level - 1, f.b[0] >> 1, f.b[1] >> 1, f.b[2] >> 1})) continue;
    out.push_back(f);
  }
  for (const auto& P : merge) out.push_back(AmrLeaf{P[0], {P[1], P[2], P[3]}});
  AmrTree check = tree_from_leaves(g, out, err);
  if (!err.empty()) return {};
  if (!tree_balanced(check)) {
    err = "coarsening broke the 2:1 balance";
    return {};
  }
  return check.leaves;
}

bool tree_balanced(const AmrTree& t) {
  const AmrGeom& g = t.geom;
  for (const AmrLeaf& f : t.leaves) {
    const int L = f.level;
    for (int d = 0; d < 27; ++d) {
      if (d == 13) continue;
      int c[3] = {f.b[0] + d % 3 - 1, f.b[1] + (d / 3) % 3 - 1, f.b[2] + d / 9 - 1};
      bool inside = true;
      for (int a = 0; a < 3; ++a) {
        const int n = t.lnb(L, a);
        if (c[a] < 0 || c[a] >= n) {
          if (g.bc[2 * a] == NB_BC_PERIODIC) c[a] = (c[a] + n) % n;
          else inside = false;
        }
      }
      if (!inside) continue;
      // leaf containing brick position c at level L
      int lv = -1;
      for (int l = std::min(L, t.nlev - 1); l >= 0; --l) {
        const int s = L - l;
        if (t.find(l, c[0] >> s, c[1] >> s, c[2] >> s) >= 0) {
          lv = l;
          break;
        }
      }
      // Every violation pairs a finer leaf with a coarser neighbour two or
      // more levels up, so checking coarser neighbours of every leaf suffices.
      if (lv >= 0 && L - lv > 1) return false;
    }
  }
  return true;
}

AmrTree coarsen_tree(const AmrTree& t, std::vector<int>& xf_brick, std::vector<int>& xf_oct) {
  const int Lm = t.nlev - 1;
  AmrGeom g = t.geom;
  States S(g);
  for (const AmrLeaf& f : t.leaves) {
    if (f.level < Lm) {
      S.at(f.level, f.b[0], f.b[1], f.b[2]) = ST_LEAF;
    } else {
      S.at(Lm - 1, f.b[0] >> 1, f.b[1] >> 1, f.b[2] >> 1) = ST_LEAF;
    }
  }
  // ancestors of every leaf are refined
  for (int L = g.lmax; L >= 1; --L)
    for (int z = 0; z < S.nb(L, 2); ++z)
      for (int y = 0; y < S.nb(L, 1); ++y)
        for (int x = 0; x < S.nb(L, 0); ++x) {
          const int8_t v = S.st[L][S.idx(L, x, y, z)];
          if (v == ST_LEAF || v == ST_REFINED) S.at(L - 1, x >> 1, y >> 1, z >> 1) = ST_REFINED;
        }
  AmrTree c = finish(g, S);
  xf_brick.assign(t.leaves.size(), -1);
  xf_oct.assign(t.leaves.size(), -1);
  for (size_t r = 0; r < t.leaves.size(); ++r) {
    const AmrLeaf& f = t.leaves[r];
    if (f.level < Lm) {
      xf_brick[r] = c.find(f.level, f.b[0], f.b[1], f.b[2]);
    } else {
      xf_brick[r] = c.find(Lm - 1, f.b[0] >> 1, f.b[1] >> 1, f.b[2] >> 1);
      xf_oct[r] = (f.b[0] & 1) | ((f.b[1] & 1) << 1) | ((f.b[2] & 1) << 2);
    }
  }
  return c;
}

}  // namespace nb
