// nb_amr_flow.cu — sm_100a kernels of the MAC step on octree-AMR bricks.
//
// The multi-level step generalises the uniform one (core/src/flow/ns_solver.cpp)
// by the conservative face rule of the octree Poisson operator
// (core/src/flow/octree_poisson.cpp:24-32): the fine side of a 2:1 interface
// owns the four sub-faces; the coarse face is their average; the projection
// corrects a sub-face with the gradient over the true centre distance 1.5 h.
// WENO halos across a level jump come from the neighbour level: a fine ghost
// face inside a coarse cell is the linear interpolation of the coarse cell's
// two faces along the normal (constant across), a coarse ghost face is the
// average of its four fine sub-faces; the scheme is locally lower order at
// the interface (the policy of docs/adr/0008-octree-native-flow-solve.md:58-62).
// On a single-level mesh every formula reduces to the uniform reference step.
//
// Every kernel walks bricks with a grid-stride loop and cells with a
// block-stride loop, so any launch shape covers the mesh.
#include <algorithm>
#include <cmath>

#include "nb_amr_flow.cuh"
#include "nb_momentum.cuh"
#include "nb_reduce.cuh"

namespace nb {

namespace {

constexpr int NT = 512;
constexpr int MAX_GRID = 148 * 4;
constexpr int RHS_NT = 256;
constexpr int TW = 15;  // tile offsets -3 .. 11: the brick, its high face layer, 3 ghosts each side
constexpr int TN = TW * TW * TW;
constexpr int8_t R_SAME = 0, R_COARSER = 1, R_FINER = 2, R_BOUNDARY = 3;
constexpr int ACC_MAX = 16;

inline int grid_for(int nbrick) { return nbrick < MAX_GRID ? nbrick : MAX_GRID; }

__device__ __forceinline__ int slab_local(int a, int li, int lj, int lk) {
  return a == 0 ? lj + 8 * lk : (a == 1 ? li + 8 * lk : li + 8 * lj);
}
__device__ __forceinline__ int local_of(const int p[3]) {
  return ((p[2] & 7) << 6) | ((p[1] & 7) << 3) | (p[0] & 7);
}
__device__ __forceinline__ int tix(int a, int b, int c) { return ((c + 3) * TW + (b + 3)) * TW + (a + 3); }

// Leaf rank at level-`lev` brick coordinates (x, y, z), or -1 (no leaf, or
// level/coordinates outside the mesh).
__device__ __forceinline__ int lut_at(const LevelView& L, int lev, int x, int y, int z) {
  if (lev < 0 || lev >= L.nlev) return -1;
  if (x < 0 || y < 0 || z < 0 || x >= L.lnb[lev][0] || y >= L.lnb[lev][1] || z >= L.lnb[lev][2]) return -1;
  return L.lut[L.lut_off[lev] + (z * L.lnb[lev][1] + y) * L.lnb[lev][0] + x];
}

// Leaf containing in-domain level-`lev0` cell p and its level (lev0 - 1,
// lev0 or lev0 + 1 on a balanced mesh); -1 if none.
__device__ __forceinline__ int leaf_of(const LevelView& L, int lev0, const int p[3], int& lev) {
  int r = lut_at(L, lev0, p[0] >> 3, p[1] >> 3, p[2] >> 3);
  if (r >= 0) {
    lev = lev0;
    return r;
  }
  r = lut_at(L, lev0 - 1, p[0] >> 4, p[1] >> 4, p[2] >> 4);
  if (r >= 0) {
    lev = lev0 - 1;
    return r;
  }
  r = lut_at(L, lev0 + 1, p[0] >> 2, p[1] >> 2, p[2] >> 2);
  lev = r >= 0 ? lev0 + 1 : -1;
  return r;
}

// Readers of the ghost walker below. ValRead reads the stored faces. AffRead
// records instead which stored faces the walker combines and with which
// weights: every rule of the walker (wrap, reflection, outlet copy, sub-face
// average, interpolation along the normal) is affine in the stored faces, so
// a halo point's value is c + sum_k w_k f[idx_k] for fixed (idx_k, w_k) on a
// given mesh. The ghost map records these forms once per case.
struct ValRead {
  using V = double;
  __device__ static double rd(const double* __restrict__ f, long long i) { return f[i]; }
  __device__ static double k(double v) { return v; }
};

constexpr int AFF_MAX = 8;  // terms of a recorded form; more: the point keeps the walker

struct Aff {
  double c;  // constant part
  int n;     // number of terms; -1 when more than AFF_MAX distinct faces (or an index past 2^31)
  int idx[AFF_MAX];
  double w[AFF_MAX];
};

__device__ __forceinline__ void aff_axpy(Aff& r, double s, const Aff& x) {  // r += s x
  if (r.n < 0 || x.n < 0) {
    r.n = -1;
    return;
  }
  r.c += s * x.c;
  for (int q = 0; q < x.n; ++q) {
    int j = 0;
    while (j < r.n && r.idx[j] != x.idx[q]) ++j;
    if (j == r.n) {
      if (r.n == AFF_MAX) {
        r.n = -1;
        return;
      }
      r.idx[j] = x.idx[q];
      r.w[j] = 0.0;
      ++r.n;
    }
    r.w[j] += s * x.w[q];
  }
}
__device__ __forceinline__ Aff operator+(Aff a, const Aff& b) {
  aff_axpy(a, 1.0, b);
  return a;
}
__device__ __forceinline__ Aff operator-(Aff a, const Aff& b) {
  aff_axpy(a, -1.0, b);
  return a;
}
__device__ __forceinline__ Aff& operator+=(Aff& a, const Aff& b) {
  aff_axpy(a, 1.0, b);
  return a;
}
__device__ __forceinline__ Aff operator*(double s, Aff a) {
  a.c *= s;
  for (int q = 0; q < a.n; ++q) a.w[q] *= s;
  return a;
}

struct AffRead {
  using V = Aff;
  __device__ static Aff rd(const double* __restrict__, long long i) {
    Aff r;
    r.c = 0.0;
    r.n = i < (1LL << 31) ? 1 : -1;
    r.idx[0] = static_cast<int>(i);
    r.w[0] = 1.0;
    return r;
  }
  __device__ static Aff k(double v) {
    Aff r;
    r.c = v;
    r.n = 0;
    return r;
  }
};

// The walker's nested boundary constants: value = c_{d-1} - (c_{d-2} - (...
// - (c_0 - term))), applied innermost-first when reading values (the
// reference's evaluation order). A recorded form needs no order: it keeps the
// alternating sum S = c_0 - c_1 + ... and returns (-1)^(d-1) (S - term).
template <class RD>
struct Nest {
  double cst[ACC_MAX];
  int d = 0;
  __device__ void push(double v) { cst[d++] = v; }
  __device__ double finish(double term) const {
    for (int q = d - 1; q >= 0; --q) term = cst[q] - term;
    return term;
  }
};
template <>
struct Nest<AffRead> {
  Aff S = AffRead::k(0.0);
  int d = 0;
  __device__ void push(const Aff& v) {
    aff_axpy(S, (d & 1) ? -1.0 : 1.0, v);
    ++d;
  }
  __device__ Aff finish(const Aff& term) const {
    if (d == 0) return term;
    const Aff r = S - term;
    return (d & 1) ? r : -1.0 * r;
  }
};

// Stored a-face at a face position of level `lev0`: p[a] in [0, N_a], the
// other coordinates in-domain. Reads the owner: the minus-side cell's slab
// when that cell is at lev0 and has one (domain high faces, coarse-fine
// sub-faces owned by the fine side), else the plus-side cell's low face
// (same level), the average of its four sub-faces (plus side finer), or the
// coarse face containing it (plus side coarser; p[a] even there).
template <class RD = ValRead>
__device__ typename RD::V face_at(const AmrFlowView& F, int a, const double* __restrict__ f, int lev0,
                                 const int p0[3]) {
  using V = typename RD::V;
  const LevelView& L = F.L;
  const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
  const int N = L.lcells[lev0][a];
  int p[3] = {p0[0], p0[1], p0[2]};
  if (F.per[a] && p[a] >= N) p[a] -= N;
  const bool has_plus = p[a] < N;
  int m[3] = {p[0], p[1], p[2]};
  m[a] -= 1;
  bool has_minus = true;
  if (m[a] < 0) {
    if (F.per[a]) m[a] += N;
    else has_minus = false;
  }
  if (has_minus) {
    int lm;
    const int rm = leaf_of(L, lev0, m, lm);
    if (rm >= 0 && (m[a] & 7) == 7) {
      const int sid = F.slab_id[3 * rm + a];
      if (lm == lev0 && sid >= 0) return RD::rd(f, F.nb + sid * 64LL + slab_local(a, m[0] & 7, m[1] & 7, m[2] & 7));
      if (!has_plus && lm == lev0 + 1 && sid >= 0) {  // domain high face over finer cells
        V s = RD::k(0.0);
        for (int d2 = 0; d2 < 2; ++d2)
          for (int d1 = 0; d1 < 2; ++d1) {
            int c[3];
            c[a] = 2 * m[a] + 1;
            c[t1] = 2 * m[t1] + d1;
            c[t2] = 2 * m[t2] + d2;
            s += RD::rd(f, F.nb + sid * 64LL + slab_local(a, c[0] & 7, c[1] & 7, c[2] & 7));
          }
        return 0.25 * s;
      }
    }
    if (!has_plus && rm >= 0 && lm == lev0 - 1) {  // domain high face over a coarser cell
      const int c[3] = {m[0] >> 1, m[1] >> 1, m[2] >> 1};
      const int sid = F.slab_id[3 * rm + a];
      if (sid >= 0) return RD::rd(f, F.nb + sid * 64LL + slab_local(a, c[0] & 7, c[1] & 7, c[2] & 7));
    }
  }
  if (!has_plus) return RD::k(0.0);
  int lp;
  const int rp = leaf_of(L, lev0, p, lp);
  if (rp < 0) return RD::k(0.0);
  if (lp == lev0) return RD::rd(f, rp * static_cast<long long>(BR3) + local_of(p));
  if (lp == lev0 + 1) {
    V s = RD::k(0.0);
    for (int d2 = 0; d2 < 2; ++d2)
      for (int d1 = 0; d1 < 2; ++d1) {
        int c[3];
        c[a] = 2 * p[a];
        c[t1] = 2 * p[t1] + d1;
        c[t2] = 2 * p[t2] + d2;
        s += RD::rd(f, rp * static_cast<long long>(BR3) + local_of(c));
      }
    return 0.25 * s;
  }
  const int c[3] = {p[0] >> 1, p[1] >> 1, p[2] >> 1};  // coarser: the coarse cell's low face
  return RD::rd(f, rp * static_cast<long long>(BR3) + local_of(c));
}

// a-face value at level `lev0` position p, including the positions that fall
// mid-cell inside a coarser leaf (linear interpolation along the normal).
template <class RD = ValRead>
__device__ typename RD::V face_read(const AmrFlowView& F, int a, const double* __restrict__ f, int lev0,
                                   const int p[3]) {
  using V = typename RD::V;
  const int N = F.L.lcells[lev0][a];
  if ((p[a] & 1) && p[a] < N && lev0 >= 1) {
    int lev;
    const int r = leaf_of(F.L, lev0, p, lev);
    if (r >= 0 && lev == lev0 - 1) {
      int q[3] = {p[0] >> 1, p[1] >> 1, p[2] >> 1};
      const V lo = face_at<RD>(F, a, f, lev0 - 1, q);
      q[a] += 1;
      const V hi = face_at<RD>(F, a, f, lev0 - 1, q);
      return 0.5 * (lo + hi);
    }
  }
  return face_at<RD>(F, a, f, lev0, p);
}

__device__ __forceinline__ double inlet_amr(const AmrFlowView& F, int face, int lev, int jidx, int comp) {
  double mag = F.inlet_speed[face];
  if (F.profile[face] == NB_PROFILE_PARABOLIC) {
    const double dy = F.h[lev][1];
    const double H = F.L.lcells[lev][1] * dy;
    const double yc = F.origin[1] + 0.5 * H;
    const double y = F.origin[1] + (jidx + 0.5) * dy;
    const double r = (y - yc) / (0.5 * H);
    mag = 1.5 * F.inlet_speed[face] * (1.0 - r * r);
  }
  return F.inlet_axis[face] == comp ? mag : 0.0;
}

// Ghost accessors U / Vv / W (core/src/flow/ns_solver.cpp:116-219) at level
// `lev`: domain rules first (wrap, wall reflection 2 u_w - u_m, reflection
// about the stored boundary face 2 u_b - u_r, outlet copy, inlet value), then
// the level-aware face read. The constants of the reference's nested
// expressions c0 - (c1 - (... - term)) are unwound innermost-first.
template <class RD = ValRead>
__device__ __noinline__ typename RD::V amr_acc(const AmrFlowView& F, int comp, const double* __restrict__ f,
                                              int lev, int i, int j, int k) {
  using V = typename RD::V;
  const int nx = F.L.lcells[lev][0], ny = F.L.lcells[lev][1], nz = F.L.lcells[lev][2];
  Nest<RD> cst;
  V term = RD::k(0.0);
  for (int guard = 0; guard < ACC_MAX; ++guard) {
    if (comp == 0) {
      if (k < 0 || k >= nz) {
        if (F.per[2]) { k = wrapi(k, nz); continue; }
        const int face = k < 0 ? 4 : 5;
        cst.push(RD::k(2.0 * F.wallv[face][0]));
        k = k < 0 ? (-1 - k) : (2 * nz - 1 - k);
        continue;
      }
      if (j < 0 || j >= ny) {
        if (F.per[1]) { j = wrapi(j, ny); continue; }
        const int face = j < 0 ? 2 : 3;
        cst.push(RD::k(2.0 * F.wallv[face][0]));
        j = j < 0 ? (-1 - j) : (2 * ny - 1 - j);
        continue;
      }
      if (i < 0 || i > nx) {
        if (F.per[0]) { i = wrapi(i, nx); continue; }
        const int ib = i < 0 ? 0 : nx, face = i < 0 ? 0 : 1;
        const int pb[3] = {ib, j, k};
        if (F.L.bc[face] == NB_BC_OUTLET) { term = face_read<RD>(F, 0, f, lev, pb); break; }
        cst.push(2.0 * face_read<RD>(F, 0, f, lev, pb));
        i = 2 * ib - i;
        continue;
      }
    } else if (comp == 1) {
      if (k < 0 || k >= nz) {
        if (F.per[2]) { k = wrapi(k, nz); continue; }
        const int face = k < 0 ? 4 : 5;
        cst.push(RD::k(2.0 * F.wallv[face][1]));
        k = k < 0 ? (-1 - k) : (2 * nz - 1 - k);
        continue;
      }
      if (i < 0 || i >= nx) {
        if (F.per[0]) { i = wrapi(i, nx); continue; }
        const int im = i < 0 ? (-1 - i) : (2 * nx - 1 - i), face = i < 0 ? 0 : 1;
        if (F.L.bc[face] == NB_BC_INLET) {
          cst.push(RD::k(2.0 * inlet_amr(F, face, lev, j, 1)));
          i = im;
          continue;
        }
        if (F.L.bc[face] == NB_BC_OUTLET) {
          // j is unresolved here; stencil points have it in range, the clamp
          // keeps unused corner points in bounds.
          const int pb[3] = {i < 0 ? 0 : nx - 1, min(max(j, 0), ny), k};
          term = face_read<RD>(F, 1, f, lev, pb);
          break;
        }
        cst.push(RD::k(2.0 * F.wallv[face][1]));
        i = im;
        continue;
      }
      if (j < 0 || j > ny) {
        if (F.per[1]) { j = wrapi(j, ny); continue; }
        const int jb = j < 0 ? 0 : ny, face = j < 0 ? 2 : 3;
        const int pb[3] = {i, jb, k};
        if (F.L.bc[face] == NB_BC_OUTLET) { term = face_read<RD>(F, 1, f, lev, pb); break; }
        cst.push(2.0 * face_read<RD>(F, 1, f, lev, pb));
        j = 2 * jb - j;
        continue;
      }
    } else {
      if (j < 0 || j >= ny) {
        if (F.per[1]) { j = wrapi(j, ny); continue; }
        const int face = j < 0 ? 2 : 3;
        cst.push(RD::k(2.0 * F.wallv[face][2]));
        j = j < 0 ? (-1 - j) : (2 * ny - 1 - j);
        continue;
      }
      if (i < 0 || i >= nx) {
        if (F.per[0]) { i = wrapi(i, nx); continue; }
        const int im = i < 0 ? (-1 - i) : (2 * nx - 1 - i), face = i < 0 ? 0 : 1;
        if (F.L.bc[face] == NB_BC_OUTLET) {
          const int pb[3] = {i < 0 ? 0 : nx - 1, j, min(max(k, 0), nz)};
          term = face_read<RD>(F, 2, f, lev, pb);
          break;
        }
        cst.push(RD::k(2.0 * F.wallv[face][2]));
        i = im;
        continue;
      }
      if (k < 0 || k > nz) {
        if (F.per[2]) { k = wrapi(k, nz); continue; }
        const int kb = k < 0 ? 0 : nz;
        const int pb[3] = {i, j, kb};
        cst.push(2.0 * face_read<RD>(F, 2, f, lev, pb));
        k = 2 * kb - k;
        continue;
      }
    }
    const int pt[3] = {i, j, k};
    term = face_read<RD>(F, comp, f, lev, pt);
    break;
  }
  return cst.finish(term);
}

// Solid flag of the level-`lev0` cell p (outside the domain: not solid).
__device__ __forceinline__ bool solid_at(const AmrFlowView& F, int lev0, const int p0[3]) {
  int p[3] = {p0[0], p0[1], p0[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int n = F.L.lcells[lev0][a];
    if (p[a] < 0 || p[a] >= n) {
      if (!F.per[a]) return false;
      p[a] = wrapi(p[a], n);
    }
  }
  int lev;
  const int r = leaf_of(F.L, lev0, p, lev);
  if (r < 0) return false;
  int q[3] = {p[0], p[1], p[2]};
  if (lev == lev0 - 1)
    for (int d = 0; d < 3; ++d) q[d] >>= 1;
  if (lev == lev0 + 1)
    for (int d = 0; d < 3; ++d) q[d] <<= 1;
  return F.L.type[r * static_cast<long long>(BR3) + local_of(q)] == CELL_SOLID;
}

template <typename T>
struct TileRef {
  const T* t;
  __device__ __forceinline__ T operator()(int i, int j, int k) const { return t[tix(i, j, k)]; }
};

// Same-level leaves of the 27 brick positions around (and at) the brick, -1
// where the position is outside the mesh or covered at another level.
__device__ __forceinline__ void fill_nb27(const LevelView& L, int brick, int lev, int* nb27) {
  if (threadIdx.x < 27) {
    const int q = threadIdx.x;
    nb27[q] = lut_at(L, lev, L.bcoord[3 * brick] + q % 3 - 1, L.bcoord[3 * brick + 1] + (q / 3) % 3 - 1,
                     L.bcoord[3 * brick + 2] + q / 9 - 1);
  }
}

// Point p of the momentum kernel's tile (offsets -3..11 around a brick at
// cell origin o of a level with N cells): never read by a stencil (skip), the
// brick's own cell, or a halo point at level cell g with, strictly inside the
// domain, the same-level leaf r that holds it (-1: another level or none).
struct HaloPt {
  bool skip, inner;
  int g[3];
  int r;
  long long slot;
  // A halo point strictly inside the domain whose leaf is at this level is
  // that leaf's stored cell slot: the ghost walker applies no domain rule
  // there and its face lookup returns the slot (the minus-side slab is read
  // only across a periodic low boundary, excluded per component).
  __device__ bool fast(int a, const int per[3]) const { return r >= 0 && (g[a] >= 1 || !per[a]); }
};

__device__ __forceinline__ HaloPt halo_pt(const int o[3], const int N[3], const int* nb27, int p) {
  HaloPt h;
  const int ti = p % TW - 3, tj = (p / TW) % TW - 3, tk = p / (TW * TW) - 3;
  h.skip = (ti < -1 || ti > 9) + (tj < -1 || tj > 9) + (tk < -1 || tk > 9) > 1;
  h.inner = ti >= 0 && ti < 8 && tj >= 0 && tj < 8 && tk >= 0 && tk < 8;
  h.g[0] = o[0] + ti;
  h.g[1] = o[1] + tj;
  h.g[2] = o[2] + tk;
  h.r = -1;
  if (!h.skip && !h.inner && h.g[0] >= 0 && h.g[1] >= 0 && h.g[2] >= 0 && h.g[0] < N[0] && h.g[1] < N[1] &&
      h.g[2] < N[2])
    h.r = nb27[(ti < 0 ? 0 : (ti < 8 ? 1 : 2)) + 3 * (tj < 0 ? 0 : (tj < 8 ? 1 : 2)) +
               9 * (tk < 0 ? 0 : (tk < 8 ? 1 : 2))];
  h.slot = ((tk & 7) << 6) | ((tj & 7) << 3) | (ti & 7);
  return h;
}

// Ghost map of the momentum kernel: one entry per (tile point, component) that
// the same-level fast path does not serve, in the brick's range
// [gm_off[b], gm_off[b + 1]). Entry .x = p | a << 12 | nt << 14 and .y = the
// first of its nt terms (index into the component's array, FP32 weight bits):
// the value is sum_q w_q f[idx_q]. nt = GM_WALK keeps the walker for the
// point: a form with a constant part (inlet values, moving walls), more than
// AFF_MAX terms, or a weight that FP32 does not hold exactly.
constexpr unsigned GM_WALK = 15;

constexpr unsigned GM_NONE = 0xFF;  // (point, component) served by the fast path: no entry

// The recorded form of halo point h's component a: its term count, or GM_WALK.
__device__ __forceinline__ unsigned ghost_form(const AmrFlowView& F, int lev, const HaloPt& h, int a, Aff& A) {
  A = amr_acc<AffRead>(F, a, nullptr, lev, h.g[0], h.g[1], h.g[2]);
  bool ok = A.n >= 0 && A.c == 0.0;
  for (int q = 0; ok && q < A.n; ++q) ok = static_cast<double>(static_cast<float>(A.w[q])) == A.w[q];
  return ok ? static_cast<unsigned>(A.n) : GM_WALK;
}

// Pass 1: entries and terms per brick into count[2b], count[2b + 1].
__global__ void __launch_bounds__(RHS_NT) k_ghost_map(AmrFlowView F, int* __restrict__ count) {
  const LevelView& L = F.L;
  __shared__ int nb27[27];
  __shared__ int ne, nterm;
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int lev = L.blevel[brick];
    const int o[3] = {L.bcoord[3 * brick] * BR, L.bcoord[3 * brick + 1] * BR, L.bcoord[3 * brick + 2] * BR};
    const int N[3] = {L.lcells[lev][0], L.lcells[lev][1], L.lcells[lev][2]};
    fill_nb27(L, brick, lev, nb27);
    if (threadIdx.x == 0) ne = nterm = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < TN; p += blockDim.x) {
      const HaloPt h = halo_pt(o, N, nb27, p);
      if (h.skip || h.inner) continue;
      for (int a = 0; a < 3; ++a) {
        if (h.fast(a, F.per)) continue;
        Aff A;
        const unsigned c = ghost_form(F, lev, h, a, A);
        atomicAdd(&ne, 1);
        if (c != GM_WALK && c > 0) atomicAdd(&nterm, static_cast<int>(c));
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      count[2 * brick] = ne;
      count[2 * brick + 1] = nterm;
    }
    __syncthreads();
  }
}

// Exclusive prefix sums of (x, y) over the CTA's threads in thread order
// (RHS_NT threads; ws holds 2 x RHS_NT / 32 ints).
__device__ __forceinline__ void block_exscan2(int& x, int& y, int* ws) {
  constexpr int NW = RHS_NT / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int ix = x, iy = y;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int ux = __shfl_up_sync(0xffffffffu, ix, d), uy = __shfl_up_sync(0xffffffffu, iy, d);
    if (lane >= d) {
      ix += ux;
      iy += uy;
    }
  }
  if (lane == 31) {
    ws[w] = ix;
    ws[NW + w] = iy;
  }
  __syncthreads();
  int px = 0, py = 0;
  for (int k = 0; k < w; ++k) {
    px += ws[k];
    py += ws[NW + k];
  }
  x = px + ix - x;
  y = py + iy - y;
  __syncthreads();
}

// Pass 2: a brick's entries at the host-scanned offsets eoff / toff, sorted by
// component, then tile position (neighbouring threads of the momentum kernel
// then gather neighbouring cells). The term codes go to a shared table first,
// a block scan in that order places every entry, and each entry's form is
// recorded again where it is written.
__global__ void __launch_bounds__(RHS_NT) k_ghost_fill(AmrFlowView F, const int* __restrict__ eoff,
                                                       const int* __restrict__ toff, uint2* __restrict__ ent,
                                                       int2* __restrict__ term) {
  constexpr int NE = 3 * TN;                         // (component, tile point) pairs, component-major
  constexpr int CH = (NE + RHS_NT - 1) / RHS_NT;     // pairs per thread, in order
  const LevelView& L = F.L;
  __shared__ int nb27[27];
  __shared__ uint8_t tcode[NE];
  __shared__ int ws[2 * (RHS_NT / 32)];
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int lev = L.blevel[brick];
    const int o[3] = {L.bcoord[3 * brick] * BR, L.bcoord[3 * brick + 1] * BR, L.bcoord[3 * brick + 2] * BR};
    const int N[3] = {L.lcells[lev][0], L.lcells[lev][1], L.lcells[lev][2]};
    fill_nb27(L, brick, lev, nb27);
    __syncthreads();
    for (int p = threadIdx.x; p < TN; p += blockDim.x) {
      const HaloPt h = halo_pt(o, N, nb27, p);
      for (int a = 0; a < 3; ++a) {
        unsigned c = GM_NONE;
        if (!h.skip && !h.inner && !h.fast(a, F.per)) {
          Aff A;
          c = ghost_form(F, lev, h, a, A);
        }
        tcode[a * TN + p] = static_cast<uint8_t>(c);
      }
    }
    __syncthreads();
    const int e0 = threadIdx.x * CH, e1 = min(e0 + CH, NE);
    int ne = 0, nt = 0;
    for (int e = e0; e < e1; ++e) {
      const unsigned c = tcode[e];
      if (c == GM_NONE) continue;
      ++ne;
      if (c != GM_WALK) nt += static_cast<int>(c);
    }
    block_exscan2(ne, nt, ws);
    int ei = eoff[brick] + ne, ti = toff[brick] + nt;
    for (int e = e0; e < e1; ++e) {
      const unsigned c = tcode[e];
      if (c == GM_NONE) continue;
      const int a = e / TN, p = e - a * TN;
      ent[ei++] = make_uint2(static_cast<unsigned>(p) | (static_cast<unsigned>(a) << 12) | (c << 14),
                             static_cast<unsigned>(ti));
      if (c != GM_WALK && c > 0) {
        Aff A;
        ghost_form(F, lev, halo_pt(o, N, nb27, p), a, A);
        for (unsigned q = 0; q < c; ++q)
          term[ti + q] = make_int2(A.idx[q], __float_as_int(static_cast<float>(A.w[q])));
        ti += static_cast<int>(c);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Fused momentum RHS + SSP-RK3 combine on AMR bricks (owned faces only).
// One CTA per brick (grid-stride): stage u, v, w at the brick's level over
// offsets -3..11 in shared memory, then every owned face of the brick (low
// faces, plus the high slab faces it owns at a coarser neighbour) gets
// R = -div(u u) + nu lap u + f and the stage combination. R = 0 on domain
// boundary faces (ns_solver.cpp:325, even when periodic) and on faces touching
// a solid.
// ---------------------------------------------------------------------------
// Bounds: FP32 tiles (40.5 KB) at 4 CTAs an SM, 64 registers; FP64 tiles
// (81 KB) fit two CTAs an SM.
template <typename T>
__global__ void __launch_bounds__(RHS_NT, sizeof(T) == 4 ? 4 : 2)
    k_amr_rhs_rk(AmrFlowView F, int stage, const double* __restrict__ dtp, const double* __restrict__ u,
                 const double* __restrict__ v, const double* __restrict__ w, const double* __restrict__ u0,
                 const double* __restrict__ v0, const double* __restrict__ w0, double* __restrict__ uo,
                 double* __restrict__ vo, double* __restrict__ wo) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tile[3];
  tile[0] = reinterpret_cast<T*>(smraw);
  tile[1] = tile[0] + TN;
  tile[2] = tile[1] + TN;
  const LevelView& L = F.L;
  const double dt = *dtp;
  const double c1 = 1.0 / 3.0, c2 = 2.0 / 3.0;
  auto comb = [&](double a0, double a, double r) -> double {
    if (stage == 1) return a0 + dt * r;
    if (stage == 2) return 0.75 * a0 + 0.25 * (a + dt * r);
    return c1 * a0 + c2 * (a + dt * r);
  };
  const double* in[3] = {u, v, w};
  const double* in0[3] = {u0, v0, w0};
  double* out[3] = {uo, vo, wo};
  __shared__ int nb27[27];
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int lev = L.blevel[brick];
    const int o[3] = {L.bcoord[3 * brick] * BR, L.bcoord[3 * brick + 1] * BR, L.bcoord[3 * brick + 2] * BR};
    const int N[3] = {L.lcells[lev][0], L.lcells[lev][1], L.lcells[lev][2]};
    fill_nb27(L, brick, lev, nb27);
    __syncthreads();
    const bool mapped = F.gm_off != nullptr;
    for (int p = threadIdx.x; p < TN; p += blockDim.x) {
      const HaloPt h = halo_pt(o, N, nb27, p);
      if (h.skip) continue;
      for (int a = 0; a < 3; ++a) {
        double val;
        if (h.inner) val = in[a][brick * static_cast<long long>(BR3) + h.slot];
        else if (h.fast(a, F.per)) val = in[a][h.r * static_cast<long long>(BR3) + h.slot];
        else if (mapped) continue;  // the brick's ghost map below
        else val = amr_acc(F, a, in[a], lev, h.g[0], h.g[1], h.g[2]);
        tile[a][p] = static_cast<T>(val);
      }
    }
    if (mapped) {  // the walker's points: recorded forms, or the walker itself (GM_WALK)
      const int e1 = F.gm_off[brick + 1];
      for (int e = F.gm_off[brick] + threadIdx.x; e < e1; e += blockDim.x) {
        const uint2 E = F.gm_ent[e];
        const int p = E.x & 4095, a = (E.x >> 12) & 3, nt = static_cast<int>(E.x >> 14);
        double val;
        if (nt == static_cast<int>(GM_WALK)) {
          val = amr_acc(F, a, in[a], lev, o[0] + p % TW - 3, o[1] + (p / TW) % TW - 3, o[2] + p / (TW * TW) - 3);
        } else {
          val = 0.0;
          for (int q = 0; q < nt; ++q) {
            const int2 t = F.gm_term[E.y + q];
            val += static_cast<double>(__int_as_float(t.y)) * in[a][t.x];
          }
        }
        tile[a][p] = static_cast<T>(val);
      }
    }
    __syncthreads();
    const T hx = T(F.h[lev][0]), hy = T(F.h[lev][1]), hz = T(F.h[lev][2]);
    const T nu = T(F.nu);
    // Face jobs: the 3 x 512 low faces, then 3 x 64 high slab faces (a brick
    // with a slab owns its high faces at a coarser neighbour or the domain
    // boundary). One RHS call site for every component and position.
    for (int job = threadIdx.x; job < 3 * BR3 + 3 * 64; job += blockDim.x) {
      const bool high = job >= 3 * BR3;
      const int a = high ? (job - 3 * BR3) >> 6 : job >> 9;
      int loc[3];
      if (high) {
        const int m = (job - 3 * BR3) & 63;
        loc[a] = 7;
        loc[a == 0 ? 1 : 0] = m & 7;
        loc[a == 2 ? 1 : 2] = m >> 3;
      } else {
        loc[0] = job & 7;
        loc[1] = (job >> 3) & 7;
        loc[2] = (job >> 6) & 7;
      }
      const int l = (loc[2] << 6) | (loc[1] << 3) | loc[0];
      const int sid = F.slab_id[3 * brick + a];
      const int rel_hi = F.rel_hi[3 * brick + a];
      // low face (derived when the -a side is finer: synced afterwards);
      // high slab face: RHS at a coarser neighbour, R = 0 at the domain boundary
      if (high ? (sid < 0 || rel_hi == R_FINER) : (loc[a] == 0 && F.rel_lo[3 * brick + a] == R_FINER)) continue;
      const int p[3] = {o[0] + loc[0], o[1] + loc[1], o[2] + loc[2]};
      const long long c = brick * static_cast<long long>(BR3) + l;
      const long long dst = high ? F.nb + sid * 64LL + slab_local(a, loc[0], loc[1], loc[2]) : c;
      bool live = L.type[c] != CELL_SOLID;
      if (high) {
        live = live && rel_hi == R_COARSER;
        if (live) {
          int q[3] = {p[0], p[1], p[2]};
          q[a] += 1;
          live = !solid_at(F, lev, q);
        }
      } else {
        live = live && p[a] != 0;
        if (live) {
          if (loc[a] > 0) {
            live = L.type[c - (a == 0 ? 1 : (a == 1 ? 8 : 64))] != CELL_SOLID;
          } else {
            int q[3] = {p[0], p[1], p[2]};
            q[a] -= 1;
            live = !solid_at(F, lev, q);
          }
        }
      }
      double r = 0.0;
      if (live) {
        const int e = tix(loc[0] + (high && a == 0), loc[1] + (high && a == 1), loc[2] + (high && a == 2));
        r = static_cast<double>(
            rhs_face<T, TW, TW * TW>(tile[0], tile[1], tile[2], a, e, F.weno, hx, hy, hz, nu, T(F.bf[a])));
      }
      out[a][dst] = comb(in0[a][dst], in[a][dst], r);
    }
    __syncthreads();
  }
}

// Derived coarse faces = average of their four fine sub-faces.
__global__ void k_amr_sync(const long long* __restrict__ list, int n, double* __restrict__ f) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const long long* e = list + 5 * static_cast<long long>(m);
    f[e[0]] = 0.25 * (((f[e[1]] + f[e[2]]) + f[e[3]]) + f[e[4]]);
  }
}

// High a-face of brick-local cell l: next cell's low face, the brick's slab,
// or the same-level +a neighbour's low face.
__device__ __forceinline__ double hi_face(const AmrFlowView& F, int a, const double* __restrict__ f, int brick,
                                          int l, const int loc[3]) {
  if (loc[a] < 7) return f[brick * static_cast<long long>(BR3) + l + (a == 0 ? 1 : (a == 1 ? 8 : 64))];
  const int sid = F.slab_id[3 * brick + a];
  if (sid >= 0) return f[F.nb + sid * 64LL + slab_local(a, loc[0], loc[1], loc[2])];
  const int nb = F.nbr_hi[3 * brick + a];
  if (nb < 0) return 0.0;
  int e[3] = {loc[0], loc[1], loc[2]};
  e[a] = 0;
  return f[nb * static_cast<long long>(BR3) + ((e[2] << 6) | (e[1] << 3) | e[0])];
}

__device__ __forceinline__ double cell_div(const AmrFlowView& F, const double* u, const double* v, const double* w,
                                           int brick, int l, int lev) {
  const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
  const long long c = brick * static_cast<long long>(BR3) + l;
  double d = (hi_face(F, 0, u, brick, l, loc) - u[c]) / F.h[lev][0] +
             (hi_face(F, 1, v, brick, l, loc) - v[c]) / F.h[lev][1];
  d += (hi_face(F, 2, w, brick, l, loc) - w[c]) / F.h[lev][2];
  return d;
}

// b = -div u* on fluid cells (ns_solver.cpp:482-498), per unit volume.
__global__ void __launch_bounds__(NT) k_amr_div(AmrFlowView F, const double* __restrict__ u,
                                                const double* __restrict__ v, const double* __restrict__ w,
                                                double* __restrict__ b) {
  const LevelView& L = F.L;
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x)
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      const long long c = brick * static_cast<long long>(BR3) + l;
      double o = 0.0;
      if (L.type[c] == CELL_FLUID) o = -cell_div(F, u, v, w, brick, l, L.blevel[brick]);
      b[c] = o;
    }
}

// phi of the level-lev0 cell p (wrapped into the domain; at a finer leaf the
// first child, which the caller never asks for).
__device__ __forceinline__ double phi_cell(const AmrFlowView& F, const double* __restrict__ phi, int lev0,
                                           const int p0[3]) {
  int p[3] = {p0[0], p0[1], p0[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) p[a] = wrapi(p[a], F.L.lcells[lev0][a]);
  int lev;
  const int r = leaf_of(F.L, lev0, p, lev);
  if (r < 0) return 0.0;
  int q[3] = {p[0], p[1], p[2]};
  if (lev == lev0 - 1)
    for (int d = 0; d < 3; ++d) q[d] >>= 1;
  if (lev == lev0 + 1)
    for (int d = 0; d < 3; ++d) q[d] <<= 1;
  return phi[r * static_cast<long long>(BR3) + local_of(q)];
}

// Projection correction on owned faces (ns_solver.cpp:528-562) + p = phi/dt.
__global__ void __launch_bounds__(NT) k_amr_correct(AmrFlowView F, const double* __restrict__ phi,
                                                    const double* __restrict__ dtp, double* __restrict__ u,
                                                    double* __restrict__ v, double* __restrict__ w,
                                                    double* __restrict__ pout) {
  const LevelView& L = F.L;
  const double dt = *dtp;
  double* f[3] = {u, v, w};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x)
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      const long long c = brick * static_cast<long long>(BR3) + l;
      pout[c] = phi[c] / dt;
      if (L.type[c] == CELL_SOLID) continue;
      const int lev = L.blevel[brick];
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      const int o[3] = {L.bcoord[3 * brick] * BR, L.bcoord[3 * brick + 1] * BR, L.bcoord[3 * brick + 2] * BR};
      const int p[3] = {o[0] + loc[0], o[1] + loc[1], o[2] + loc[2]};
      const double pc = phi[c];
      for (int a = 0; a < 3; ++a) {
        const int stride = a == 0 ? 1 : (a == 1 ? 8 : 64);
        const double h = F.h[lev][a];
        if (loc[a] > 0) {
          if (L.type[c - stride] != CELL_SOLID) f[a][c] -= (pc - phi[c - stride]) / h;
        } else {
          const int8_t rel = F.rel_lo[3 * brick + a];
          if (rel == R_BOUNDARY) {
            // outlet ghost -phi (Dirichlet 0), Neumann ghost phi (ns_solver.cpp:508-526)
            const double g = L.bc[2 * a] == NB_BC_OUTLET ? -pc : pc;
            f[a][c] -= (pc - g) / h;
          } else if (rel == R_SAME) {
            // the -a cell is the same-level neighbour's (periodic wrap applied)
            // cell with loc[a] = 7: the cell solid_at and phi_cell resolve
            const long long cn = F.nbr_lo[3 * brick + a] * static_cast<long long>(BR3) + l + 7 * stride;
            if (L.type[cn] != CELL_SOLID) f[a][c] -= (pc - phi[cn]) / h;
          } else if (rel != R_FINER) {
            int q[3] = {p[0], p[1], p[2]};
            q[a] -= 1;
            if (!solid_at(F, lev, q)) {
              const double d = rel == R_COARSER ? 1.5 * h : h;
              f[a][c] -= (pc - phi_cell(F, phi, lev, q)) / d;
            }
          }
        }
        const int sid = F.slab_id[3 * brick + a];
        if (loc[a] == 7 && sid >= 0) {
          const int8_t rel = F.rel_hi[3 * brick + a];
          const long long s = F.nb + sid * 64LL + slab_local(a, loc[0], loc[1], loc[2]);
          if (rel == R_BOUNDARY) {
            const double g = L.bc[2 * a + 1] == NB_BC_OUTLET ? -pc : pc;
            f[a][s] -= (g - pc) / h;
          } else if (rel == R_COARSER) {
            int q[3] = {p[0], p[1], p[2]};
            q[a] += 1;
            if (!solid_at(F, lev, q)) f[a][s] -= (phi_cell(F, phi, lev, q) - pc) / (1.5 * h);
          }
        }
      }
    }
}

// Step diagnostics: [0] sum (u-u0)^2 over owned faces, [1] sum div^2 and
// [2] max |div| over fluid cells, [3] net boundary mass flux.
__global__ void __launch_bounds__(NT) k_amr_diag(AmrFlowView F, const double* __restrict__ u,
                                                 const double* __restrict__ v, const double* __restrict__ w,
                                                 const double* __restrict__ u0, const double* __restrict__ v0,
                                                 const double* __restrict__ w0, RedBuf rb, AmrStepScalars* out) {
  const LevelView& L = F.L;
  const double* f[3] = {u, v, w};
  const double* f0[3] = {u0, v0, w0};
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x)
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      const long long c = brick * static_cast<long long>(BR3) + l;
      const int lev = L.blevel[brick];
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      for (int a = 0; a < 3; ++a) {
        const double area = F.h[lev][(a + 1) % 3] * F.h[lev][(a + 2) % 3];
        if (!(loc[a] == 0 && F.rel_lo[3 * brick + a] == R_FINER)) {
          const double d = f[a][c] - f0[a][c];
          acc[0] += d * d;
          if (loc[a] == 0 && F.rel_lo[3 * brick + a] == R_BOUNDARY) acc[3] += f[a][c] * area;
        }
        const int sid = F.slab_id[3 * brick + a];
        if (loc[a] == 7 && sid >= 0 && F.rel_hi[3 * brick + a] != R_FINER) {
          const long long s = F.nb + sid * 64LL + slab_local(a, loc[0], loc[1], loc[2]);
          const double d = f[a][s] - f0[a][s];
          acc[0] += d * d;
          if (F.rel_hi[3 * brick + a] == R_BOUNDARY) acc[3] -= f[a][s] * area;
        }
      }
      if (L.type[c] == CELL_FLUID) {
        const double d = cell_div(F, u, v, w, brick, l, lev);
        acc[1] += d * d;
        acc[2] = fmax(acc[2], fabs(d));
      }
    }
  grid_reduce<4, (1u << 2)>(acc, rb, [=] __device__(const double* t) {
    out->du2 = t[0];
    out->div2 = t[1];
    out->divmax = t[2];
    out->mass = t[3];
  });
}

// computeDt over leaf cells (ns_solver.cpp:581-603), each with its own spacing;
// the running maximum starts from the level-0 viscous term as the reference's does.
__global__ void __launch_bounds__(NT) k_amr_max_inv(AmrFlowView F, const double* __restrict__ u,
                                                    const double* __restrict__ v, const double* __restrict__ w,
                                                    double cfl, double* dt_out, RedBuf rb, AmrStepScalars* out) {
  const LevelView& L = F.L;
  auto visc_of = [&](int lev) {
    return 2.0 * F.nu *
           (1.0 / (F.h[lev][0] * F.h[lev][0]) + 1.0 / (F.h[lev][1] * F.h[lev][1]) +
            1.0 / (F.h[lev][2] * F.h[lev][2]));
  };
  double m[1] = {visc_of(0) + 1e-300};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x)
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      const long long c = brick * static_cast<long long>(BR3) + l;
      if (L.type[c] != CELL_FLUID) continue;
      const int lev = L.blevel[brick];
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      const double uc = fabs(0.5 * (u[c] + hi_face(F, 0, u, brick, l, loc)));
      const double vc = fabs(0.5 * (v[c] + hi_face(F, 1, v, brick, l, loc)));
      const double wc = fabs(0.5 * (w[c] + hi_face(F, 2, w, brick, l, loc)));
      const double inv = uc / F.h[lev][0] + vc / F.h[lev][1] + wc / F.h[lev][2] + visc_of(lev);
      m[0] = fmax(m[0], inv);
    }
  grid_reduce<1, 1u>(m, rb, [=] __device__(const double* t) {
    out->maxinv = t[0];
    if (dt_out) *dt_out = cfl / t[0];
  });
}

// Cell-centred values at points on an octree: the leaf cell containing the
// point (finest level first; indices truncated toward zero and clamped into
// the domain), then the average of its two a-faces (NSSolver::cellU/V/W,
// ns_solver.cpp:677-688, on that cell) or its pressure.
__global__ void k_amr_sample(AmrFlowView F, int comp, long long n, const double* __restrict__ xyz,
                             const double* __restrict__ u, const double* __restrict__ v,
                             const double* __restrict__ w, const double* __restrict__ p, double* __restrict__ out) {
  const LevelView& L = F.L;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    int brick = -1, loc[3] = {0, 0, 0};
    for (int lev = L.nlev - 1; lev >= 0 && brick < 0; --lev) {
      int c[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int N = L.lcells[lev][a];
        const double d = fmin(fmax((xyz[3 * q + a] - F.origin[a]) / F.h[lev][a], -1.0), static_cast<double>(N));
        c[a] = min(max(static_cast<int>(d), 0), N - 1);
      }
      brick = lut_at(L, lev, c[0] >> 3, c[1] >> 3, c[2] >> 3);
      for (int a = 0; a < 3; ++a) loc[a] = c[a] & 7;
    }
    double val = 0.0;
    if (brick >= 0) {
      const int l = (loc[2] << 6) | (loc[1] << 3) | loc[0];
      const long long cell = brick * static_cast<long long>(BR3) + l;
      if (comp < 3) {
        const double* f = comp == 0 ? u : (comp == 1 ? v : w);
        val = 0.5 * (f[cell] + hi_face(F, comp, f, brick, l, loc));
      } else {
        val = p[cell];
      }
    }
    out[q] = val;
  }
}

// Per-brick refinement sensors, the velocity-gradient sensors of
// PhysicalSensorEvaluator::evaluate (core/src/adaptive/adaptive_core.cpp:
// 96-113) on brick cells: cell-centred u, v, w, p; gradients by central
// differences inside the brick (one-sided on its faces); per brick the
// maximum over fluid cells of |omega|, sqrt(2 S:S), Q = (O:O - S:S)/2 and
// |grad p| (0 for a brick without fluid cells).
__global__ void __launch_bounds__(NT) k_amr_sensors(AmrFlowView F, const double* __restrict__ u,
                                                    const double* __restrict__ v, const double* __restrict__ w,
                                                    const double* __restrict__ p, double* __restrict__ out) {
  __shared__ double cv[4][BR3];
  __shared__ double sh[4 * 32];
  const LevelView& L = F.L;
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int lev = L.blevel[brick];
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      const long long c = brick * static_cast<long long>(BR3) + l;
      cv[0][l] = 0.5 * (u[c] + hi_face(F, 0, u, brick, l, loc));
      cv[1][l] = 0.5 * (v[c] + hi_face(F, 1, v, brick, l, loc));
      cv[2][l] = 0.5 * (w[c] + hi_face(F, 2, w, brick, l, loc));
      cv[3][l] = p[c];
    }
    __syncthreads();
    double best[4] = {-1.0e308, -1.0e308, -1.0e308, -1.0e308};
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      if (L.type[brick * static_cast<long long>(BR3) + l] != CELL_FLUID) continue;
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      double g[4][3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int st = d == 0 ? 1 : (d == 1 ? 8 : 64);
        const double h = F.h[lev][d];
        const int lo = loc[d] == 0 ? l : l - st, hi = loc[d] == 7 ? l : l + st;
        const double span = (loc[d] == 0 || loc[d] == 7) ? h : 2.0 * h;
#pragma unroll
        for (int f = 0; f < 4; ++f) g[f][d] = (cv[f][hi] - cv[f][lo]) / span;
      }
      const double* du = g[0];
      const double* dv = g[1];
      const double* dw = g[2];
      const double ox = dw[1] - dv[2], oy = du[2] - dw[0], oz = dv[0] - du[1];
      const double vort = sqrt(ox * ox + oy * oy + oz * oz);
      const double sxy = 0.5 * (du[1] + dv[0]), sxz = 0.5 * (du[2] + dw[0]), syz = 0.5 * (dv[2] + dw[1]);
      const double ss = du[0] * du[0] + dv[1] * dv[1] + dw[2] * dw[2] + 2 * (sxy * sxy + sxz * sxz + syz * syz);
      const double axy = 0.5 * (du[1] - dv[0]), axz = 0.5 * (du[2] - dw[0]), ayz = 0.5 * (dv[2] - dw[1]);
      const double oo = 2 * (axy * axy + axz * axz + ayz * ayz);
      const double gp = sqrt(g[3][0] * g[3][0] + g[3][1] * g[3][1] + g[3][2] * g[3][2]);
      const double val[4] = {vort, sqrt(2.0 * ss), 0.5 * (oo - ss), gp};
#pragma unroll
      for (int k = 0; k < 4; ++k) best[k] = fmax(best[k], val[k]);
    }
    block_reduce<4, 0xFu>(best, sh);
    if (threadIdx.x == 0)
      for (int k = 0; k < 4; ++k) out[4LL * brick + k] = best[k] < -1.0e300 ? 0.0 : best[k];
    __syncthreads();
  }
}

// State transfer between two meshes of one geometry whose levels differ by
// at most one everywhere (one regrid pass). Every face the destination stores
// takes the source's value at that face through the level-aware face rule
// (same level: the face; finer source: the average of its four sub-faces;
// coarser source: the coarse face, or the midpoint of the coarse cell's two
// normal faces), which keeps a discretely divergence-free field free of
// divergence; cells take the same-level value, the coarser cell's value, or
// the mean of their eight finer cells.
__global__ void k_amr_transfer_faces(AmrFlowView D, AmrFlowView S, int a, const int* __restrict__ dslab_brick,
                                     long long nslot, const double* __restrict__ fsrc, double* __restrict__ fdst) {
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < nslot;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    int brick, loc[3];
    if (q < D.nb) {
      brick = static_cast<int>(q >> 9);
      const int l = static_cast<int>(q & 511);
      loc[0] = l & 7;
      loc[1] = (l >> 3) & 7;
      loc[2] = l >> 6;
    } else {  // high slab face: the inverse of slab_local
      const long long r = q - D.nb;
      const int m = static_cast<int>(r & 63);
      brick = dslab_brick[r >> 6];
      loc[a] = 8;
      loc[a == 0 ? 1 : 0] = m & 7;
      loc[a == 2 ? 1 : 2] = m >> 3;
    }
    const int lev = D.L.blevel[brick];
    const int pos[3] = {D.L.bcoord[3 * brick] * BR + loc[0], D.L.bcoord[3 * brick + 1] * BR + loc[1],
                        D.L.bcoord[3 * brick + 2] * BR + loc[2]};
    fdst[q] = face_read(S, a, fsrc, lev, pos);
  }
}

__global__ void k_amr_transfer_cells(AmrFlowView D, AmrFlowView S, const double* __restrict__ psrc,
                                     double* __restrict__ pdst) {
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < D.nb;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int brick = static_cast<int>(q >> 9), l = static_cast<int>(q & 511);
    const int lev = D.L.blevel[brick];
    const int pos[3] = {D.L.bcoord[3 * brick] * BR + (l & 7), D.L.bcoord[3 * brick + 1] * BR + ((l >> 3) & 7),
                        D.L.bcoord[3 * brick + 2] * BR + (l >> 6)};
    int ls = -1;
    const int r = leaf_of(S.L, lev, pos, ls);
    double val = 0.0;
    if (r >= 0 && ls == lev) {
      val = psrc[r * static_cast<long long>(BR3) + local_of(pos)];
    } else if (r >= 0 && ls == lev - 1) {
      const int cp[3] = {pos[0] >> 1, pos[1] >> 1, pos[2] >> 1};
      val = psrc[r * static_cast<long long>(BR3) + local_of(cp)];
    } else if (r >= 0 && ls == lev + 1) {
      double sum = 0.0;
      for (int d = 0; d < 8; ++d) {
        const int ch[3] = {2 * pos[0] + (d & 1), 2 * pos[1] + ((d >> 1) & 1), 2 * pos[2] + (d >> 2)};
        sum += psrc[r * static_cast<long long>(BR3) + local_of(ch)];
      }
      val = 0.125 * sum;
    }
    pdst[q] = val;
  }
}

}  // namespace

void amr_flow_setup() {
  NB_CUDA(cudaFuncSetAttribute(k_amr_rhs_rk<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               3 * TN * static_cast<int>(sizeof(double))));
  NB_CUDA(cudaFuncSetAttribute(k_amr_rhs_rk<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               3 * TN * static_cast<int>(sizeof(float))));
}

void launch_ghost_count(cudaStream_t s, const AmrFlowView& F, int* count) {
  k_ghost_map<<<grid_for(F.L.nbrick), RHS_NT, 0, s>>>(F, count);
  NB_CUDA(cudaGetLastError());
}

void launch_ghost_fill(cudaStream_t s, const AmrFlowView& F, const int* eoff, const int* toff, uint2* ent,
                       int2* term) {
  k_ghost_fill<<<grid_for(F.L.nbrick), RHS_NT, 0, s>>>(F, eoff, toff, ent, term);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_rhs_rk(cudaStream_t s, const AmrFlowView& F, int stage, const double* dtp, const double* u,
                       const double* v, const double* w, const double* u0, const double* v0,
                       const double* w0, double* uo, double* vo, double* wo, int mixed, int grid_cap) {
  const int grid = std::min(F.L.nbrick, std::max(grid_cap, 1));
  if (mixed)
    k_amr_rhs_rk<float><<<grid, RHS_NT, 3 * TN * sizeof(float), s>>>(F, stage, dtp, u, v, w, u0, v0, w0, uo, vo,
                                                                     wo);
  else
    k_amr_rhs_rk<double><<<grid, RHS_NT, 3 * TN * sizeof(double), s>>>(F, stage, dtp, u, v, w, u0, v0, w0, uo,
                                                                       vo, wo);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_sync(cudaStream_t s, const long long* list, int n, double* f) {
  if (n <= 0) return;
  k_amr_sync<<<std::min((n + 255) / 256, 1024), 256, 0, s>>>(list, n, f);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_div(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v, const double* w,
                    double* b) {
  k_amr_div<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, b);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_correct(cudaStream_t s, const AmrFlowView& F, const double* phi, const double* dtp,
                        double* u, double* v, double* w, double* p) {
  k_amr_correct<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, phi, dtp, u, v, w, p);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_diag(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v,
                     const double* w, const double* u0, const double* v0, const double* w0, RedBuf rb,
                     AmrStepScalars* out) {
  k_amr_diag<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, u0, v0, w0, rb, out);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_sample(cudaStream_t s, const AmrFlowView& F, int comp, long long n, const double* xyz,
                       const double* u, const double* v, const double* w, const double* p, double* out) {
  if (n <= 0) return;
  const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, 148 * 8));
  k_amr_sample<<<grid, 256, 0, s>>>(F, comp, n, xyz, u, v, w, p, out);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_sensors(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v, const double* w,
                        const double* p, double* out) {
  k_amr_sensors<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, p, out);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_transfer(cudaStream_t s, const AmrFlowView& D, const AmrFlowView& S, const int* const dslab[3],
                         const long long nstore[3], const double* const fsrc[3], double* const fdst[3],
                         const double* psrc, double* pdst) {
  for (int a = 0; a < 3; ++a) {
    const int grid = static_cast<int>(std::min<long long>((nstore[a] + 255) / 256, 148 * 8));
    k_amr_transfer_faces<<<grid, 256, 0, s>>>(D, S, a, dslab[a], nstore[a], fsrc[a], fdst[a]);
    NB_CUDA(cudaGetLastError());
  }
  const int grid = static_cast<int>(std::min<long long>((D.nb + 255) / 256, 148 * 8));
  k_amr_transfer_cells<<<grid, 256, 0, s>>>(D, S, psrc, pdst);
  NB_CUDA(cudaGetLastError());
}

void launch_amr_max_inv(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v,
                        const double* w, double cfl, double* dt_out, RedBuf rb, AmrStepScalars* out) {
  k_amr_max_inv<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, cfl, dt_out, rb, out);
  NB_CUDA(cudaGetLastError());
}

}  // namespace nb
