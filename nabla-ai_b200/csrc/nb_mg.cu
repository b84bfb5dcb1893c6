// nb_mg.cu — sm_100a kernels and host driver of the MG-PCG pressure solve.
//
// Bandwidth-bound stencils on bricks: one 512-thread CTA walks bricks
// (grid-stride), thread t owns cell t of the brick. No tensor cores (the
// operator is a 7-point stencil, not a dense contraction).
//
// Reference arithmetic followed (paths within the reference project):
//   stencil / diagonal     core/src/flow/poisson.cpp:18-134
//   smooth / removeMean    core/src/flow/multigrid.cpp:81-114
//   residual + restrict    core/src/flow/multigrid.cpp:116-154
//   prolongAdd             core/src/flow/multigrid.cpp:158-173
//   vcycle                 core/src/flow/multigrid.cpp:175-194
//   coarsest CgPoisson     core/src/flow/poisson.cpp:136-252
//   flexible PCG           core/src/flow/multigrid.cpp:268-355
#include <algorithm>
#include <cmath>
#include <cstring>

#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "nb_mg.cuh"
#include "nb_reduce.cuh"

namespace nb {

namespace cg = cooperative_groups;

namespace {

constexpr int NT = 512;          // threads per CTA = cells per brick
constexpr int MAX_GRID = 148 * 16;  // grid-stride CTA cap (16 CTAs of 128 per SM)
constexpr double kOmega = 0.8;   // multigrid.cpp:38
constexpr int COARSE_MAX_CELLS = 4096;
constexpr int COARSE_PRE_CELLS = 2048;  // coarsest levels up to this size keep a resolved stencil

// Dynamic shared memory of the coarsest-level CTA for n cells.
inline size_t coarse_smem(size_t n) {
  return n * (6 * sizeof(double) + 1) + (n <= static_cast<size_t>(COARSE_PRE_CELLS) ? n * 6 * sizeof(int16_t) : 0);
}

__device__ __forceinline__ bool stopped(const SolveFlags* f, int maxit) {
  return f != nullptr && (f->stop != 0 || f->iters >= maxit);
}

// Value of a level vector at an (in-grid, fluid) cell after the operations
// still pending on it: the lazy removeMean (x - mean) and the lazy
// prolongAdd (+ e[parent], itself with the coarse level's pending mean).
//
// CV is how the coarse level is held (by value in kernel parameters, or as a
// pointer into shared memory in the cluster tail); ACC is how level vectors
// are addressed (global memory, or distributed over a cluster's shared memory).
__device__ __forceinline__ const LevelView& lv_of(const LevelView& v) { return v; }
__device__ __forceinline__ const LevelView& lv_of(const LevelView* v) { return *v; }
template <bool CG, typename T>
__device__ __forceinline__ T ldv(const T* p) {
  if constexpr (CG) return __ldcg(p);
  else return *p;
}
// Level vectors in global memory.
struct GAcc {
  static constexpr bool kCG = false;  // pending means: plain loads
  template <typename T>
  __device__ __forceinline__ T ld(const T* p, int n) const { return p[n]; }
  template <typename T>
  __device__ __forceinline__ void st(T* p, int n, T v) const { p[n] = v; }
};
// BF16 storage of a coarse level's restricted residual (mixed form, optional):
// the value is rounded to nearest on the store and widened on the load; BF16
// keeps FP32's 8-bit exponent, so no scaling is needed for range.
template <typename T>
__device__ __forceinline__ T ld_b16(const T* p, int n) {
  return static_cast<T>(__bfloat162float(reinterpret_cast<const __nv_bfloat16*>(p)[n]));
}
template <typename T>
__device__ __forceinline__ T st_b16(T* p, int n, T v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(static_cast<float>(v));
  reinterpret_cast<__nv_bfloat16*>(p)[n] = h;
  return static_cast<T>(__bfloat162float(h));
}
// Level vectors distributed over the shared memory of a thread-block
// cluster: brick g of a vector lives in CTA g mod cs at slot g / cs of the
// vector's array, and a vector "pointer" is that array's byte offset in every
// CTA's arena plus kArenaBias (so that no vector encodes as null).
constexpr uintptr_t kArenaBias = 128;
struct DAcc {
  static constexpr bool kCG = true;  // pending means (global) are written inside the launch
  char* arena;                       // this CTA's arena
  int lcs;                           // log2 of the cluster size
  template <typename T>
  __device__ __forceinline__ T* at(const T* p, int n) const {
    const int g = n >> 9;
    T* local = reinterpret_cast<T*>(arena + (reinterpret_cast<uintptr_t>(p) - kArenaBias)) + ((g >> lcs) << 9) +
               (n & 511);
    return cg::this_cluster().map_shared_rank(local, static_cast<unsigned>(g & ((1 << lcs) - 1)));
  }
  template <typename T>
  __device__ __forceinline__ T ld(const T* p, int n) const { return *at(p, n); }
  template <typename T>
  __device__ __forceinline__ void st(T* p, int n, T v) const { *at(p, n) = v; }
};

template <typename T, class CV = LevelView, class ACC = GAcc>
struct XFetchT {
  const T* x;            // nullptr => the vector is identically zero
  const double* xmean;   // pending mean (nullptr => none)
  const T* ec;           // pending prolongation source (nullptr => none)
  const double* ecmean;  // pending mean of ec
  CV C;                  // coarse level (for parent lookup)
  int fx, fy, fz;
  const int* xfb = nullptr;  // composite fine level: parent brick per brick
  const int* xfo = nullptr;  // composite fine level: octant in the parent (-1 kept)
  ACC acc{};
  __device__ __forceinline__ int parent(int n, int gi, int gj, int gk) const {
    if (xfb) {
      const int b = n >> 9, l = n & 511, oct = xfo[b];
      if (oct < 0) return xfb[b] * BR3 + l;
      const int ci = (oct & 1) * 4 + ((l & 7) >> 1), cj = ((oct >> 1) & 1) * 4 + (((l >> 3) & 7) >> 1),
                ck = (oct >> 2) * 4 + ((l >> 6) >> 1);
      return xfb[b] * BR3 + ((ck << 6) | (cj << 3) | ci);
    }
    return cell_index(lv_of(C), gi / fx, gj / fy, gk / fz);
  }
  __device__ __forceinline__ T operator()(int n, int gi, int gj, int gk) const {
    T v = x ? acc.ld(x, n) : T(0);
    if (xmean) v = v - static_cast<T>(ldv<ACC::kCG>(xmean));
    if (ec) {
      T e = acc.ld(ec, parent(n, gi, gj, gk));
      if (ecmean) e = e - static_cast<T>(ldv<ACC::kCG>(ecmean));
      v = v + e;
    }
    return v;
  }
  __device__ __forceinline__ bool prolongs() const { return ec != nullptr; }
  // The same value for the one-round staging: the parent of cell n lies in
  // brick pb of the coarser level at octant po (-1: cell for cell); composite
  // levels merge by 2 on every axis, uniform levels by fx, fy, fz.
  __device__ __forceinline__ T at(int n, int pb, int po, int amr) const {
    T v = x ? acc.ld(x, n) : T(0);
    if (xmean) v = v - static_cast<T>(ldv<ACC::kCG>(xmean));
    if (ec) {
      const int l = n & 511;
      int pl = l;
      if (po >= 0) {
        const int li = l & 7, lj = (l >> 3) & 7, lk = l >> 6;
        const int ci = (amr || fx == 2) ? ((po & 1) << 2) + (li >> 1) : li;
        const int cj = (amr || fy == 2) ? (((po >> 1) & 1) << 2) + (lj >> 1) : lj;
        const int ck = (amr || fz == 2) ? (((po >> 2) & 1) << 2) + (lk >> 1) : lk;
        pl = (ck << 6) | (cj << 3) | ci;
      }
      T e = acc.ld(ec, pb * BR3 + pl);
      if (ecmean) e = e - static_cast<T>(ldv<ACC::kCG>(ecmean));
      v = v + e;
    }
    return v;
  }
};
template <typename T>
using XFetch = XFetchT<T>;

__device__ __forceinline__ double cell_weight(const LevelView& L, int brick) {
  return L.amr ? L.bweight[brick] : 1.0;
}

// Row of the -Laplacian at fluid cell (gi,gj,gk): returns diag (raw sum of
// face coefficients) and off = sum coeff * x[n] in the reference's order
// (axis 0 side -1, +1, axis 1, axis 2).
template <typename T, class F>
__device__ __forceinline__ void stencil_row(const LevelView& L, int gi, int gj, int gk, const F& fx,
                                            T& diag, T& off) {
  diag = T(0);
  off = T(0);
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    if (axis == 2 && L.twoD) continue;
    const T h2 = static_cast<T>(L.h2[axis]);
#pragma unroll
    for (int side = -1; side <= 1; side += 2) {
      int n = 0;
      const int kind = resolve_face(L, gi, gj, gk, axis, side, n);
      if (kind == 1) {
        int c[3] = {gi, gj, gk};
        const int dims[3] = {L.nx, L.ny, L.nz};
        c[axis] = wrapi(c[axis] + side, dims[axis]);
        diag += h2;
        off += h2 * fx(n, c[0], c[1], c[2]);
      } else if (kind == 2) {
        diag += T(2) * h2;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Shared-memory halo staging. A CTA works on one brick at a time: it stages
// the brick's 8^3 values plus the one-cell face halo from the six neighbour
// bricks (10^3 positions minus edges and corners, which a 7-point stencil
// never reads), applying the vector's pending operations on the way in, then
// every cell evaluates its row from shared memory with its precomputed code.
// ---------------------------------------------------------------------------
constexpr int TS = 10;
constexpr int TSN = TS * TS * TS;

__device__ __forceinline__ int tpos(int i, int j, int k) { return ((k + 1) * TS + (j + 1)) * TS + (i + 1); }
__device__ __forceinline__ int tpos_local(int l) { return tpos(l & 7, (l >> 3) & 7, l >> 6); }
__device__ __forceinline__ int code_type(uint32_t code) { return (code >> CODE_TYPE) & 3; }

template <typename T, class F>
__device__ __forceinline__ void fill_halo_amr(const LevelView& L, int brick, T* tile, const F& fx) {
  const int lev = L.blevel[brick];
  const int ox = L.bcoord[3 * brick] * BR, oy = L.bcoord[3 * brick + 1] * BR,
            oz = L.bcoord[3 * brick + 2] * BR;
  const int dims[3] = {L.lcells[lev][0], L.lcells[lev][1], L.lcells[lev][2]};
  for (int p = threadIdx.x; p < TSN; p += blockDim.x) {
    const int ti = p % TS - 1, tj = (p / TS) % TS - 1, tk = p / (TS * TS) - 1;
    const int outc = (ti < 0 || ti > 7) + (tj < 0 || tj > 7) + (tk < 0 || tk > 7);
    if (outc > 1) continue;
    int g[3] = {ox + ti, oy + tj, oz + tk};
    T v = T(0);
    if (outc == 0) {
      v = fx(brick * BR3 + ((tk << 6) | (tj << 3) | ti), g[0], g[1], g[2]);
    } else {
      bool ok = true;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (g[a] < 0 || g[a] >= dims[a]) {
          if (L.bc[2 * a] == NB_BC_PERIODIC) g[a] = wrapi(g[a], dims[a]);
          else ok = false;
        }
      if (ok) {
        // same-level neighbour only; other halo cells are never read
        const int nb = L.lut[L.lut_off[lev] + ((g[2] >> 3) * L.lnb[lev][1] + (g[1] >> 3)) * L.lnb[lev][0] +
                             (g[0] >> 3)];
        if (nb >= 0) v = fx(nb * BR3 + (((g[2] & 7) << 6) | ((g[1] & 7) << 3) | (g[0] & 7)), g[0], g[1], g[2]);
      }
    }
    tile[p] = v;
  }
}

// Static maps of the brick a CTA stages next, in shared memory: the six face
// neighbours, for a pending prolongation the parent brick and octant of the
// brick and of each neighbour, and on a composite restriction the coarse
// brick, octant and weight its residual goes to. The maps are never written
// during a solve, so a kernel reads its first brick's before pdl_wait() (a CTA
// that becomes resident while its predecessor grid drains has them before the
// wait returns, and its halo loads then depend on no further map load) and
// each later brick's during the previous brick's arithmetic, right after that
// brick's staging barrier. Two records alternate by iteration parity: a
// brick's record is still read after its first barrier (the restriction's
// coarse target) while the next brick's is being written.
struct BrickPre {
  int pb, po, xcb, xoct;
  double wc;
  int nb[6], npb[6], npo[6];
};

__device__ __forceinline__ void prefetch_brick(const LevelView& L, int brick, bool pro, BrickPre& P,
                                               const LevelView* C = nullptr) {
  const int t = threadIdx.x;
  if (brick >= L.nbrick) return;
  if (L.fast && t < 6) {
    P.nb[t] = L.nbr6[brick * 6 + t];
    P.npb[t] = pro ? L.npar6[brick * 6 + t] : 0;
    P.npo[t] = pro ? L.npoct6[brick * 6 + t] : -1;
  } else if (L.fast && t == 6) {
    P.pb = pro ? L.par[brick] : 0;
    P.po = pro ? L.poct[brick] : -1;
  } else if (t == 7 && C && L.amr) {
    P.xcb = L.xf_brick[brick];
    P.xoct = L.xf_oct[brick];
    P.wc = C->amr ? C->bweight[P.xcb] : 1.0;
  }
}

// The loads of fill_halo_fast into registers (the brick's own values and its
// face halo), and their stores into the tile: split so that a CTA can have the
// next brick's loads in flight while it computes the current one.
template <typename T, int NTH, class F>
__device__ __forceinline__ void halo_load(const LevelView& L, int brick, const F& fx, T* own, T* halo, int* hpos) {
  constexpr int CPT = BR3 / NTH;
  constexpr int HPT = (384 + NTH - 1) / NTH;
  const int t = threadIdx.x;
  const bool pro = fx.prolongs();
  const int pb = pro ? L.par[brick] : 0, po = pro ? L.poct[brick] : -1;
#pragma unroll
  for (int q = 0; q < CPT; ++q) own[q] = fx.at(brick * BR3 + t + q * NTH, pb, po, L.amr);
#pragma unroll
  for (int q = 0; q < HPT; ++q) {
    const int h = t + q * NTH;
    halo[q] = T(0);
    hpos[q] = -1;
    if (h < 384) {
      // face f = 2a + s, position (u, w) on it: the tile position just outside
      // the brick and the facing cell of the neighbour brick (the two
      // tangential axes take u then w, in increasing axis order); selects
      // rather than arrays indexed by a, which would live in local memory
      const int f = h >> 6, m = h & 63, u = m & 7, w = m >> 3, a = f >> 1, s = f & 1;
      const int et = s ? 8 : -1, el = s ? 0 : 7;
      const int ti = a == 0 ? et : u, tj = a == 1 ? et : (a == 0 ? u : w), tk = a == 2 ? et : w;
      const int li = a == 0 ? el : u, lj = a == 1 ? el : (a == 0 ? u : w), lk = a == 2 ? el : w;
      hpos[q] = tpos(ti, tj, tk);
      const int nb = L.nbr6[brick * 6 + f];
      if (nb >= 0) {
        const int npb = pro ? L.npar6[brick * 6 + f] : 0, npo = pro ? L.npoct6[brick * 6 + f] : -1;
        halo[q] = fx.at(nb * BR3 + ((lk << 6) | (lj << 3) | li), npb, npo, L.amr);
      }
    }
  }
}

template <typename T, int NTH>
__device__ __forceinline__ void halo_store(T* tile, const T* own, const T* halo, const int* hpos) {
  constexpr int CPT = BR3 / NTH;
  constexpr int HPT = (384 + NTH - 1) / NTH;
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < CPT; ++q) tile[tpos_local(t + q * NTH)] = own[q];
#pragma unroll
  for (int q = 0; q < HPT; ++q)
    if (hpos[q] >= 0) tile[hpos[q]] = halo[q];
}

// One-round staging (levels with per-brick maps): a CTA of NTH threads loads
// the brick's 512 cells (512/NTH per thread) and the 384 face-halo cells from
// the six neighbour bricks (6 faces x 64). Every load is issued before the
// first store to shared memory, so all of them are in flight together.
template <typename T, int NTH, class F>
__device__ __forceinline__ void fill_halo_fast(const LevelView& L, int brick, T* tile, const F& fx,
                                               const BrickPre* pre = nullptr) {
  constexpr int CPT = BR3 / NTH;
  constexpr int HPT = (384 + NTH - 1) / NTH;
  const int t = threadIdx.x;
  const bool pro = fx.prolongs();
  const int pb = pre ? pre->pb : (pro ? L.par[brick] : 0), po = pre ? pre->po : (pro ? L.poct[brick] : -1);
  T own[CPT];
#pragma unroll
  for (int q = 0; q < CPT; ++q) own[q] = fx.at(brick * BR3 + t + q * NTH, pb, po, L.amr);
  T halo[HPT];
  int hpos[HPT];
#pragma unroll
  for (int q = 0; q < HPT; ++q) {
    const int h = t + q * NTH;
    halo[q] = T(0);
    hpos[q] = -1;
    if (h < 384) {
      // face f = 2a + s, position (u, w) on it: the tile position just outside
      // the brick and the facing cell of the neighbour brick (the two
      // tangential axes take u then w, in increasing axis order); selects
      // rather than arrays indexed by a, which would live in local memory
      const int f = h >> 6, m = h & 63, u = m & 7, w = m >> 3, a = f >> 1, s = f & 1;
      const int et = s ? 8 : -1, el = s ? 0 : 7;
      const int ti = a == 0 ? et : u, tj = a == 1 ? et : (a == 0 ? u : w), tk = a == 2 ? et : w;
      const int li = a == 0 ? el : u, lj = a == 1 ? el : (a == 0 ? u : w), lk = a == 2 ? el : w;
      hpos[q] = tpos(ti, tj, tk);
      const int nb = pre ? pre->nb[f] : L.nbr6[brick * 6 + f];
      if (nb >= 0) {
        const int npb = pre ? pre->npb[f] : (pro ? L.npar6[brick * 6 + f] : 0);
        const int npo = pre ? pre->npo[f] : (pro ? L.npoct6[brick * 6 + f] : -1);
        halo[q] = fx.at(nb * BR3 + ((lk << 6) | (lj << 3) | li), npb, npo, L.amr);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < CPT; ++q) tile[tpos_local(t + q * NTH)] = own[q];
#pragma unroll
  for (int q = 0; q < HPT; ++q)
    if (hpos[q] >= 0) tile[hpos[q]] = halo[q];
}

// Stages brick `brick` of L into `tile`; NTH is the CTA's thread count.
template <typename T, int NTH = NT, class F>
__device__ __forceinline__ void fill_halo(const LevelView& L, int brick, T* tile, const F& fx,
                                          const BrickPre* pre = nullptr) {
  if (L.fast) {
    fill_halo_fast<T, NTH>(L, brick, tile, fx, pre);
    return;
  }
  if (L.amr) {
    fill_halo_amr<T>(L, brick, tile, fx);
    return;
  }
  const int ox = L.bcoord[3 * brick] * BR, oy = L.bcoord[3 * brick + 1] * BR,
            oz = L.bcoord[3 * brick + 2] * BR;
  const int dims[3] = {L.nx, L.ny, L.nz};
  for (int p = threadIdx.x; p < TSN; p += blockDim.x) {
    const int ti = p % TS - 1, tj = (p / TS) % TS - 1, tk = p / (TS * TS) - 1;
    const int outc = (ti < 0 || ti > 7) + (tj < 0 || tj > 7) + (tk < 0 || tk > 7);
    if (outc > 1) continue;
    int g[3] = {ox + ti, oy + tj, oz + tk};
    T v = T(0);
    if (outc == 0 && g[0] < dims[0] && g[1] < dims[1] && g[2] < dims[2]) {
      v = fx(brick * BR3 + ((tk << 6) | (tj << 3) | ti), g[0], g[1], g[2]);
    } else {
      bool ok = true;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (g[a] < 0 || g[a] >= dims[a]) {
          if (L.bc[2 * a] == NB_BC_PERIODIC) g[a] = wrapi(g[a], dims[a]);
          else ok = false;
        }
      if (ok) v = fx(cell_index(L, g[0], g[1], g[2]), g[0], g[1], g[2]);
    }
    tile[p] = v;
  }
}

// Row of the -Laplacian from the staged tile: diag = sum of face coefficients,
// off = sum coeff * neighbour, faces in the reference's order (poisson.cpp:114-129).
template <typename T>
__device__ __forceinline__ void row_from_tile(const LevelView& L, uint32_t code, const T* tile, int ctr,
                                              T& diag, T& off, int lev = 0) {
  diag = T(0);
  off = T(0);
  const int step[6] = {-1, 1, -TS, TS, -TS * TS, TS * TS};
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const T h2 = static_cast<T>(L.amr ? L.lh2[lev][f >> 1] : L.h2[f >> 1]);
    if (code & (1u << f)) {
      diag += h2;
      off += h2 * tile[ctr + step[f]];
    } else if (code & (1u << (CODE_DIRICHLET + f))) {
      diag += T(2) * h2;
    }
  }
}

// Coarse-fine couplings of a composite-level cell (added after the six
// same-level faces): coefficient c with neighbour value x_n.
template <typename T, class F>
__device__ __forceinline__ void add_cf(const LevelView& L, uint32_t code, int c, const F& fx, T& diag, T& off) {
  if (!(code & (1u << CODE_HASCF))) return;
  for (int q = L.cf_off[c]; q < L.cf_off[c + 1]; ++q) {
    const T coef = static_cast<T>(L.cf_coef[q]);
    diag += coef;
    off += coef * fx(L.cf_nbr[q], 0, 0, 0);
  }
}

// Full row: same-level faces from the tile, then coarse-fine couplings.
template <typename T, class F>
__device__ __forceinline__ void full_row(const LevelView& L, uint32_t code, const T* tile, int brick, int c,
                                         const F& fx, T& diag, T& off) {
  const int lev = L.amr ? L.blevel[brick] : 0;
  row_from_tile<T>(L, code, tile, tpos_local(c & 511), diag, off, lev);
  if (L.amr) add_cf<T>(L, code, c, fx, diag, off);
}

// ---------------------------------------------------------------------------
// Damped-Jacobi sweep (multigrid.cpp:102-114), one sweep per launch.
//   xout = fluid ? x' + c2 (b' - A x') / D + c1 (x' - x_prev) : 0
// where x' / b' include pending mean / prolongation. c2 = omega, c1 = 0 is the
// reference's Jacobi (prev_mode 0); the mixed form may run a Chebyshev
// polynomial instead, whose later sweeps add c1 times the last step: x_prev
// is 0 (prev_mode 2, the first step of a phase from x = 0) or the previous
// iterate as P fetches it at the cell (prev_mode 1: its buffer is xout's,
// read before it is overwritten, with its pending mean and prolongation).
// Optionally reduces the fluid sum of xout into `mean_out` (= sum / nfluid)
// for the next removeMean.
// ---------------------------------------------------------------------------
// Where a sweep's result goes: xout (addressed by acc) and this thread's part
// of the weighted fluid sum for the next removeMean.
template <typename T, class ACC>
struct SweepOut {
  T* xout;
  const ACC& acc;
  double part = 0.0;
  __device__ __forceinline__ void operator()(int c, double wgt, T out, bool fluid) {
    if (fluid) part += wgt * static_cast<double>(out);
    acc.st(xout, c, out);
  }
};

// One cell of a sweep: xout = fluid ? x' + c2 (b' - A x') / D + c1 (x' - x_prev) : 0.
template <typename T, class ACC, class FX, class FP>
__device__ __forceinline__ T sweep_cell(const LevelView& L, int brick, int l, uint32_t code, T bc, const double* bmean,
                                        const FX& X, T c2, T c1, int prev_mode, const FP& P, const T* tile,
                                        bool staged, bool& fluid) {
  const int c = brick * BR3 + l;
  T out = T(0);
  fluid = code_type(code) == CELL_FLUID;
  if (fluid) {
    T diag, off, xc;
    if (staged) {
      full_row<T>(L, code, tile, brick, c, X, diag, off);
      xc = tile[tpos_local(l)];
    } else {  // first sweep from x = 0: A x = 0
      const int lev = L.amr ? L.blevel[brick] : 0;
      diag = T(0);
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const T h2 = static_cast<T>(L.amr ? L.lh2[lev][f >> 1] : L.h2[f >> 1]);
        if (code & (1u << f)) diag += h2;
        else if (code & (1u << (CODE_DIRICHLET + f))) diag += T(2) * h2;
      }
      if (L.amr && (code & (1u << CODE_HASCF)))
        for (int k = L.cf_off[c]; k < L.cf_off[c + 1]; ++k) diag += static_cast<T>(L.cf_coef[k]);
      off = T(0);
      xc = T(0);
    }
    if (bmean) bc = bc - static_cast<T>(ldv<ACC::kCG>(bmean));
    const T Ax = diag * xc - off;
    const T dM = diag > T(0) ? diag : T(1);
    if constexpr (sizeof(T) == 4)  // FP32 smoother (a preconditioner): the fast division
      out = xc + c2 * __fdividef(bc - Ax, dM);
    else  // FP64: the reference's omega * r / diag
      out = xc + c2 * (bc - Ax) / dM;
    if (prev_mode) {
      T xp = T(0);
      if (prev_mode == 1) {
        int gi, gj, gk;
        cell_coords(L, c, gi, gj, gk);
        xp = P(c, gi, gj, gk);
      }
      out = out + c1 * (xc - xp);
    }
  }
  return out;
}

// Bricks first, first + stride, ... of one sweep; every cell's result goes
// to out(c, weight, value, fluid). `acc` addresses b. With PIPE (levels with
// per-brick maps and several bricks per CTA) the next brick's code, rhs, own
// and halo values are loaded while the current brick computes.
template <typename T, int NTH, class ACC, class FX, class FP, class OUT, bool PIPE = false>
__device__ __forceinline__ void smooth_bricks(const LevelView& L, const T* b, const double* bmean, const FX& X,
                                             OUT& sink, T c2, T c1, int prev_mode, const FP& P, int first,
                                             int stride, T* tile, const ACC& acc, int b16 = 0,
                                             BrickPre* pre = nullptr) {
  constexpr int CPT = BR3 / NTH;  // cells per thread
  constexpr int HPT = (384 + NTH - 1) / NTH;
  const bool staged = X.x || X.ec;
  if constexpr (PIPE) {
    if (staged && L.fast) {
      if (first >= L.nbrick) return;
      uint32_t code[CPT];
      T bv[CPT], own[CPT], halo[HPT];
      int hpos[HPT];
      const auto load = [&](int brick) {
#pragma unroll
        for (int q = 0; q < CPT; ++q) {
          const int c = brick * BR3 + threadIdx.x + q * NTH;
          code[q] = L.code[c];
          bv[q] = b16 ? ld_b16(b, c) : acc.ld(b, c);
        }
        halo_load<T, NTH>(L, brick, X, own, halo, hpos);
      };
      load(first);
      for (int brick = first;; brick += stride) {
        halo_store<T, NTH>(tile, own, halo, hpos);
        uint32_t cc[CPT];
        T cb[CPT];
#pragma unroll
        for (int q = 0; q < CPT; ++q) {
          cc[q] = code[q];
          cb[q] = bv[q];
        }
        __syncthreads();
        const bool more = brick + stride < L.nbrick;
        if (more) load(brick + stride);  // in flight during this brick's arithmetic
        const double wgt = cell_weight(L, brick);
#pragma unroll
        for (int q = 0; q < CPT; ++q) {
          const int l = threadIdx.x + q * NTH;
          bool fluid;
          const T out = sweep_cell<T, ACC>(L, brick, l, cc[q], cb[q], bmean, X, c2, c1, prev_mode, P, tile, true,
                                           fluid);
          sink(brick * BR3 + l, wgt, out, fluid);
        }
        __syncthreads();
        if (!more) return;
      }
    }
  }
  for (int brick = first, it = 0; brick < L.nbrick; brick += stride, ++it) {
    uint32_t code[CPT];
    T bv[CPT];
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int c = brick * BR3 + threadIdx.x + q * NTH;
      code[q] = L.code[c];
      bv[q] = b16 ? ld_b16(b, c) : acc.ld(b, c);
    }
    if (staged) fill_halo<T, NTH>(L, brick, tile, X, pre ? pre + (it & 1) : nullptr);
    __syncthreads();
    // the next brick's maps, in flight during this brick's arithmetic (the other record)
    if (pre) prefetch_brick(L, brick + stride, X.prolongs(), pre[(it + 1) & 1]);
    const double wgt = cell_weight(L, brick);
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int l = threadIdx.x + q * NTH;
      const int c = brick * BR3 + l;
      T out = T(0);
      const bool fluid = code_type(code[q]) == CELL_FLUID;
      if (fluid) {
        T diag, off, xc;
        if (staged) {
          full_row<T>(L, code[q], tile, brick, c, X, diag, off);
          xc = tile[tpos_local(l)];
        } else {  // first sweep from x = 0: A x = 0
          const int lev = L.amr ? L.blevel[brick] : 0;
          diag = T(0);
#pragma unroll
          for (int f = 0; f < 6; ++f) {
            const T h2 = static_cast<T>(L.amr ? L.lh2[lev][f >> 1] : L.h2[f >> 1]);
            if (code[q] & (1u << f)) diag += h2;
            else if (code[q] & (1u << (CODE_DIRICHLET + f))) diag += T(2) * h2;
          }
          if (L.amr && (code[q] & (1u << CODE_HASCF)))
            for (int k = L.cf_off[c]; k < L.cf_off[c + 1]; ++k) diag += static_cast<T>(L.cf_coef[k]);
          off = T(0);
          xc = T(0);
        }
        T bc = bv[q];
        if (bmean) bc = bc - static_cast<T>(ldv<ACC::kCG>(bmean));
        const T Ax = diag * xc - off;
        const T dM = diag > T(0) ? diag : T(1);
        if constexpr (sizeof(T) == 4)  // FP32 smoother (a preconditioner): the fast division
          out = xc + c2 * __fdividef(bc - Ax, dM);
        else  // FP64: the reference's omega * r / diag
          out = xc + c2 * (bc - Ax) / dM;
        if (prev_mode) {
          T xp = T(0);
          if (prev_mode == 1) {
            int gi, gj, gk;
            cell_coords(L, c, gi, gj, gk);
            xp = P(c, gi, gj, gk);
          }
          out = out + c1 * (xc - xp);
        }
      }
      sink(c, wgt, out, fluid);
    }
    __syncthreads();
  }
}

// Flexible beta of the PCG (multigrid.cpp:330-338) from t = {z'.rnew, z'.r}.
__device__ __forceinline__ void flex_beta(const double* t, double* S, SolveFlags* flags) {
  S[S_RNEWZ] = t[0];
  S[S_RZCROSS] = t[1];
  S[S_BETA] = (t[0] - t[1]) / S[S_RZ];
  S[S_RZ] = t[0];
  flags->iters += 1;
}

template <typename T, int NTH, bool PIPE>
__device__ __forceinline__ void smooth_launch(const LevelView& L, const T* __restrict__ b, const double* bmean,
                                              const XFetch<T>& X, T* xout, const RedBuf& rb, double* mean_out,
                                              double inv_nfluid, const SolveFlags* flags, int maxit, T c2, T c1,
                                              int prev_mode, const XFetch<T>& P, int b16) {
  __shared__ BrickPre pre[2];
  if (!PIPE) prefetch_brick(L, blockIdx.x, X.prolongs(), pre[0]);
  pdl_wait();
  __syncthreads();
  if (stopped(flags, maxit)) return;
  __shared__ T tile[TSN];
  const GAcc acc{};
  SweepOut<T, GAcc> sink{xout, acc};
  smooth_bricks<T, NTH, GAcc, XFetch<T>, XFetch<T>, SweepOut<T, GAcc>, PIPE>(
      L, b, bmean, X, sink, c2, c1, prev_mode, P, blockIdx.x, gridDim.x, tile, acc, b16, PIPE ? nullptr : pre);
  if (mean_out) {
    double part[1] = {sink.part};
    grid_reduce<1>(part, rb, [=] __device__(const double* t) { *mean_out = t[0] * inv_nfluid; });
  }
}

// CTAs an SM each sweep instantiation is built for, from its register budget
// (32 registers for FP32 at 512 threads, 40 for FP64): the bound also sizes
// the driver's shared-memory carveout for that many CTAs.
template <typename T, int NTH>
constexpr int sweep_ctas() {
  return NTH == 512 ? (sizeof(T) == 4 ? 4 : 3) : (NTH == 256 ? 5 : 8);
}

template <typename T, int NTH>
__global__ void __launch_bounds__(NTH, sweep_ctas<T, NTH>()) k_smooth(LevelView L, const T* __restrict__ b, const double* bmean,
                                                XFetch<T> X, T* xout, RedBuf rb, double* mean_out,
                                                double inv_nfluid, const SolveFlags* flags, int maxit, T c2, T c1,
                                                int prev_mode, XFetch<T> P, int b16) {
  smooth_launch<T, NTH, false>(L, b, bmean, X, xout, rb, mean_out, inv_nfluid, flags, maxit, c2, c1, prev_mode, P,
                               b16);
}

// The pipelined sweep (two bricks' loads in registers): 64 registers a thread,
// 1024 threads an SM. The bound also tells the driver to size the shared
// memory for that many CTAs; a bound of one CTA an SM would let it choose a
// carveout that holds one.
template <typename T, int NTH>
__global__ void __launch_bounds__(NTH, 1024 / NTH) k_smooth_pipe(LevelView L, const T* __restrict__ b,
                                                                 const double* bmean, XFetch<T> X, T* xout,
                                                                 RedBuf rb, double* mean_out, double inv_nfluid,
                                                                 const SolveFlags* flags, int maxit, T c2, T c1,
                                                                 int prev_mode, XFetch<T> P, int b16) {
  smooth_launch<T, NTH, true>(L, b, bmean, X, xout, rb, mean_out, inv_nfluid, flags, maxit, c2, c1, prev_mode, P,
                              b16);
}

// The last post-smoothing sweep of level 0 on a non-singular system, fused
// with the PCG dots that follow it (k_pcg_dots, first = 0): z' = fluid ? z :
// 0 goes to zo (FP64) and z'.rnew, z'.r are reduced in the same pass, cell for
// cell in k_pcg_dots' order, into the flexible beta.
template <typename T>
struct DotsOut {
  double* zo;
  const double* rnew;
  const double* r;
  double part[2] = {0.0, 0.0};
  __device__ __forceinline__ void operator()(int c, double wgt, T out, bool fluid) {
    const double v = fluid ? static_cast<double>(out) : 0.0;
    zo[c] = v;
    part[0] += wgt * (v * rnew[c]);
    part[1] += wgt * (v * r[c]);
  }
};

template <typename T, int NTH>
__global__ void __launch_bounds__(NTH, sweep_ctas<T, NTH>()) k_smooth_dots(LevelView L, const T* __restrict__ b, XFetch<T> X,
                                                     double* __restrict__ zo, const double* __restrict__ rnew,
                                                     const double* __restrict__ r, RedBuf rb, double* S,
                                                     SolveFlags* flags, int maxit, T c2, T c1, int prev_mode,
                                                     XFetch<T> P) {
  __shared__ BrickPre pre[2];
  prefetch_brick(L, blockIdx.x, X.prolongs(), pre[0]);
  pdl_wait();
  __syncthreads();
  if (stopped(flags, maxit)) return;
  __shared__ T tile[TSN];
  DotsOut<T> sink{zo, rnew, r};
  smooth_bricks<T, NTH>(L, b, nullptr, X, sink, c2, c1, prev_mode, P, blockIdx.x, gridDim.x, tile, GAcc{}, 0, pre);
  grid_reduce<2>(sink.part, rb, [=] __device__(const double* t) { flex_beta(t, S, flags); });
}

// The first pre-smoothing sweep of a coarse level, from x = 0, at one cell:
// pointwise in the cell's restricted residual, so the restriction that
// produces the residual can also write the sweep's result. The same
// statements as smooth_bricks' sweep from zero (diagonal from the cell's code
// and coarse-fine couplings, x' = 0 + c2 (b - 0) / D), so the bits agree.
template <typename T>
__device__ __forceinline__ T first_sweep(const LevelView& C, int c, T bc, T c2) {
  const uint32_t code = C.code[c];
  if (code_type(code) != CELL_FLUID) return T(0);
  const int lev = C.amr ? C.blevel[c >> 9] : 0;
  T diag = T(0);
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const T h2 = static_cast<T>(C.amr ? C.lh2[lev][f >> 1] : C.h2[f >> 1]);
    if (code & (1u << f)) diag += h2;
    else if (code & (1u << (CODE_DIRICHLET + f))) diag += T(2) * h2;
  }
  if (C.amr && (code & (1u << CODE_HASCF)))
    for (int k = C.cf_off[c]; k < C.cf_off[c + 1]; ++k) diag += static_cast<T>(C.cf_coef[k]);
  const T off = T(0), xc = T(0);
  const T Ax = diag * xc - off;
  const T dM = diag > T(0) ? diag : T(1);
  if constexpr (sizeof(T) == 4)
    return xc + c2 * __fdividef(bc - Ax, dM);
  else
    return xc + c2 * (bc - Ax) / dM;
}

// ---------------------------------------------------------------------------
// Residual + full-weighting restriction (multigrid.cpp:116-154): one CTA per
// fine brick computes r = fluid ? b' - A x' : 0 into shared memory, then each
// coarse cell covered by the brick averages its fluid children, summed in the
// reference's lexicographic child order (k, then j, then i).
// ---------------------------------------------------------------------------
template <typename T, int NTH, class ACC, class FX>
__device__ __forceinline__ double resid_restrict_bricks(const LevelView& F, const T* b, const double* bmean,
                                                       const FX& X, const LevelView& C, int fx, int fy, int fz,
                                                       T* rc, int first, int stride, T* tile, T* rs, uint8_t* fl,
                                                       const ACC& acc, int bio = 0, T* xf = nullptr,
                                                       T c2f = T(0), BrickPre* pre = nullptr) {
  constexpr int CPT = BR3 / NTH;  // cells per thread
  double part = 0.0;
  const int cx = BR / fx, cy = BR / fy, cz = BR / fz;
  for (int brick = first, it = 0; brick < F.nbrick; brick += stride, ++it) {
    BrickPre* const cur = pre ? pre + (it & 1) : nullptr;
    uint32_t code[CPT];
    T bv[CPT];
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int c = brick * BR3 + threadIdx.x + q * NTH;
      code[q] = F.code[c];
      bv[q] = (bio & 1) ? ld_b16(b, c) : acc.ld(b, c);
    }
    fill_halo<T, NTH>(F, brick, tile, X, cur);
    __syncthreads();
    // the next brick's maps, in flight during this brick's arithmetic (the other record)
    if (pre) prefetch_brick(F, brick + stride, X.prolongs(), pre[(it + 1) & 1], &C);
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int l = threadIdx.x + q * NTH;
      const int c = brick * BR3 + l;
      const bool fluid = code_type(code[q]) == CELL_FLUID;
      T r = T(0);
      if (fluid) {
        T diag, off;
        full_row<T>(F, code[q], tile, brick, c, X, diag, off);
        T bc = bv[q];
        if (bmean) bc = bc - static_cast<T>(ldv<ACC::kCG>(bmean));
        r = bc - (diag * tile[tpos_local(l)] - off);
      }
      rs[l] = r;
      fl[l] = fluid;
    }
    __syncthreads();
    if (F.amr) {
      // composite transfer: a kept brick maps cell-for-cell; a merged brick
      // fills one octant (4^3 cells) of its parent with child averages.
      const int cb = cur ? cur->xcb : F.xf_brick[brick], oct = cur ? cur->xoct : F.xf_oct[brick];
      const double wc = cur ? cur->wc : cell_weight(C, cb);
      if (oct < 0) {
        for (int t = threadIdx.x; t < BR3; t += NTH) {
          const T val = fl[t] ? rs[t] : T(0);
          const T sv = (bio & 2) ? st_b16(rc, cb * BR3 + t, val) : (acc.st(rc, cb * BR3 + t, val), val);
          if (xf) acc.st(xf, cb * BR3 + t, first_sweep(C, cb * BR3 + t, sv, c2f));
          part += wc * static_cast<double>(sv);
        }
      } else {
        for (int t = threadIdx.x; t < 64; t += NTH) {
          const int lci = t & 3, lcj = (t >> 2) & 3, lck = t >> 4;
          T sum = T(0);
          int count = 0;
          for (int dk = 0; dk < 2; ++dk)
            for (int dj = 0; dj < 2; ++dj)
              for (int di = 0; di < 2; ++di) {
                const int l = ((2 * lck + dk) << 6) | ((2 * lcj + dj) << 3) | (2 * lci + di);
                if (fl[l]) {
                  sum += rs[l];
                  ++count;
                }
              }
          const T val = count > 0 ? sum / static_cast<T>(count) : T(0);
          const int ci = (oct & 1) * 4 + lci, cj = ((oct >> 1) & 1) * 4 + lcj, ck = (oct >> 2) * 4 + lck;
          const int at = cb * BR3 + ((ck << 6) | (cj << 3) | ci);
          const T sv = (bio & 2) ? st_b16(rc, at, val) : (acc.st(rc, at, val), val);
          if (xf) acc.st(xf, at, first_sweep(C, at, sv, c2f));
          part += wc * static_cast<double>(sv);
        }
      }
    } else {
      for (int t = threadIdx.x; t < cx * cy * cz; t += NTH) {
        const int lci = t % cx, lcj = (t / cx) % cy, lck = t / (cx * cy);
        const int gci = F.bcoord[3 * brick] * cx + lci;
        const int gcj = F.bcoord[3 * brick + 1] * cy + lcj;
        const int gck = F.bcoord[3 * brick + 2] * cz + lck;
        if (gci < C.nx && gcj < C.ny && gck < C.nz) {
          T sum = T(0);
          int count = 0;
          for (int dk = 0; dk < fz; ++dk)
            for (int dj = 0; dj < fy; ++dj)
              for (int di = 0; di < fx; ++di) {
                const int l = ((lck * fz + dk) << 6) | ((lcj * fy + dj) << 3) | (lci * fx + di);
                if (fl[l]) {
                  sum += rs[l];
                  ++count;
                }
              }
          const T val = count > 0 ? sum / static_cast<T>(count) : T(0);
          const int at = cell_index(C, gci, gcj, gck);
          const T sv = (bio & 2) ? st_b16(rc, at, val) : (acc.st(rc, at, val), val);
          if (xf) acc.st(xf, at, first_sweep(C, at, sv, c2f));
          part += static_cast<double>(sv);
        }
      }
    }
    __syncthreads();
  }
  return part;
}

// Bounds: 4 CTAs an SM at 512 threads (32 registers), and for the smaller
// CTAs the count their registers already allow (4 at 128, 2 at 256), so that
// the driver sizes the shared memory for that many CTAs and not for one.
template <typename T, int NTH>
__global__ void __launch_bounds__(NTH, NTH == 256 ? 2 : 4) k_resid_restrict(LevelView F, const T* __restrict__ b,
                                                        const double* bmean, XFetch<T> X, LevelView C,
                                                        int fx, int fy, int fz, T* __restrict__ rc,
                                                        RedBuf rb, double* mean_out, double inv_nfluid_c,
                                                        const SolveFlags* flags, int maxit, int bio, T* xf,
                                                        T c2f) {
  __shared__ BrickPre pre[2];
  prefetch_brick(F, blockIdx.x, X.prolongs(), pre[0], &C);
  pdl_wait();
  __syncthreads();
  if (stopped(flags, maxit)) return;
  __shared__ T tile[TSN];
  __shared__ T rs[BR3];
  __shared__ uint8_t fl[BR3];
  double part[1] = {resid_restrict_bricks<T, NTH>(F, b, bmean, X, C, fx, fy, fz, rc, blockIdx.x, gridDim.x, tile,
                                                  rs, fl, GAcc{}, bio, xf, c2f, pre)};
  if (mean_out) {
    grid_reduce<1>(part, rb, [=] __device__(const double* tt) { *mean_out = tt[0] * inv_nfluid_c; });
  }
}

// ---------------------------------------------------------------------------
// Coarsest-level solve: CgPoisson(1e-6, 500)::solve (poisson.cpp:136-252) in
// one CTA with every vector in shared memory (FP64 in both forms). The level
// is held lexicographically in shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double bsum_bcast(double v, double* sh) {
  double a[1] = {v};
  block_reduce<1>(a, sh);
  if (threadIdx.x == 0) sh[64] = a[0];
  __syncthreads();
  return sh[64];
}
__device__ __forceinline__ void bsum2_bcast(double& v0, double& v1, double* sh) {
  double a[2] = {v0, v1};
  block_reduce<2>(a, sh);
  if (threadIdx.x == 0) {
    sh[64] = a[0];
    sh[65] = a[1];
  }
  __syncthreads();
  v0 = sh[64];
  v1 = sh[65];
}

// One CTA; `sm` holds coarse_smem(cells) bytes; `acc` addresses b and xout.
template <typename T, class ACC>
__device__ __forceinline__ void coarse_cg_body(const LevelView& C, const T* b, const double* bmean, T* xout,
                                               int singular, double tol, int maxit_cg, double* sm, const ACC& acc) {
  const int n = C.nx * C.ny * C.nz;
  const bool pre = n <= COARSE_PRE_CELLS;
  double* xs = sm;
  double* rs = xs + n;
  double* ps = rs + n;
  double* zs = ps + n;  // z, then Ap
  double* ds = zs + n;  // preconditioner diagonal
  double* rh = ds + n;  // rhs
  // Per-cell stencil, resolved once (levels of <= COARSE_PRE_CELLS cells): the
  // six neighbours in the row order below; >= 0 coupled cell, -1 no coupling,
  // -2 Dirichlet outlet face.
  int16_t* nb6 = reinterpret_cast<int16_t*>(rh + n);
  uint8_t* fl = pre ? reinterpret_cast<uint8_t*>(nb6 + 6 * n) : reinterpret_cast<uint8_t*>(rh + n);
  __shared__ double red[128];
  const int tid = threadIdx.x;
  auto lex_coords = [&](int m, int& i, int& j, int& k) {
    i = m % C.nx;
    j = (m / C.nx) % C.ny;
    k = m / (C.nx * C.ny);
  };
  // Row of A at lexicographic cell m (fluid), on shared-memory vector v.
  auto rowA = [&](int m, const double* v, double& diag, double& off) {
    int i, j, k;
    lex_coords(m, i, j, k);
    diag = 0.0;
    off = 0.0;
    for (int axis = 0; axis < 3; ++axis) {
      if (axis == 2 && C.twoD) continue;
      const double h2 = C.h2[axis];
      for (int side = -1; side <= 1; side += 2) {
        int c[3] = {i, j, k};
        const int dims[3] = {C.nx, C.ny, C.nz};
        c[axis] += side;
        int kind;
        if (c[axis] < 0 || c[axis] >= dims[axis]) {
          const int bt = C.bc[2 * axis + (side > 0 ? 1 : 0)];
          if (bt == NB_BC_PERIODIC) {
            c[axis] = (c[axis] + dims[axis]) % dims[axis];
            kind = 1;
          } else {
            kind = (bt == NB_BC_OUTLET) ? 2 : 0;
          }
        } else {
          kind = 1;
        }
        if (kind == 1) {
          const int nn = c[0] + C.nx * (c[1] + C.ny * c[2]);
          if (!fl[nn]) continue;  // solid neighbour: Neumann
          diag += h2;
          off += h2 * v[nn];
        } else if (kind == 2) {
          diag += 2.0 * h2;
        }
      }
    }
  };
  // load
  double bm = bmean ? ldv<ACC::kCG>(bmean) : 0.0;
  int nf_local = 0;
  for (int m = tid; m < n; m += blockDim.x) {
    int i, j, k;
    lex_coords(m, i, j, k);
    const int gidx = cell_index(C, i, j, k);
    const bool f = C.type[gidx] == CELL_FLUID;
    fl[m] = f;
    nf_local += f;
    rh[m] = f ? static_cast<double>(acc.ld(b, gidx)) - (bmean ? bm : 0.0) : 0.0;
    xs[m] = 0.0;
  }
  __syncthreads();
  if (pre) {  // resolve every fluid row once, in rowA's face order
    for (int m = tid; m < n; m += blockDim.x) {
      if (!fl[m]) continue;
      int i, j, k;
      lex_coords(m, i, j, k);
      const int dims[3] = {C.nx, C.ny, C.nz};
      for (int f = 0; f < 6; ++f) {
        const int axis = f >> 1, side = (f & 1) ? 1 : -1;
        int16_t code = -1;
        if (!(axis == 2 && C.twoD)) {
          int c[3] = {i, j, k};
          c[axis] += side;
          if (c[axis] < 0 || c[axis] >= dims[axis]) {
            const int bt = C.bc[2 * axis + (side > 0 ? 1 : 0)];
            if (bt == NB_BC_PERIODIC) {
              c[axis] = (c[axis] + dims[axis]) % dims[axis];
              const int nn = c[0] + C.nx * (c[1] + C.ny * c[2]);
              if (fl[nn]) code = static_cast<int16_t>(nn);
            } else if (bt == NB_BC_OUTLET) {
              code = -2;
            }
          } else {
            const int nn = c[0] + C.nx * (c[1] + C.ny * c[2]);
            if (fl[nn]) code = static_cast<int16_t>(nn);
          }
        }
        nb6[6 * m + f] = code;
      }
    }
  }
  // Row of A from the resolved stencil (same face order and sums as rowA).
  auto rowP = [&](int m, const double* v, double& diag, double& off) {
    diag = 0.0;
    off = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int code = nb6[6 * m + f];
      const double h2 = C.h2[f >> 1];
      if (code >= 0) {
        diag += h2;
        off += h2 * v[code];
      } else if (code == -2) {
        diag += 2.0 * h2;
      }
    }
  };
  for (int m = tid; m < n; m += blockDim.x) {
    double d = 1.0;
    if (fl[m]) {
      double dg, off;
      if (pre) rowP(m, xs, dg, off);
      else rowA(m, xs, dg, off);
      d = dg > 0.0 ? dg : 1.0;
    }
    ds[m] = d;
  }
  const double nfluid = bsum_bcast(static_cast<double>(nf_local), red);
  if (singular && nfluid > 0.0) {  // poisson.cpp:160-178
    double s = 0.0;
    for (int m = tid; m < n; m += blockDim.x)
      if (fl[m]) s += rh[m];
    const double mean = bsum_bcast(s, red) / nfluid;
    for (int m = tid; m < n; m += blockDim.x) rh[m] = fl[m] ? rh[m] - mean : 0.0;
    __syncthreads();
  }
  double rz_l = 0.0, bb_l = 0.0;
  for (int m = tid; m < n; m += blockDim.x) {
    rs[m] = rh[m];
    zs[m] = rs[m] / ds[m];
    ps[m] = zs[m];
    rz_l += rs[m] * zs[m];
    bb_l += rh[m] * rh[m];
  }
  bsum2_bcast(rz_l, bb_l, red);
  double rz = rz_l;
  const double bnorm = sqrt(bb_l) + 1e-300;
  for (int it = 0; it < maxit_cg; ++it) {
    double pap_l = 0.0;
    for (int m = tid; m < n; m += blockDim.x) {
      double ap;
      if (!fl[m]) {
        ap = ps[m];
      } else {
        double dg, off;
        if (pre) rowP(m, ps, dg, off);
        else rowA(m, ps, dg, off);
        ap = dg * ps[m] - off;
      }
      zs[m] = ap;
      pap_l += ps[m] * ap;
    }
    const double pAp = bsum_bcast(pap_l, red);
    if (fabs(pAp) < 1e-300) break;
    const double alpha = rz / pAp;
    // x, r update with |r|^2 and the next r.z in one pass (each thread owns
    // its cells; z overwrites Ap cell by cell); z is unused if r has converged.
    double rr_l = 0.0, rzn_l = 0.0;
    for (int m = tid; m < n; m += blockDim.x) {
      xs[m] += alpha * ps[m];
      rs[m] -= alpha * zs[m];
      rr_l += rs[m] * rs[m];
      zs[m] = rs[m] / ds[m];
      rzn_l += rs[m] * zs[m];
    }
    bsum2_bcast(rr_l, rzn_l, red);
    const double rnorm = sqrt(rr_l);
    if (rnorm <= tol * bnorm) break;
    const double rzNew = rzn_l;
    const double beta = rzNew / rz;
    for (int m = tid; m < n; m += blockDim.x) ps[m] = zs[m] + beta * ps[m];
    rz = rzNew;
    __syncthreads();
  }
  __syncthreads();
  double mean = 0.0;
  if (singular && nfluid > 0.0) {
    double s = 0.0;
    for (int m = tid; m < n; m += blockDim.x)
      if (fl[m]) s += xs[m];
    mean = bsum_bcast(s, red) / nfluid;
  }
  for (int m = tid; m < n; m += blockDim.x) {
    int i, j, k;
    lex_coords(m, i, j, k);
    const double v = (singular && fl[m]) ? xs[m] - mean : xs[m];
    acc.st(xout, cell_index(C, i, j, k), static_cast<T>(v));
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k_coarse_cg(LevelView C, const T* __restrict__ b,
                                                  const double* bmean, T* __restrict__ xout,
                                                  int singular, double tol, int maxit_cg,
                                                  const SolveFlags* flags, int maxit) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  extern __shared__ double sm[];
  coarse_cg_body<T>(C, b, bmean, xout, singular, tol, maxit_cg, sm, GAcc{});
}

// ---------------------------------------------------------------------------
// Exact coarsest-level solve (composite hierarchies): x = Minv (b - mean) on
// the fluid cells with the host-factored inverse, FP64, one CTA (a warp per
// row, lanes across columns). rhs preparation and the final mean removal are
// those of the CG path above.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_coarse_direct(LevelView C, const T* __restrict__ b, const double* bmean,
                                                      T* __restrict__ xout, const double* __restrict__ inv,
                                                      const int* __restrict__ fmap, const int* __restrict__ lexpos,
                                                      const int* __restrict__ lexcell, int nf, int singular,
                                                      const SolveFlags* flags, int maxit) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  extern __shared__ double sm[];
  double* rh = sm;       // [nf]
  double* xs = rh + nf;  // [nf]
  __shared__ double red[128];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const double bm = bmean ? *bmean : 0.0;
  double s = 0.0;
  for (int q = tid; q < nf; q += blockDim.x) {
    const double v = static_cast<double>(b[fmap[q]]) - (bmean ? bm : 0.0);
    rh[q] = v;
    s += v;
  }
  if (singular && nf > 0) {  // poisson.cpp:160-178 (rhs projected to zero mean)
    const double mean = bsum_bcast(s, red) / nf;
    for (int q = tid; q < nf; q += blockDim.x) rh[q] -= mean;
  }
  __syncthreads();
  for (int q = warp; q < nf; q += nwarp) {
    const double* row = inv + static_cast<size_t>(q) * nf;
    double acc = 0.0;
    for (int c = lane; c < nf; c += 32) acc += row[c] * rh[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) xs[q] = acc;
  }
  __syncthreads();
  double mean = 0.0;
  if (singular && nf > 0) {
    double t = 0.0;
    for (int q = tid; q < nf; q += blockDim.x) t += xs[q];
    mean = bsum_bcast(t, red) / nf;
  }
  const int n = C.nx * C.ny * C.nz;
  for (int m = tid; m < n; m += blockDim.x) {
    const int q = lexpos[m];
    xout[lexcell[m]] = static_cast<T>(q >= 0 ? (singular ? xs[q] - mean : xs[q]) : 0.0);
  }
}

// ---------------------------------------------------------------------------
// Cluster-resident V-cycle tail. The coarse end of every V-cycle (the levels
// from the first one of at most `tail_bricks` bricks down to the coarsest
// solve) costs one launch and a chain of dependent global loads per sweep
// when each sweep is its own kernel, whatever the level's size. Here one
// thread-block cluster of up to 16 CTAs runs all of it with every vector of
// those levels resident in the cluster's distributed shared memory (brick g in
// CTA g mod cs): each phase (sweep, residual + restriction, coarsest solve) is
// the launch path's own per-brick code over bricks rank, rank + cs, ...,
// reading neighbours and parents from the owning CTA's shared memory, and the
// phases are separated by the cluster's hardware barrier (barrier.cluster
// arrive.release / wait.acquire). The tail level's rhs is loaded from global
// memory at the start and its result stored back at the end. Pending means
// stay in global memory, summed over the CTAs' partials in rank order. Every
// CTA executes the same barriers: no CTA waits on a flag.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ XFetchT<T, const LevelView*, DAcc> tail_fetch(const TailFetch& f, const LevelView* lv,
                                                                         const DAcc& acc) {
  return XFetchT<T, const LevelView*, DAcc>{static_cast<const T*>(f.x), f.xmean, static_cast<const T*>(f.ec),
                                            f.ecmean, f.clvl >= 0 ? lv + f.clvl : lv, f.fx, f.fy, f.fz, f.xfb,
                                            f.xfo, acc};
}

// Exact coarsest solve spread over the cluster: every CTA stages the rhs, CTA
// r forms the rows of warps r * nwarp + w, ... into the (global) scratch
// vector, and after a cluster barrier every CTA scatters its share of the level.
template <typename T>
__device__ __forceinline__ void tail_direct(const TailProg* prog, const LevelView& C, const TailPhase& ph, int rank,
                                           int cs, cg::cluster_group& cl, double* rh, double* red, const DAcc& acc) {
  const int nf = prog->nf, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const T* b = static_cast<const T*>(ph.b);
  const double bm = ph.bmean ? ldv<true>(ph.bmean) : 0.0;
  double s = 0.0;
  for (int q = tid; q < nf; q += blockDim.x) {
    const double v = static_cast<double>(acc.ld(b, prog->fmap[q])) - bm;
    rh[q] = v;
    s += v;
  }
  if (prog->singular && nf > 0) {  // poisson.cpp:160-178 (rhs projected to zero mean)
    const double mean = bsum_bcast(s, red) / nf;
    for (int q = tid; q < nf; q += blockDim.x) rh[q] -= mean;
  }
  __syncthreads();
  double* xs = prog->xs;
  for (int q = rank * nwarp + warp; q < nf; q += cs * nwarp) {
    const double* row = prog->inv + static_cast<size_t>(q) * nf;
    double acc_r = 0.0;
    for (int c = lane; c < nf; c += 32) acc_r += row[c] * rh[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc_r += __shfl_down_sync(0xffffffffu, acc_r, off);
    if (lane == 0) xs[q] = acc_r;
  }
  cl.sync();
  double mean = 0.0;
  if (prog->singular && nf > 0) {
    double t = 0.0;
    for (int q = tid; q < nf; q += blockDim.x) t += __ldcg(xs + q);
    mean = bsum_bcast(t, red) / nf;
  }
  const int n = C.nx * C.ny * C.nz;
  T* xout = static_cast<T*>(ph.out);
  for (int m = rank * static_cast<int>(blockDim.x) + tid; m < n; m += cs * static_cast<int>(blockDim.x)) {
    const int q = prog->lexpos[m];
    const double v = q >= 0 ? __ldcg(xs + q) : 0.0;
    acc.st(xout, prog->lexcell[m], static_cast<T>(q >= 0 && prog->singular ? v - mean : v));
  }
}

// Copies this CTA's bricks (rank, rank + cs, ... of nbrick) between a global
// vector and its arena array at byte offset `off`.
template <typename T, bool TO_ARENA>
__device__ __forceinline__ void tail_copy(T* global, char* arena, uintptr_t off, int nbrick, int rank, int lcs) {
  T* local = reinterpret_cast<T*>(arena + (off - kArenaBias));
  for (int g = rank; g < nbrick; g += 1 << lcs)
    for (int l = threadIdx.x; l < BR3; l += blockDim.x) {
      if constexpr (TO_ARENA) local[((g >> lcs) << 9) + l] = global[g * BR3 + l];
      else global[g * BR3 + l] = local[((g >> lcs) << 9) + l];
    }
}

template <typename T>
__global__ void __launch_bounds__(NT) k_vtail(const TailProg* __restrict__ prog, const SolveFlags* flags, int maxit) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = static_cast<int>(cl.block_rank()), cs = static_cast<int>(cl.num_blocks());
  __shared__ LevelView slv[MAX_TAIL_LEV];
  __shared__ TailPhase sph[MAX_TAIL_PH];
  __shared__ T tile[TSN];
  __shared__ T rs[BR3];
  __shared__ uint8_t fl[BR3];
  __shared__ double red[128];
  __shared__ double cpart;
  extern __shared__ __align__(128) char dsm[];  // [arena | coarsest-solve scratch]
  const int nlev = prog->nlev, nph = prog->nphase, lcs = prog->lcs;
  const DAcc acc{dsm, lcs};
  double* scratch = reinterpret_cast<double*>(dsm + prog->arena_bytes);
  {
    const int* src = reinterpret_cast<const int*>(prog->lv);
    int* dst = reinterpret_cast<int*>(slv);
    for (int i = threadIdx.x; i < nlev * static_cast<int>(sizeof(LevelView) / 4); i += blockDim.x) dst[i] = src[i];
    src = reinterpret_cast<const int*>(prog->ph);
    dst = reinterpret_cast<int*>(sph);
    for (int i = threadIdx.x; i < nph * static_cast<int>(sizeof(TailPhase) / 4); i += blockDim.x) dst[i] = src[i];
  }
  // The program above is written once, when the solve is recorded: it is read
  // before the wait, while the predecessor grid drains.
  pdl_wait();
  if (stopped(flags, maxit)) return;  // the same answer in every CTA: nothing writes the flags meanwhile
  tail_copy<T, true>(static_cast<T*>(prog->b_in), dsm, prog->b_enc, prog->nbrick, rank, lcs);
  cl.sync();
  for (int p = 0; p < nph; ++p) {
    const TailPhase& ph = sph[p];
    const LevelView& L = slv[ph.lvl];
    double part = 0.0;
    if (ph.op == TAIL_SMOOTH) {
      SweepOut<T, DAcc> sink{static_cast<T*>(ph.out), acc};
      smooth_bricks<T, NT>(L, static_cast<const T*>(ph.b), ph.bmean, tail_fetch<T>(ph.X, slv, acc), sink,
                           static_cast<T>(ph.c2), static_cast<T>(ph.c1), ph.prev_mode, tail_fetch<T>(ph.P, slv, acc),
                           rank, cs, tile, acc);
      part = sink.part;
    } else if (ph.op == TAIL_RESID) {
      part = resid_restrict_bricks<T, NT>(L, static_cast<const T*>(ph.b), ph.bmean, tail_fetch<T>(ph.X, slv, acc),
                                          slv[ph.clvl], ph.fx, ph.fy, ph.fz, static_cast<T*>(ph.out), rank, cs, tile,
                                          rs, fl, acc);
    } else if (ph.op == TAIL_DIRECT) {
      tail_direct<T>(prog, L, ph, rank, cs, cl, scratch, red, acc);
    } else if (rank == 0) {  // TAIL_CG: CgPoisson(1e-6, 500) on one CTA
      coarse_cg_body<T>(L, static_cast<const T*>(ph.b), ph.bmean, static_cast<T*>(ph.out), prog->singular, 1e-6, 500,
                        scratch, acc);
    }
    if (ph.mean_out) {
      double a[1] = {part};
      block_reduce<1>(a, red);
      if (threadIdx.x == 0) cpart = a[0];
    }
    cl.sync();
    if (ph.mean_out) {
      if (rank == 0 && threadIdx.x == 0) {
        double t = 0.0;
        for (int r = 0; r < cs; ++r) t += *cl.map_shared_rank(&cpart, r);
        *ph.mean_out = t * ph.inv_nf;
      }
      cl.sync();
    }
  }
  tail_copy<T, false>(static_cast<T*>(prog->x_out), dsm, prog->x_enc, prog->nbrick, rank, lcs);
}

// ---------------------------------------------------------------------------
// Grid-resident V-cycle. Each sweep as its own kernel costs a launch, the
// scheduling of its CTAs and the drain of its stores, several microseconds on
// levels whose data movement takes one; a V-cycle has 15-20 of them. Here one
// cooperative launch (every CTA resident) runs the V-cycle's phase program:
// each phase is the launch path's own per-brick code (smooth_bricks,
// resid_restrict_bricks, the coarsest solves) over bricks blockIdx.x,
// blockIdx.x + gridDim.x, ..., and consecutive phases are separated by a grid
// barrier. Level vectors stay in global memory and are read through L2
// (ld.global.cg), since L1 is not coherent across SMs within a launch. A
// phase with a pending mean writes one partial per CTA; after the barrier
// every CTA sums the partials in the same fixed order and writes the same
// mean, so no second barrier is needed. Barrier waits are bounded: after about
// a second a CTA marks the launch aborted, sets the solve's stop code to
// STOP_TIMEOUT and every CTA returns.
// ---------------------------------------------------------------------------
struct GCAcc {
  static constexpr bool kCG = true;  // pending means are written inside the launch
  template <typename T>
  __device__ __forceinline__ T ld(const T* p, int n) const { return __ldcg(p + n); }
  template <typename T>
  __device__ __forceinline__ void st(T* p, int n, T v) const { p[n] = v; }
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The k-th barrier of the launch (k = 1, 2, ...): every CTA arrives once.
// Returns false if the launch was aborted (this CTA or another gave up).
__device__ __forceinline__ bool grid_barrier(const GridProg* prog, unsigned k, int* sh_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* cnt = prog->sync;
    unsigned* abort = prog->sync + 1;
    __threadfence();
    atomicAdd(cnt, 1u);
    const unsigned target = k * gridDim.x;
    const unsigned long long t0 = global_ns();
    int ok = 1;
    while (ld_acquire_u32(cnt) < target) {
      if (ld_acquire_u32(abort)) {
        ok = 0;
        break;
      }
      if (global_ns() - t0 > 1000000000ull) {  // about a second: give up
        atomicExch(abort, 1u);
        prog->flags->stop = STOP_TIMEOUT;
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    *sh_ok = ok;
  }
  __syncthreads();
  return *sh_ok != 0;
}

template <typename T>
__device__ __forceinline__ XFetchT<T, const LevelView*, GCAcc> grid_fetch(const TailFetch& f, const LevelView* lv) {
  return XFetchT<T, const LevelView*, GCAcc>{static_cast<const T*>(f.x), f.xmean, static_cast<const T*>(f.ec),
                                             f.ecmean, f.clvl >= 0 ? lv + f.clvl : lv, f.fx, f.fy, f.fz, f.xfb,
                                             f.xfo, GCAcc{}};
}

template <typename T, int NTH>
__global__ void __launch_bounds__(NTH, 1024 / NTH) k_vgrid(const GridProg* __restrict__ prog, const SolveFlags* flags, int maxit) {
  if (stopped(flags, maxit)) return;  // the same answer in every CTA: nothing writes the flags meanwhile
  __shared__ T tile[TSN];
  __shared__ T rs[BR3];
  __shared__ uint8_t fl[BR3];
  __shared__ double red[128];
  __shared__ int sh_ok;
  // dynamic shared memory: [level views | phases | coarsest-solve scratch]
  extern __shared__ __align__(16) double gdsm_all[];
  const int nlev = prog->nlev, nph = prog->nphase;
  LevelView* lv = reinterpret_cast<LevelView*>(gdsm_all);
  TailPhase* sph = reinterpret_cast<TailPhase*>(lv + nlev);
  double* gdsm = reinterpret_cast<double*>(sph + nph);
  {  // the program is read in every phase: one copy per CTA up front
    const int* src = reinterpret_cast<const int*>(prog->lv);
    int* dst = reinterpret_cast<int*>(lv);
    for (int i = threadIdx.x; i < nlev * static_cast<int>(sizeof(LevelView) / 4); i += NTH) dst[i] = src[i];
    src = reinterpret_cast<const int*>(prog->ph);
    dst = reinterpret_cast<int*>(sph);
    for (int i = threadIdx.x; i < nph * static_cast<int>(sizeof(TailPhase) / 4); i += NTH) dst[i] = src[i];
  }
  __syncthreads();
  const GCAcc acc{};
  unsigned nbar = 0;
  for (int p = 0; p < nph; ++p) {
    const TailPhase& ph = sph[p];
    const LevelView& L = lv[ph.lvl];
    double part = 0.0;
    if (ph.op == TAIL_SMOOTH) {
      SweepOut<T, GCAcc> sink{static_cast<T*>(ph.out), acc};
      smooth_bricks<T, NTH>(L, static_cast<const T*>(ph.b), ph.bmean, grid_fetch<T>(ph.X, lv), sink,
                            static_cast<T>(ph.c2), static_cast<T>(ph.c1), ph.prev_mode, grid_fetch<T>(ph.P, lv),
                            blockIdx.x, gridDim.x, tile, acc);
      part = sink.part;
    } else if (ph.op == TAIL_RESID) {
      part = resid_restrict_bricks<T, NTH>(L, static_cast<const T*>(ph.b), ph.bmean, grid_fetch<T>(ph.X, lv),
                                           lv[ph.clvl], ph.fx, ph.fy, ph.fz, static_cast<T*>(ph.out), blockIdx.x,
                                           gridDim.x, tile, rs, fl, acc);
    } else if (ph.op == TAIL_DIRECT) {
      // the exact coarsest solve: every CTA stages the rhs, the rows of the
      // dense inverse are spread over all warps of the grid, then (after a
      // barrier) every CTA scatters its share of the level
      const int nf = prog->nf, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = NTH >> 5;
      const T* b = static_cast<const T*>(ph.b);
      const double bm = ph.bmean ? __ldcg(ph.bmean) : 0.0;
      double* rh = gdsm;
      double sum = 0.0;
      for (int q = tid; q < nf; q += NTH) {
        const double v = static_cast<double>(acc.ld(b, prog->fmap[q])) - bm;
        rh[q] = v;
        sum += v;
      }
      if (prog->singular && nf > 0) {  // poisson.cpp:160-178 (rhs projected to zero mean)
        const double mean = bsum_bcast(sum, red) / nf;
        for (int q = tid; q < nf; q += NTH) rh[q] -= mean;
      }
      __syncthreads();
      for (int q = blockIdx.x * nwarp + warp; q < nf; q += gridDim.x * nwarp) {
        const double* row = prog->inv + static_cast<size_t>(q) * nf;
        double a = 0.0;
        for (int c = lane; c < nf; c += 32) a += row[c] * rh[c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if (lane == 0) prog->xs[q] = a;
      }
      if (!grid_barrier(prog, ++nbar, &sh_ok)) return;
      double mean = 0.0;
      if (prog->singular && nf > 0) {
        double t = 0.0;
        for (int q = tid; q < nf; q += NTH) t += __ldcg(prog->xs + q);
        mean = bsum_bcast(t, red) / nf;
      }
      const int n = L.nx * L.ny * L.nz;
      T* xout = static_cast<T*>(ph.out);
      for (int m = blockIdx.x * NTH + tid; m < n; m += gridDim.x * NTH) {
        const int q = prog->lexpos[m];
        const double v = q >= 0 ? __ldcg(prog->xs + q) : 0.0;
        acc.st(xout, prog->lexcell[m], static_cast<T>(q >= 0 && prog->singular ? v - mean : v));
      }
    } else if (blockIdx.x == 0) {  // TAIL_CG: CgPoisson(1e-6, 500) on one CTA
      coarse_cg_body<T>(L, static_cast<const T*>(ph.b), ph.bmean, static_cast<T*>(ph.out), prog->singular, 1e-6,
                        500, gdsm, acc);
    }
    // partials alternate between two halves by phase parity: a CTA that has
    // moved on cannot overwrite what a slower one is still summing
    double* parts = prog->partials + (p & 1) * gridDim.x;
    if (ph.mean_out) {
      double a[1] = {part};
      block_reduce<1>(a, red);
      if (threadIdx.x == 0) parts[blockIdx.x] = a[0];
    }
    if (p + 1 == nph && !ph.mean_out) break;  // the end of the launch orders the last phase
    if (!grid_barrier(prog, ++nbar, &sh_ok)) return;
    if (ph.mean_out) {  // every CTA forms the same mean from the partials, in the same order
      double a[1] = {0.0};
      for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += NTH) a[0] += __ldcg(parts + i);
      block_reduce<1>(a, red);
      if (threadIdx.x == 0) *ph.mean_out = a[0] * ph.inv_nf;
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// PCG vector kernels on level 0 (FP64).
// ---------------------------------------------------------------------------
struct DFetch {
  const double* x;
  const double* xmean;
  __device__ __forceinline__ double operator()(int n, int, int, int) const {
    return xmean ? x[n] - *xmean : x[n];
  }
  __device__ __forceinline__ bool prolongs() const { return false; }
  __device__ __forceinline__ double at(int n, int, int, int) const { return xmean ? x[n] - *xmean : x[n]; }
};

// out = A x, identity rows on solid cells (poisson.cpp:102-134); void cells 0.
__global__ void __launch_bounds__(NT) k_apply_a(LevelView L, const double* __restrict__ x,
                                                double* __restrict__ out) {
  pdl_wait();
  DFetch X{x, nullptr};
  __shared__ double tile[TSN];
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    fill_halo<double>(L, brick, tile, X);
    __syncthreads();
    const int c = brick * BR3 + threadIdx.x;
    const uint32_t code = L.code[c];
    const int ty = code_type(code);
    double o = 0.0;
    if (ty == CELL_SOLID) {
      o = x[c];
    } else if (ty == CELL_FLUID) {
      const int ctr = tpos_local(threadIdx.x);
      double diag, off;
      full_row<double>(L, code, tile, brick, c, X, diag, off);
      o = diag * tile[ctr] - off;
    }
    out[c] = o;
    __syncthreads();
  }
}

// Sum of b over fluid cells -> S[S_BSUM] = mean (singular rhs projection).
__global__ void __launch_bounds__(NT) k_fluid_mean(LevelView L, const double* __restrict__ v,
                                                   const double* vmean, RedBuf rb, double* mean_out,
                                                   double inv_nfluid, const SolveFlags* flags,
                                                   int maxit) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    if (L.type[c] == CELL_FLUID) part[0] += cell_weight(L, brick) * (vmean ? v[c] - *vmean : v[c]);
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) { *mean_out = t[0] * inv_nfluid; });
}

// Float variant (mixed form: the V-cycle output z is FP32).
__global__ void __launch_bounds__(NT) k_fluid_mean_f(LevelView L, const float* __restrict__ v,
                                                     const double* vmean, RedBuf rb, double* mean_out,
                                                     double inv_nfluid, const SolveFlags* flags,
                                                     int maxit) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    if (L.type[c] == CELL_FLUID) {
      const double z = static_cast<double>(v[c]);
      part[0] += cell_weight(L, brick) * (vmean ? z - *vmean : z);
    }
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) { *mean_out = t[0] * inv_nfluid; });
}

// rhs = fluid ? b - mean : 0 ; r = rhs ; S_BNORM2 = rhs.rhs ; early-exit test
// (multigrid.cpp:279-298).
__global__ void __launch_bounds__(NT) k_pcg_setup(LevelView L, const double* __restrict__ b,
                                                  const double* bmean, double* __restrict__ rhs,
                                                  double* __restrict__ r, double* __restrict__ x,
                                                  float* __restrict__ r_f, RedBuf rb, double* S,
                                                  SolveFlags* flags, double tol) {
  pdl_wait();
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    double v = 0.0;
    if (L.type[c] == CELL_FLUID) v = bmean ? b[c] - *bmean : b[c];
    rhs[c] = v;
    r[c] = v;
    x[c] = 0.0;
    if (r_f) r_f[c] = static_cast<float>(v);
    part[0] += cell_weight(L, brick) * (v * v);
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) {
    S[S_BNORM2] = t[0];
    const double bnorm = sqrt(t[0]) + 1e-300;
    flags->iters = 0;
    flags->restarts = 0;
    flags->checked = 0;
    flags->nan = isnan(t[0]) ? 1 : 0;
    if (sqrt(t[0]) <= tol * bnorm || isnan(t[0])) {
      flags->stop = 1;
      flags->early = 1;
    } else {
      flags->stop = 0;
      flags->early = 0;
    }
  });
}

// Setup from an initial guess: x = fluid ? scale * guess : 0 with scale =
// alpha * (*dt), r = rhs - A x (rhs as k_pcg_setup forms it), the same |rhs|^2
// and early exit (the stopping test stays relative to |rhs|).

// The initial guess of a warm-started solve: s1 g1 + s2 g2 + s3 g3 (g2, g3 optional).
struct GuessFetch {
  const double* g1;
  const double* g2;
  const double* g3;
  double s1, s2, s3;
  __device__ __forceinline__ double val(int n) const {
    double v = s1 * g1[n];
    if (g2) v += s2 * g2[n];
    if (g3) v += s3 * g3[n];
    return v;
  }
  __device__ __forceinline__ double operator()(int n, int, int, int) const { return val(n); }
  __device__ __forceinline__ bool prolongs() const { return false; }
  __device__ __forceinline__ double at(int n, int, int, int) const { return val(n); }
};

__global__ void __launch_bounds__(NT) k_pcg_setup_warm(LevelView L, const double* __restrict__ b,
                                                       const double* bmean, const double* __restrict__ guess,
                                                       const double* __restrict__ dtp, double alpha,
                                                       const double* __restrict__ h1, const double* __restrict__ h2,
                                                       const double* __restrict__ h3, double k2, double k3,
                                                       const int* nhist,
                                                       double* __restrict__ rhs, double* __restrict__ r,
                                                       double* __restrict__ x, float* __restrict__ r_f, RedBuf rb,
                                                       double* S, SolveFlags* flags, double tol) {
  pdl_wait();
  const int nh = nhist ? *nhist : 0;
  const double dt = *dtp;
  const GuessFetch X = nh >= 2 ? GuessFetch{h1, h2, h3, dt, k2 * dt, k3 * dt}
                               : GuessFetch{guess, nullptr, nullptr, alpha * dt, 0.0, 0.0};
  __shared__ double tile[TSN];
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    fill_halo<double>(L, brick, tile, X);
    __syncthreads();
    const int c = brick * BR3 + threadIdx.x;
    const uint32_t code = L.code[c];
    double v = 0.0, xv = 0.0, rv = 0.0;
    if (code_type(code) == CELL_FLUID) {
      v = bmean ? b[c] - *bmean : b[c];
      double diag, off;
      full_row<double>(L, code, tile, brick, c, X, diag, off);
      xv = tile[tpos_local(threadIdx.x)];
      rv = v - (diag * xv - off);
    }
    rhs[c] = v;
    r[c] = rv;
    x[c] = xv;
    if (r_f) r_f[c] = static_cast<float>(rv);
    part[0] += cell_weight(L, brick) * (v * v);
    __syncthreads();
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) {
    S[S_BNORM2] = t[0];
    const double bnorm = sqrt(t[0]) + 1e-300;
    flags->iters = 0;
    flags->restarts = 0;
    flags->checked = 0;
    flags->nan = isnan(t[0]) ? 1 : 0;
    if (sqrt(t[0]) <= tol * bnorm || isnan(t[0])) {
      flags->stop = 1;
      flags->early = 1;
    } else {
      flags->stop = 0;
      flags->early = 0;
    }
  });
}

// z' = fluid ? (z - m1) - m2 : 0 (the smoother's last removeMean, then Minv's,
// multigrid.cpp:283-288); written to zo (FP64). With `first`, p = z' and
// S_RZ = r.z'; otherwise S_RNEWZ = z'.rnew, S_RZCROSS = z'.r and the finaliser
// forms the flexible beta (multigrid.cpp:330-338).
template <typename TZ>
__global__ void __launch_bounds__(NT) k_pcg_dots(LevelView L, const TZ* __restrict__ z,
                                                 const double* m1, const double* m2,
                                                 double* __restrict__ zo, double* __restrict__ p,
                                                 const double* __restrict__ rnew,
                                                 const double* __restrict__ r, int first, RedBuf rb,
                                                 double* S, SolveFlags* flags, int maxit) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  double part[2] = {0.0, 0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    double v = 0.0;
    if (L.type[c] == CELL_FLUID) {
      v = static_cast<double>(z[c]);
      if (m1) v = v - *m1;
      if (m2) v = v - *m2;
    }
    zo[c] = v;
    if (first) {
      p[c] = v;
      part[0] += cell_weight(L, brick) * (r[c] * v);
    } else {
      part[0] += cell_weight(L, brick) * (v * rnew[c]);
      part[1] += cell_weight(L, brick) * (v * r[c]);
    }
  }
  grid_reduce<2>(part, rb, [=] __device__(const double* t) {
    if (first) {
      S[S_RZ] = t[0];
      S[S_BETA] = 0.0;  // the first matvec's direction is p = z' + 0 p
    } else {
      flex_beta(t, S, flags);
    }
  });
}

// The search direction p = z' + beta p_old (multigrid.cpp:335-337) as the
// matvec stages it: every CTA forms it for its own cells and its halo with
// the same fma, and the owner stores it.
struct DirFetch {
  const double* z;
  const double* p;
  double beta;
  __device__ __forceinline__ double operator()(int n, int, int, int) const { return fma(beta, p[n], z[n]); }
  __device__ __forceinline__ bool prolongs() const { return false; }
  __device__ __forceinline__ double at(int n, int, int, int) const { return fma(beta, p[n], z[n]); }
};

// p = z' + beta p_old into pnew ; Ap = A p ; S_PAP = p.Ap ; alpha = rz / pAp
// or breakdown (multigrid.cpp:303-308, 335-337). pold and pnew alternate from
// one cycle to the next, so no CTA reads a direction another CTA overwrote.
template <int NTH>
__global__ void __launch_bounds__(NTH) k_pcg_matvec(LevelView L, const double* __restrict__ z,
                                                    const double* __restrict__ pold, double* __restrict__ pnew,
                                                    double* __restrict__ Ap, RedBuf rb, double* S,
                                                    SolveFlags* flags, int maxit) {
  constexpr int CPT = BR3 / NTH;  // cells per thread
  pdl_wait();
  if (stopped(flags, maxit)) return;
  const DirFetch X{z, pold, S[S_BETA]};
  __shared__ double tile[TSN];
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    uint32_t code[CPT];
    double pv[CPT];
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int c = brick * BR3 + threadIdx.x + q * NTH;
      code[q] = L.code[c];
      pv[q] = X(c, 0, 0, 0);
      pnew[c] = pv[q];
    }
    fill_halo<double, NTH>(L, brick, tile, X);
    __syncthreads();
    const double wgt = cell_weight(L, brick);
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int l = threadIdx.x + q * NTH;
      const int c = brick * BR3 + l;
      const int ty = code_type(code[q]);
      const double pc = pv[q];
      double o = 0.0;
      if (ty == CELL_SOLID) {
        o = pc;
      } else if (ty == CELL_FLUID) {
        double diag, off;
        full_row<double>(L, code[q], tile, brick, c, X, diag, off);
        o = diag * pc - off;
      }
      Ap[c] = o;
      part[0] += wgt * (pc * o);
    }
    __syncthreads();
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) {
    S[S_PAP] = t[0];
    if (fabs(t[0]) < 1e-300 || isnan(t[0])) {
      flags->stop = 2;
      if (isnan(t[0])) flags->nan = 1;
    } else {
      S[S_ALPHA] = S[S_RZ] / t[0];
    }
  });
}

__device__ __forceinline__ void conv_check(double rnorm2, double* S, SolveFlags* flags, double tol) {
  S[S_RNORM2] = rnorm2;
  const double bnorm = sqrt(S[S_BNORM2]) + 1e-300;
  if (isnan(rnorm2)) {
    flags->nan = 1;
    flags->stop = 2;
  } else if (sqrt(rnorm2) <= tol * bnorm) {
    flags->stop = 1;
    flags->iters += 1;
  }
}

// x += alpha p ; rnew = r - alpha Ap (multigrid.cpp:309-316). Non-singular:
// reduces rnew.rnew and tests convergence; singular: reduces the fluid sum of
// rnew for removeMean (then k_pcg_center finishes).
__global__ void __launch_bounds__(NT) k_pcg_update(LevelView L, double* __restrict__ x,
                                                   const double* __restrict__ p,
                                                   const double* __restrict__ r,
                                                   const double* __restrict__ Ap,
                                                   double* __restrict__ rnew, float* __restrict__ rnew_f,
                                                   int singular, double inv_nfluid, RedBuf rb,
                                                   double* S, SolveFlags* flags, int maxit,
                                                   double tol, void* __restrict__ x0, double c2f) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  const double alpha = S[S_ALPHA];
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    x[c] += alpha * p[c];
    const double rn = r[c] - alpha * Ap[c];
    rnew[c] = rn;
    if (singular) {
      if (L.type[c] == CELL_FLUID) part[0] += cell_weight(L, brick) * rn;
    } else {
      part[0] += cell_weight(L, brick) * (rn * rn);
      if (rnew_f) rnew_f[c] = static_cast<float>(rn);
      // level 0's first pre-smoothing sweep from x = 0, pointwise in the
      // residual it smooths (rnew_f in the mixed form, rnew in FP64)
      if (x0) {
        if (rnew_f) static_cast<float*>(x0)[c] = first_sweep<float>(L, c, static_cast<float>(rn), static_cast<float>(c2f));
        else static_cast<double*>(x0)[c] = first_sweep<double>(L, c, rn, c2f);
      }
    }
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) {
    if (singular) S[S_RMEAN] = t[0] * inv_nfluid;
    else conv_check(t[0], S, flags, tol);
  });
}

// rnew = fluid ? rnew - mean : 0 ; rnew.rnew ; convergence (multigrid.cpp:317-325).
__global__ void __launch_bounds__(NT) k_pcg_center(LevelView L, double* __restrict__ rnew,
                                                   float* __restrict__ rnew_f, RedBuf rb, double* S,
                                                   SolveFlags* flags, int maxit, double tol) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  const double mean = S[S_RMEAN];
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    const double v = L.type[c] == CELL_FLUID ? rnew[c] - mean : 0.0;
    rnew[c] = v;
    if (rnew_f) rnew_f[c] = static_cast<float>(v);
    part[0] += cell_weight(L, brick) * (v * v);
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) { conv_check(t[0], S, flags, tol); });
}

// Final removeMean(x) + true residual (multigrid.cpp:341-353):
//   xf = fluid ? x - mean : x ; S_TRUERES2 = |rhs - A xf|^2
__global__ void __launch_bounds__(NT) k_true_residual(LevelView L, const double* __restrict__ x,
                                                      const double* xmean,
                                                      const double* __restrict__ rhs,
                                                      double* __restrict__ xf, RedBuf rb, double* S) {
  pdl_wait();
  DFetch X{x, xmean};
  __shared__ double tile[TSN];
  double part[1] = {0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    fill_halo<double>(L, brick, tile, X);
    __syncthreads();
    const int c = brick * BR3 + threadIdx.x;
    const uint32_t code = L.code[c];
    const int ty = code_type(code);
    double ax = 0.0, xv = x[c];
    if (ty == CELL_FLUID) {
      const int ctr = tpos_local(threadIdx.x);
      double diag, off;
      full_row<double>(L, code, tile, brick, c, X, diag, off);
      xv = tile[ctr];
      ax = diag * xv - off;
    } else if (ty == CELL_SOLID) {
      ax = xv;
    }
    xf[c] = xv;
    const double e = rhs[c] - ax;
    part[0] += cell_weight(L, brick) * (e * e);
    __syncthreads();
  }
  grid_reduce<1>(part, rb, [=] __device__(const double* t) { S[S_TRUERES2] = t[0]; });
}

// Loop condition of the graph form: keep cycling while not converged, not
// broken down and under the cycle cap.
// Outer iterative refinement (mixed form). The flexible PCG updates its FP64
// residual recursively; once it stops converged, the FP64 true residual
// rhs - A x decides: above tol |rhs| (and within kMaxRefine restarts and the
// cycle cap) the solve restarts from x with that residual, mean-removed on
// singular systems (multigrid.cpp:341-353 computes the same residual, for
// the report only). k_ir_residual forms the residual into `rt` and decides in
// its finaliser (stop back to 0 and restarts + 1 to restart); inside a graph
// it also sets the restart branch (h_if) and the second cycle loop (h_loop).
constexpr int kMaxRefine = 2;
__global__ void __launch_bounds__(NT) k_ir_residual(LevelView L, const double* __restrict__ x,
                                                    const double* __restrict__ rhs, double* __restrict__ rt,
                                                    RedBuf rb, double* S, SolveFlags* flags, double tol, int maxit,
                                                    double inv_nf, int cond, cudaGraphConditionalHandle h_if,
                                                    cudaGraphConditionalHandle h_loop) {
  pdl_wait();
  const bool act = flags->stop == 1 && !flags->early && !flags->checked && flags->iters < maxit &&
                   flags->restarts < kMaxRefine;
  if (!act) {
    if (cond && blockIdx.x == 0 && threadIdx.x == 0) {
      cudaGraphSetConditional(h_if, 0u);
      cudaGraphSetConditional(h_loop, 0u);
    }
    return;
  }
  DFetch X{x, nullptr};
  __shared__ double tile[TSN];
  double part[2] = {0.0, 0.0};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    fill_halo<double>(L, brick, tile, X);
    __syncthreads();
    const int c = brick * BR3 + threadIdx.x;
    const uint32_t code = L.code[c];
    double e = 0.0;
    if (code_type(code) == CELL_FLUID) {
      double diag, off;
      full_row<double>(L, code, tile, brick, c, X, diag, off);
      e = rhs[c] - (diag * tile[tpos_local(threadIdx.x)] - off);
    }
    rt[c] = e;
    const double w = cell_weight(L, brick);
    part[0] += w * (e * e);
    part[1] += w * e;
    __syncthreads();
  }
  grid_reduce<2>(part, rb, [=] __device__(const double* t) {
    S[S_IRRES2] = t[0];
    S[S_IRMEAN] = t[1] * inv_nf;
    const bool again = t[0] > tol * tol * S[S_BNORM2];
    if (again) {
      flags->stop = 0;
      flags->restarts += 1;
    } else {
      flags->checked = 1;
    }
    if (cond) {
      cudaGraphSetConditional(h_if, again ? 1u : 0u);
      cudaGraphSetConditional(h_loop, again ? 1u : 0u);
    }
  });
}

// The restart: r = true residual (fluid mean removed when singular) and its
// FP32 copy for the V-cycle; then the first direction as at the start.
__global__ void __launch_bounds__(NT) k_ir_restart(LevelView L, const double* __restrict__ rt, double* __restrict__ r,
                                                   float* __restrict__ rf, const double* S, const SolveFlags* flags,
                                                   int sing, int maxit) {
  pdl_wait();
  if (stopped(flags, maxit)) return;
  const double m = sing ? S[S_IRMEAN] : 0.0;
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    const double v = L.type[c] == CELL_FLUID ? rt[c] - m : 0.0;
    r[c] = v;
    if (rf) rf[c] = static_cast<float>(v);
  }
}

__global__ void k_set_cond(cudaGraphConditionalHandle h, const SolveFlags* f, int maxit,
                           unsigned long long* execs) {
  cudaGraphSetConditional(h, (f->stop == 0 && f->iters < maxit) ? 1u : 0u);
  if (execs) *execs += 1ull;
}

// Per-solve report: iterations, stop code, early exit, |rhs|^2, |true residual|^2, NaN.
__global__ void k_report(const SolveFlags* f, const double* S, double* out) {
  pdl_wait();
  out[0] = static_cast<double>(f->iters);
  out[1] = static_cast<double>(f->stop);
  out[2] = static_cast<double>(f->early);
  out[3] = S[S_BNORM2];
  out[4] = S[S_TRUERES2];
  out[5] = static_cast<double>(f->nan);
}

}  // namespace

// ===========================================================================
// host driver
// ===========================================================================
void* MgSolver::alloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  const cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw ApiError{NB_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed"};
  }
  allocs_.push_back(p);
  bytes_ += bytes;
  return p;
}

void MgSolver::upload_uniform(DevLevel& D, const int bcs[6]) {
  build_codes(D.h, bcs);
  const HostLevel& h = D.h;
  const size_t tsz = precision_ == NB_PRECISION_MIXED ? sizeof(float) : sizeof(double);
  const size_t ncs = static_cast<size_t>(h.nbrick) * BR3;
  D.d_lut = static_cast<int*>(alloc(h.lut.size() * sizeof(int)));
  D.d_bcoord = static_cast<int*>(alloc(h.bcoord.size() * sizeof(int)));
  D.d_type = static_cast<uint8_t*>(alloc(ncs));
  D.d_code = static_cast<uint16_t*>(alloc(ncs * sizeof(uint16_t)));
  NB_CUDA(cudaMemcpy(D.d_lut, h.lut.data(), h.lut.size() * sizeof(int), cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(D.d_bcoord, h.bcoord.data(), h.bcoord.size() * sizeof(int), cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(D.d_type, h.type.data(), ncs, cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(D.d_code, h.code.data(), ncs * sizeof(uint16_t), cudaMemcpyHostToDevice));
  D.b = alloc(ncs * tsz);
  D.x0 = alloc(ncs * tsz);
  D.x1 = alloc(ncs * tsz);
  NB_CUDA(cudaMemset(D.b, 0, ncs * tsz));
  NB_CUDA(cudaMemset(D.x0, 0, ncs * tsz));
  NB_CUDA(cudaMemset(D.x1, 0, ncs * tsz));
  D.wfluid = static_cast<double>(h.nfluid);
  D.ncell = static_cast<double>(h.nx) * h.ny * h.nz;
  LevelView& v = D.v;
  v = LevelView{};
  v.nx = h.nx;
  v.ny = h.ny;
  v.nz = h.nz;
  v.nbx = h.nbx;
  v.nby = h.nby;
  v.nbz = h.nbz;
  v.nbrick = h.nbrick;
  for (int f = 0; f < 6; ++f) v.bc[f] = bcs[f];
  v.dxyz[0] = h.dx;
  v.dxyz[1] = h.dy;
  v.dxyz[2] = h.dz;
  v.h2[0] = 1.0 / (h.dx * h.dx);
  v.h2[1] = 1.0 / (h.dy * h.dy);
  v.h2[2] = 1.0 / (h.dz * h.dz);
  v.twoD = h.nz == 1;
  v.lut = D.d_lut;
  v.bcoord = D.d_bcoord;
  v.type = D.d_type;
  v.code = D.d_code;
}

void MgSolver::upload_amr(DevLevel& D, const AmrLevelHost& A, const int bcs[6]) {
  const AmrTree& t = A.tree;
  const size_t tsz = precision_ == NB_PRECISION_MIXED ? sizeof(float) : sizeof(double);
  const int nbrick = static_cast<int>(t.leaves.size());
  const size_t ncs = static_cast<size_t>(nbrick) * BR3;
  auto up = [&](const void* src, size_t bytes) {
    void* d = alloc(bytes);
    if (src) NB_CUDA(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice));  // empty lists stay unread
    else NB_CUDA(cudaMemset(d, 0, bytes));
    return d;
  };
  D.h = HostLevel{};
  D.h.nbrick = nbrick;
  D.h.nfluid = A.nfluid;
  D.wfluid = A.wfluid;
  D.ncell = static_cast<double>(ncs);
  D.d_lut = static_cast<int*>(up(t.lut.data(), t.lut.size() * sizeof(int)));
  D.d_bcoord = static_cast<int*>(up(A.bcoord.data(), A.bcoord.size() * sizeof(int)));
  D.d_type = static_cast<uint8_t*>(up(A.type.data(), ncs));
  D.d_code = static_cast<uint16_t*>(up(A.code.data(), ncs * sizeof(uint16_t)));
  D.b = alloc(ncs * tsz);
  D.x0 = alloc(ncs * tsz);
  D.x1 = alloc(ncs * tsz);
  NB_CUDA(cudaMemset(D.b, 0, ncs * tsz));
  NB_CUDA(cudaMemset(D.x0, 0, ncs * tsz));
  NB_CUDA(cudaMemset(D.x1, 0, ncs * tsz));
  LevelView& v = D.v;
  v = LevelView{};
  v.amr = 1;
  v.nbrick = nbrick;
  v.nlev = t.nlev;
  for (int f = 0; f < 6; ++f) v.bc[f] = bcs[f];
  v.nx = t.cells(0, 0);
  v.ny = t.cells(0, 1);
  v.nz = t.cells(0, 2);
  for (int L = 0; L < t.nlev && L < AMR_MAXLEV; ++L) {
    v.lut_off[L] = t.lut_off[L];
    for (int a = 0; a < 3; ++a) {
      v.lnb[L][a] = t.lnb(L, a);
      v.lcells[L][a] = t.cells(L, a);
      const double h = t.h(L, a);
      v.lh2[L][a] = 1.0 / (h * h);
    }
  }
  for (int a = 0; a < 3; ++a) v.dxyz[a] = t.h(0, a);
  v.lut = D.d_lut;
  v.bcoord = D.d_bcoord;
  v.type = D.d_type;
  v.code = D.d_code;
  v.blevel = static_cast<const int8_t*>(up(A.blevel.data(), A.blevel.size()));
  v.bweight = static_cast<const double*>(up(A.bweight.data(), A.bweight.size() * sizeof(double)));
  v.cf_off = static_cast<const int*>(up(A.cf_off.data(), A.cf_off.size() * sizeof(int)));
  v.cf_nbr = static_cast<const int*>(up(A.cf_nbr.data(), std::max<size_t>(1, A.cf_nbr.size()) * sizeof(int)));
  v.cf_coef = static_cast<const double*>(
      up(A.cf_coef.data(), std::max<size_t>(1, A.cf_coef.size()) * sizeof(double)));
  if (!A.xf_brick.empty()) {
    D.d_xfb = static_cast<int*>(up(A.xf_brick.data(), A.xf_brick.size() * sizeof(int)));
    D.d_xfo = static_cast<int*>(up(A.xf_oct.data(), A.xf_oct.size() * sizeof(int)));
    v.xf_brick = D.d_xfb;
    v.xf_oct = D.d_xfo;
  }
  // same-level face neighbours (the staged halo never reads across a level jump)
  D.h_nbr6.assign(static_cast<size_t>(nbrick) * 6, -1);
  for (int r = 0; r < nbrick; ++r) {
    const AmrLeaf& f = t.leaves[r];
    for (int face = 0; face < 6; ++face) {
      const int a = face >> 1;
      int c[3] = {f.b[0], f.b[1], f.b[2]};
      c[a] += (face & 1) ? 1 : -1;
      const int n = t.lnb(f.level, a);
      if (c[a] < 0 || c[a] >= n) {
        if (bcs[2 * a] != NB_BC_PERIODIC) continue;
        c[a] = (c[a] + n) % n;
      }
      D.h_nbr6[6 * r + face] = t.find(f.level, c[0], c[1], c[2]);
    }
  }
  D.h_par = A.xf_brick;
  D.h_poct = A.xf_oct;
}

// Exact coarsest-level operator for composite hierarchies: the fluid block of
// the coarsest uniform level's -Laplacian (the rows k_coarse_cg applies),
// plus alpha * 1 1^T on the constant mode when the system is singular, inverted
// by Gauss-Jordan elimination with partial pivoting. Returns false (the CG
// path stays) when the level is too large or the block is singular (e.g. a
// fluid region split by solids).
bool MgSolver::build_dense_coarse() {
  const DevLevel& D = lv_.back();
  if (D.v.amr) return false;
  const HostLevel& h = D.h;
  const int n = h.nx * h.ny * h.nz;
  // Gauss-Jordan costs ~2 n^3 on the host (the default limit of 256 cells
  // keeps set-up cheap; larger coarsest levels converge in a few CG iterations).
  if (n > direct_max_ || h.solid.size() != static_cast<size_t>(n)) return false;
  std::vector<int> pos(n, -1), fidx;
  for (int m = 0; m < n; ++m)
    if (!h.solid[m]) {
      pos[m] = static_cast<int>(fidx.size());
      fidx.push_back(m);
    }
  const int nf = static_cast<int>(fidx.size());
  if (nf == 0) return false;
  const int dims[3] = {h.nx, h.ny, h.nz};
  const double h2[3] = {1.0 / (h.dx * h.dx), 1.0 / (h.dy * h.dy), 1.0 / (h.dz * h.dz)};
  std::vector<double> A(static_cast<size_t>(nf) * nf, 0.0);
  double diag_sum = 0.0;
  for (int q = 0; q < nf; ++q) {
    const int m = fidx[q];
    const int ijk[3] = {m % h.nx, (m / h.nx) % h.ny, m / (h.nx * h.ny)};
    double diag = 0.0;
    for (int axis = 0; axis < 3; ++axis) {
      if (axis == 2 && h.nz == 1) continue;
      for (int side = -1; side <= 1; side += 2) {
        int c[3] = {ijk[0], ijk[1], ijk[2]};
        c[axis] += side;
        if (c[axis] < 0 || c[axis] >= dims[axis]) {
          const int bt = D.v.bc[2 * axis + (side > 0 ? 1 : 0)];
          if (bt == NB_BC_OUTLET) {
            diag += 2.0 * h2[axis];
            continue;
          }
          if (bt != NB_BC_PERIODIC) continue;
          c[axis] = (c[axis] + dims[axis]) % dims[axis];
        }
        const int nn = c[0] + h.nx * (c[1] + h.ny * c[2]);
        if (h.solid[nn]) continue;
        diag += h2[axis];
        A[static_cast<size_t>(q) * nf + pos[nn]] -= h2[axis];
      }
    }
    A[static_cast<size_t>(q) * nf + q] += diag;
    diag_sum += diag;
  }
  if (singular_) {
    const double alpha = diag_sum / nf / nf;
    for (double& a : A) a += alpha;
  }
  // Gauss-Jordan with partial pivoting: [A | I] -> [I | A^-1]
  std::vector<double> I(static_cast<size_t>(nf) * nf, 0.0);
  for (int q = 0; q < nf; ++q) I[static_cast<size_t>(q) * nf + q] = 1.0;
  double amax = 0.0;
  for (double a : A) amax = std::max(amax, std::fabs(a));
  for (int col = 0; col < nf; ++col) {
    int piv = col;
    for (int r = col + 1; r < nf; ++r)
      if (std::fabs(A[static_cast<size_t>(r) * nf + col]) > std::fabs(A[static_cast<size_t>(piv) * nf + col])) piv = r;
    const double pv = A[static_cast<size_t>(piv) * nf + col];
    if (!(std::fabs(pv) > 1e-12 * amax)) return false;
    if (piv != col)
      for (int c = 0; c < nf; ++c) {
        std::swap(A[static_cast<size_t>(piv) * nf + c], A[static_cast<size_t>(col) * nf + c]);
        std::swap(I[static_cast<size_t>(piv) * nf + c], I[static_cast<size_t>(col) * nf + c]);
      }
    const double inv = 1.0 / pv;
    for (int c = 0; c < nf; ++c) {
      A[static_cast<size_t>(col) * nf + c] *= inv;
      I[static_cast<size_t>(col) * nf + c] *= inv;
    }
    for (int r = 0; r < nf; ++r) {
      if (r == col) continue;
      const double f = A[static_cast<size_t>(r) * nf + col];
      if (f == 0.0) continue;
      for (int c = 0; c < nf; ++c) {
        A[static_cast<size_t>(r) * nf + c] -= f * A[static_cast<size_t>(col) * nf + c];
        I[static_cast<size_t>(r) * nf + c] -= f * I[static_cast<size_t>(col) * nf + c];
      }
    }
  }
  auto cell = [&](int m) {
    const int i = m % h.nx, j = (m / h.nx) % h.ny, k = m / (h.nx * h.ny);
    const int b = h.lut[((k >> 3) * h.nby + (j >> 3)) * h.nbx + (i >> 3)];
    return b * BR3 + (((k & 7) << 6) | ((j & 7) << 3) | (i & 7));
  };
  std::vector<int> fmap(nf), lexcell(n);
  for (int q = 0; q < nf; ++q) fmap[q] = cell(fidx[q]);
  for (int m = 0; m < n; ++m) lexcell[m] = cell(m);
  dense_inv_ = static_cast<double*>(alloc(I.size() * sizeof(double)));
  dense_fmap_ = static_cast<int*>(alloc(fmap.size() * sizeof(int)));
  dense_lexpos_ = static_cast<int*>(alloc(pos.size() * sizeof(int)));
  dense_lexcell_ = static_cast<int*>(alloc(lexcell.size() * sizeof(int)));
  NB_CUDA(cudaMemcpy(dense_inv_, I.data(), I.size() * sizeof(double), cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(dense_fmap_, fmap.data(), fmap.size() * sizeof(int), cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(dense_lexpos_, pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice));
  NB_CUDA(cudaMemcpy(dense_lexcell_, lexcell.data(), lexcell.size() * sizeof(int), cudaMemcpyHostToDevice));
  dense_nf_ = nf;
  dense_ = true;
  return true;
}

// Per-brick maps that let a CTA stage a brick and its face halo (and the
// parents of both, for the prolongation folded into the first post-smoothing
// sweep) with one round of independent loads instead of chained LUT lookups.
void MgSolver::build_halo_maps() {
  const int nl = static_cast<int>(lv_.size());
  for (int m = 0; m < nl; ++m) {
    DevLevel& D = lv_[m];
    LevelView& v = D.v;
    const int nb = v.nbrick;
    if (!v.amr) {
      const HostLevel& h = D.h;
      if (h.nx % BR || h.ny % BR || h.nz % BR) continue;  // partial bricks: staged through the LUT
      D.h_nbr6.assign(static_cast<size_t>(nb) * 6, -1);
      const int nbs[3] = {h.nbx, h.nby, h.nbz};
      for (int r = 0; r < nb; ++r)
        for (int face = 0; face < 6; ++face) {
          const int a = face >> 1;
          int c[3] = {h.bcoord[3 * r], h.bcoord[3 * r + 1], h.bcoord[3 * r + 2]};
          c[a] += (face & 1) ? 1 : -1;
          if (c[a] < 0 || c[a] >= nbs[a]) {
            if (v.bc[2 * a] != NB_BC_PERIODIC) continue;
            c[a] = (c[a] + nbs[a]) % nbs[a];
          }
          D.h_nbr6[6 * r + face] = h.lut[(c[2] * h.nby + c[1]) * h.nbx + c[0]];
        }
      D.h_par.assign(nb, -1);
      D.h_poct.assign(nb, -1);
      if (m + 1 < nl && !lv_[m + 1].v.amr) {
        const HostLevel& C = lv_[m + 1].h;
        for (int r = 0; r < nb; ++r) {
          const int bx = h.bcoord[3 * r], by = h.bcoord[3 * r + 1], bz = h.bcoord[3 * r + 2];
          const int cx = C.fx == 2 ? bx >> 1 : bx, cy = C.fy == 2 ? by >> 1 : by, cz = C.fz == 2 ? bz >> 1 : bz;
          D.h_par[r] = C.lut[(cz * C.nby + cy) * C.nbx + cx];
          D.h_poct[r] = (bx & 1) | ((by & 1) << 1) | ((bz & 1) << 2);
        }
      }
    }
    if (D.h_par.size() != static_cast<size_t>(nb)) D.h_par.assign(nb, -1);
    if (D.h_poct.size() != static_cast<size_t>(nb)) D.h_poct.assign(nb, -1);
    std::vector<int> npar(static_cast<size_t>(nb) * 6, -1), npoct(static_cast<size_t>(nb) * 6, -1);
    for (size_t q = 0; q < npar.size(); ++q) {
      const int n = D.h_nbr6[q];
      if (n >= 0) {
        npar[q] = D.h_par[n];
        npoct[q] = D.h_poct[n];
      }
    }
    auto up = [&](const std::vector<int>& src) {
      int* d = static_cast<int*>(alloc(std::max<size_t>(1, src.size()) * sizeof(int)));
      if (!src.empty()) NB_CUDA(cudaMemcpy(d, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice));
      return d;
    };
    v.nbr6 = up(D.h_nbr6);
    v.par = up(D.h_par);
    v.poct = up(D.h_poct);
    v.npar6 = up(npar);
    v.npoct6 = up(npoct);
    v.fast = 1;
  }
}

void MgSolver::common_alloc() {
  const HostLevel& last = lv_.back().h;
  if (lv_.back().v.amr || static_cast<size_t>(last.nx) * last.ny * last.nz > COARSE_MAX_CELLS)
    throw ApiError{NB_ERR_UNSUPPORTED, "coarsest multigrid level exceeds 4096 cells"};
  if (lv_.size() > static_cast<size_t>(MAX_LEVELS))
    throw ApiError{NB_ERR_UNSUPPORTED, "multigrid hierarchy deeper than " + std::to_string(MAX_LEVELS) + " levels"};
  if (halo_mode_ == 0) build_halo_maps();
  n0_ = static_cast<size_t>(lv_[0].h.nbrick) * BR3;
  double** vecs[] = {&rhs_, &x_, &r_, &rnew_, &z_, &p_, &p2_, &Ap_, &xfin_};
  for (double** v : vecs) {
    *v = static_cast<double*>(alloc(n0_ * sizeof(double)));
    NB_CUDA(cudaMemset(*v, 0, n0_ * sizeof(double)));
  }
  if (precision_ == NB_PRECISION_MIXED) {
    rnew_f_ = static_cast<float*>(alloc(n0_ * sizeof(float)));
    NB_CUDA(cudaMemset(rnew_f_, 0, n0_ * sizeof(float)));
  }
  S_ = static_cast<double*>(alloc(S_COUNT * sizeof(double)));
  NB_CUDA(cudaMemset(S_, 0, S_COUNT * sizeof(double)));
  flags_ = static_cast<SolveFlags*>(alloc(sizeof(SolveFlags)));
  NB_CUDA(cudaMemset(flags_, 0, sizeof(SolveFlags)));
  body_execs_ = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long)));
  NB_CUDA(cudaMemset(body_execs_, 0, sizeof(unsigned long long)));
  rb_.max_blocks = MAX_GRID;
  rb_.partials = static_cast<double*>(alloc(RED_KMAX * MAX_GRID * sizeof(double)));
  rb_.counter = static_cast<unsigned*>(alloc(sizeof(unsigned)));
  NB_CUDA(cudaMemset(rb_.counter, 0, sizeof(unsigned)));
  NB_CUDA(cudaMallocHost(&h_flags_, sizeof(SolveFlags)));
  NB_CUDA(cudaMallocHost(&h_S_, S_COUNT * sizeof(double)));
  // The coarsest-level CTA keeps 6 FP64 vectors + flags in shared memory.
  const int smem_max = COARSE_MAX_CELLS * static_cast<int>(6 * sizeof(double) + 1);
  NB_CUDA(cudaFuncSetAttribute(k_coarse_cg<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
  NB_CUDA(cudaFuncSetAttribute(k_coarse_cg<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
}

void MgSolver::set_tuning(const nb_tuning* tune) {
  nb_tuning t;
  nb_tuning_default(&t);
  if (tune) t = *tune;
  int dev = 0, nsm = 148;
  NB_CUDA(cudaGetDevice(&dev));
  NB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  tpb_ = (t.threads_per_brick == 128 || t.threads_per_brick == 256) ? t.threads_per_brick : 512;
  const int per_sm = std::min(std::max(t.mg_ctas_per_sm, 1), 16);
  grid_cap_ = std::min(per_sm * nsm, MAX_GRID);  // the reduction buffer holds MAX_GRID partials
  pdl_ = t.pdl != 0;
  sweeps_ = precision_ == NB_PRECISION_MIXED ? std::min(std::max(t.sweeps, 1), 3) : 2;  // FP64: V(2,2) as the reference
  halo_mode_ = t.halo_mode == 1 ? 1 : 0;
  direct_max_ = std::min(std::max(t.coarse_direct_max, 0), 512);
  tail_bricks_ = std::min(std::max(t.tail_bricks, 0), 4096);
  vgrid_ = t.vgrid != 0;
  coarse_bf16_ = precision_ == NB_PRECISION_MIXED && t.coarse_bf16 != 0;
  // Smoother coefficients per sweep of a phase: damped Jacobi (the reference's,
  // c2 = omega) or, mixed form only, Chebyshev on [lmax / 6, lmax] of D^-1 A
  // with lmax = 2, the Gershgorin bound (every row of D^-1 A has diagonal 1
  // and off-diagonal magnitudes summing to at most 1) (three-term recurrence:
  // theta = (lmax + lmin) / 2, delta = (lmax - lmin) / 2, sigma = theta / delta,
  // rho_0 = 1 / sigma, rho_k = 1 / (2 sigma - rho_(k-1)); sweep 0 steps by
  // r / theta, sweep k by 2 rho_k / delta r + rho_k rho_(k-1) times the last step).
  cheb_ = precision_ == NB_PRECISION_MIXED && t.smoother == 1;
  for (int k = 0; k < 4; ++k) {
    cheb_c2_[k] = kOmega;
    cheb_c1_[k] = 0.0;
  }
  if (cheb_) {
    const double lmax = 2.0, lmin = lmax / 6.0;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
    double rho = 1.0 / sigma;
    cheb_c2_[0] = 1.0 / theta;
    for (int k = 1; k < 4; ++k) {
      const double r = 1.0 / (2.0 * sigma - rho);
      cheb_c1_[k] = r * rho;
      cheb_c2_[k] = 2.0 * r / delta;
      rho = r;
    }
  }
}

MgSolver::MgSolver(const nb_grid_desc& g, int precision, LaunchCounter lc, const nb_tuning* tune)
    : precision_(precision), lc_(lc) {
  set_tuning(tune);
  std::vector<HostLevel> H = build_hierarchy(g);
  singular_ = true;
  for (int f = 0; f < 6; ++f)
    if (g.face[f].type == NB_BC_OUTLET) singular_ = false;  // hasDirichlet, poisson.cpp:93-100
  int bcs[6];
  for (int f = 0; f < 6; ++f) bcs[f] = g.face[f].type;
  lv_.resize(H.size());
  for (size_t l = 0; l < H.size(); ++l) {
    lv_[l].h = std::move(H[l]);
    upload_uniform(lv_[l], bcs);
  }
  common_alloc();
  build_tail();
  build_grid();
  mark_bf16();
}

// Composite hierarchy: MG level m+1 merges the finest octree level of level m
// into its parents (cells fluid if any child is); once a single octree level
// remains the grid is uniform and coarsens as MgPoisson does
// (core/src/flow/multigrid.cpp:211-266).
MgSolver::MgSolver(const AmrLevelHost& fine, int precision, LaunchCounter lc, const nb_tuning* tune)
    : precision_(precision), lc_(lc) {
  set_tuning(tune);
  const AmrGeom& geo = fine.tree.geom;
  singular_ = true;
  for (int f = 0; f < 6; ++f)
    if (geo.bc[f] == NB_BC_OUTLET) singular_ = false;
  std::vector<AmrLevelHost> comp;
  comp.push_back(fine);
  while (comp.back().tree.nlev > 1) {
    AmrLevelHost& F = comp.back();
    AmrLevelHost C;
    C.tree = coarsen_tree(F.tree, F.xf_brick, F.xf_oct);
    C.wlmax = F.wlmax;
    amr_level_geometry(C);
    amr_level_types_coarsened(C, F);
    amr_level_codes(C);
    comp.push_back(std::move(C));
  }
  // The last composite level has one octree level: hand it to the uniform chain.
  const AmrLevelHost& U = comp.back();
  const int nx = U.tree.cells(0, 0), ny = U.tree.cells(0, 1), nz = U.tree.cells(0, 2);
  std::vector<uint8_t> solid(static_cast<size_t>(nx) * ny * nz, 0);
  for (size_t r = 0; r < U.tree.leaves.size(); ++r)
    for (int l = 0; l < BR3; ++l) {
      const AmrLeaf& f = U.tree.leaves[r];
      const int i = f.b[0] * BR + (l & 7), j = f.b[1] * BR + ((l >> 3) & 7), k = f.b[2] * BR + (l >> 6);
      solid[static_cast<size_t>(i) + static_cast<size_t>(nx) * (j + static_cast<size_t>(ny) * k)] =
          U.type[r * BR3 + l] == CELL_SOLID;
    }
  nb_grid_desc g0{};
  g0.nx = nx;
  g0.ny = ny;
  g0.nz = nz;
  g0.dx = U.tree.h(0, 0);
  g0.dy = U.tree.h(0, 1);
  g0.dz = U.tree.h(0, 2);
  for (int f = 0; f < 6; ++f) g0.face[f].type = geo.bc[f];
  g0.solid = solid.data();
  // A single-level mesh is a uniform grid and keeps the reference hierarchy
  // (<= 2048 coarsest cells). Below a multi-level mesh the uniform tail is
  // coarsened on to <= 512 cells: the coarsest level is solved by one CTA,
  // whose Jacobi-CG cost grows with the level's size.
  const size_t coarsest = fine.tree.nlev > 1 ? 512 : 2048;
  std::vector<HostLevel> H = build_hierarchy(g0, coarsest);
  // Uniform brick ranks equal the single-level tree's ranks (both Morton).
  for (size_t r = 0; r < U.tree.leaves.size(); ++r) {
    const AmrLeaf& f = U.tree.leaves[r];
    if (H[0].lut[(f.b[2] * H[0].nby + f.b[1]) * H[0].nbx + f.b[0]] != static_cast<int>(r))
      throw ApiError{NB_ERR_UNSUPPORTED, "brick ranking mismatch between composite and uniform levels"};
  }
  const size_t ncomp = comp.size() - 1;  // composite levels with >= 2 octree levels
  lv_.resize(ncomp + H.size());
  for (size_t m = 0; m < ncomp; ++m) upload_amr(lv_[m], comp[m], geo.bc);
  for (size_t l = 0; l < H.size(); ++l) {
    lv_[ncomp + l].h = std::move(H[l]);
    upload_uniform(lv_[ncomp + l], geo.bc);
  }
  common_alloc();
  // Below a multi-level mesh (no reference hierarchy to reproduce) the
  // coarsest level is solved exactly instead of by CgPoisson(1e-6, 500).
  if (fine.tree.nlev > 1) build_dense_coarse();
  build_tail();
  build_grid();
  mark_bf16();
}

MgSolver::~MgSolver() {
  for (void* p : allocs_) cudaFree(p);
  if (h_flags_) cudaFreeHost(h_flags_);
  if (h_S_) cudaFreeHost(h_S_);
  if (side_) cudaStreamDestroy(side_);
}

void MgSolver::apply_a(cudaStream_t s, const double* x, double* out) {
  const LevelView& L = lv_[0].v;
  NB_LAUNCH(lc_, "apply_a", s, lv_[0].ncell * 17,
            launch_pdl(pdl_, k_apply_a, dim3(grid_of(L.nbrick)), dim3(NT), 0, s, L, x, out));
  NB_CUDA(cudaGetLastError());
}

// One V-cycle at level `lvl` on rhs b (pending mean slot bmean_slot or -1).
// Returns the level's x buffer and the slot of its pending mean (-1 if none).
// With `prog`, every launch below is appended to prog as a cluster-tail phase
// (same arguments) instead of being issued.
template <typename T>
void MgSolver::vcycle(cudaStream_t s, int lvl, const void* bv, int bmean_slot, void* /*unused*/,
                      int* out_mean_slot, void** out_x, std::vector<TailPhase>* prog, bool first_done) {
  if (!prog && lvl == tail_lvl_) {
    launch_tail(s);
    *out_x = tail_x_;
    *out_mean_slot = tail_slot_;
    return;
  }
  DevLevel& D = lv_[lvl];
  const LevelView& L = D.v;
  const T* b = static_cast<const T*>(bv);
  const double* bmean = (singular_ && bmean_slot >= 0) ? S_ + bmean_slot : nullptr;
  const int grid = grid_of(L.nbrick);
  const double tsz = sizeof(T);
  const double ncell = D.ncell;
  const int rl = lvl - tail_lvl_;  // tail-relative level (prog only)
  // Records a phase (prog) or runs the launch.
#define MG_EMIT(fam, nbytes, phase, launch)           \
  do {                                                \
    if (prog) {                                       \
      prog->push_back(phase);                         \
      tail_bytes_ += static_cast<double>(nbytes);     \
    } else {                                          \
      NB_LAUNCH(lc_, fam, s, nbytes, launch);         \
    }                                                 \
  } while (0)
  const auto fetch = [&](const XFetch<T>& f, int clvl) {
    return TailFetch{f.x, f.xmean, f.ec, f.ecmean, f.ec ? clvl : -1, f.fx, f.fy, f.fz, f.xfb, f.xfo};
  };
  if (lvl + 1 == static_cast<int>(lv_.size())) {
    const size_t nco = static_cast<size_t>(L.nx) * L.ny * L.nz;
    TailPhase ph{};
    ph.op = dense_ ? TAIL_DIRECT : TAIL_CG;
    ph.lvl = rl;
    ph.clvl = -1;
    ph.b = b;
    ph.bmean = bmean;
    ph.X.clvl = ph.P.clvl = -1;
    ph.out = D.x0;
    if (dense_) {
      MG_EMIT("coarse_cg", ncell * (2 * tsz + 1) + 8.0 * dense_nf_ * dense_nf_, ph,
              launch_pdl(pdl_, k_coarse_direct<T>, dim3(1), dim3(NT), 2 * sizeof(double) * dense_nf_, s, L, b, bmean,
                         static_cast<T*>(D.x0), dense_inv_, dense_fmap_, dense_lexpos_, dense_lexcell_, dense_nf_,
                         singular_ ? 1 : 0, flags_, maxit_));
    } else {
      const size_t smem = coarse_smem(nco);
      MG_EMIT("coarse_cg", ncell * (2 * tsz + 1), ph,
              (launch_pdl(pdl_, k_coarse_cg<T>, dim3(1), dim3(NT), smem, s, L, b, bmean, static_cast<T*>(D.x0),
                          singular_ ? 1 : 0, 1e-6, 500, flags_, maxit_)));
    }
    *out_x = D.x0;
    *out_mean_slot = -1;
    return;
  }
  const double inv_nf = D.h.nfluid ? 1.0 / D.wfluid : 0.0;
  const bool sing = singular_ && D.h.nfluid > 0;
  T* xa = static_cast<T*>(D.x0);
  T* xb = static_cast<T*>(D.x1);
  double* mA = sing ? S_ + lvl_slot(lvl, 0) : nullptr;
  double* mB = sing ? S_ + lvl_slot(lvl, 1) : nullptr;
  const LevelView dummy = L;
  DevLevel& Cd = lv_[lvl + 1];
  const LevelView& C = Cd.v;
  const double ncoarse = Cd.ncell;
  // kernels for the tuned CTA size (threads per brick)
  // several bricks per CTA: the pipelined smoother (next brick's loads in flight)
  const bool pipe = sizeof(T) == 8 && L.fast && L.nbrick > grid;
  const auto ks = pipe ? (tpb_ == 128 ? k_smooth_pipe<T, 128> : (tpb_ == 256 ? k_smooth_pipe<T, 256> : k_smooth_pipe<T, 512>))
                       : (tpb_ == 128 ? k_smooth<T, 128> : (tpb_ == 256 ? k_smooth<T, 256> : k_smooth<T, 512>));
  const auto kr = tpb_ == 128 ? k_resid_restrict<T, 128>
                              : (tpb_ == 256 ? k_resid_restrict<T, 256> : k_resid_restrict<T, 512>);
  // Ping-pong buffers with their pending means: xa <-> slot 0, xb <-> slot 1.
  T* buf[2] = {xa, xb};
  double* mean[2] = {mA, mB};
  int cur = 0;
  const XFetch<T> none{nullptr, nullptr, nullptr, nullptr, dummy, 1, 1, 1};
  auto plain = [&](int i) { return XFetch<T>{buf[i], mean[i], nullptr, nullptr, dummy, 1, 1, 1}; };
  const auto smooth_phase = [&](const XFetch<T>& X, T* out, double* mout, double c2, double c1, int pm,
                                const XFetch<T>& P) {
    TailPhase ph{};
    ph.op = TAIL_SMOOTH;
    ph.lvl = rl;
    ph.clvl = rl + 1;
    ph.prev_mode = pm;
    ph.b = b;
    ph.bmean = bmean;
    ph.X = fetch(X, rl + 1);
    ph.P = fetch(P, rl + 1);
    ph.out = out;
    ph.mean_out = mout;
    ph.inv_nf = inv_nf;
    ph.c2 = c2;
    ph.c1 = c1;
    return ph;
  };
  // BF16 residual storage (recorded phases never carry it: the option leaves
  // the tail and the grid program's levels in FP32)
  const int b16 = (!prog && D.b16) ? 1 : 0;
  const int bio = b16 | ((!prog && Cd.b16) ? 2 : 0);
  const double bsz = b16 ? 2.0 : tsz;           // bytes of one b value of this level
  const double csz = (bio & 2) ? 2.0 : tsz;     // bytes of one coarse b value
  // pre-smoothing (sweeps_ sweeps; 2 as the reference), the first from x = 0
  // (already written by the restriction that made b when first_done)
  if (!first_done)
  MG_EMIT("smooth", ncell * (tsz + bsz + 1), smooth_phase(none, buf[cur], mean[cur], cheb_c2_[0], 0.0, 0, none),
          (launch_pdl(pdl_, ks, dim3(grid), dim3(tpb_), 0, s, L, b, bmean, none, buf[cur], rb_, mean[cur], inv_nf,
                      flags_, maxit_, static_cast<T>(cheb_c2_[0]), T(0), 0, none, b16)));
  for (int sw = 1; sw < sweeps_; ++sw, cur ^= 1)  // a Chebyshev step from sweep 2 on also reads x_prev
    MG_EMIT("smooth", ncell * (2 * tsz + bsz + 1) + (cheb_ && sw >= 2 ? ncell * tsz : 0.0),
            smooth_phase(plain(cur), buf[cur ^ 1], mean[cur ^ 1], cheb_c2_[sw], cheb_c1_[sw],
                         cheb_ ? (sw == 1 ? 2 : 1) : 0, plain(cur ^ 1)),
            (launch_pdl(pdl_, ks, dim3(grid), dim3(tpb_), 0, s, L, b, bmean, plain(cur), buf[cur ^ 1], rb_,
                        mean[cur ^ 1], inv_nf, flags_, maxit_, static_cast<T>(cheb_c2_[sw]),
                        static_cast<T>(cheb_c1_[sw]), cheb_ ? (sw == 1 ? 2 : 1) : 0, plain(cur ^ 1), b16)));
  // residual + restriction; on non-singular systems (no pending means) it also
  // writes the coarse level's first sweep when that level smooths by launches
  const bool fuse_first = !prog && !singular_ && lvl + 1 != tail_lvl_ && lvl + 2 < static_cast<int>(lv_.size());
  const double inv_nfc = Cd.h.nfluid ? 1.0 / Cd.wfluid : 0.0;
  const int cb_slot = lvl_slot(lvl + 1, 2);
  double* cmean = (singular_ && Cd.h.nfluid > 0) ? S_ + cb_slot : nullptr;
  {
    TailPhase ph{};
    ph.op = TAIL_RESID;
    ph.lvl = rl;
    ph.clvl = rl + 1;
    ph.b = b;
    ph.bmean = bmean;
    ph.X = fetch(plain(cur), -1);
    ph.P = fetch(none, -1);
    ph.out = Cd.b;
    ph.mean_out = cmean;
    ph.inv_nf = inv_nfc;
    ph.fx = Cd.h.fx;
    ph.fy = Cd.h.fy;
    ph.fz = Cd.h.fz;
    MG_EMIT("resid_restrict", ncell * (tsz + bsz + 1) + ncoarse * (csz + (fuse_first ? tsz : 0.0)), ph,
            (launch_pdl(pdl_, kr, dim3(grid), dim3(tpb_), 0, s, L, b, bmean,
                        XFetch<T>{buf[cur], mean[cur], nullptr, nullptr, dummy, 1, 1, 1}, C, Cd.h.fx, Cd.h.fy,
                        Cd.h.fz, static_cast<T*>(Cd.b), rb_, cmean, inv_nfc, flags_, maxit_, bio,
                        fuse_first ? static_cast<T*>(Cd.x0) : static_cast<T*>(nullptr),
                        static_cast<T>(cheb_c2_[0]))));
  }
  void* ec = nullptr;
  int ec_slot = -1;
  vcycle<T>(s, lvl + 1, Cd.b, cmean ? cb_slot : -1, nullptr, &ec_slot, &ec, prog, fuse_first);
  const double* ecmean = (singular_ && ec_slot >= 0) ? S_ + ec_slot : nullptr;
  // post-smoothing: the first sweep folds in the prolongation x += P e
  const XFetch<T> prolonged{buf[cur], mean[cur], static_cast<const T*>(ec), ecmean, C, Cd.h.fx, Cd.h.fy,
                            Cd.h.fz, D.d_xfb, D.d_xfo};
  const bool dots_here = !prog && lvl == 0 && fuse_dots_;  // level 0's last sweep forms z' and the PCG dots
  const auto kd = tpb_ == 128 ? k_smooth_dots<T, 128> : (tpb_ == 256 ? k_smooth_dots<T, 256> : k_smooth_dots<T, 512>);
  if (dots_here && sweeps_ == 1) {
    NB_LAUNCH(lc_, "smooth", s, ncell * (3 * tsz + 1) + ncoarse * tsz - ncell * tsz + ncell * 24,
              (launch_pdl(pdl_, kd, dim3(grid), dim3(tpb_), 0, s, L, b, prolonged, z_, rnew_, r_, rb_, S_, flags_,
                          maxit_, static_cast<T>(cheb_c2_[0]), T(0), 0, none)));
  } else {
    MG_EMIT("smooth", ncell * (2 * tsz + bsz + 1) + ncoarse * tsz,
            smooth_phase(prolonged, buf[cur ^ 1], mean[cur ^ 1], cheb_c2_[0], 0.0, 0, none),
            (launch_pdl(pdl_, ks, dim3(grid), dim3(tpb_), 0, s, L, b, bmean, prolonged, buf[cur ^ 1], rb_,
                        mean[cur ^ 1], inv_nf, flags_, maxit_, static_cast<T>(cheb_c2_[0]), T(0), 0, none, b16)));
  }
  cur ^= 1;
  for (int sw = 1; sw < sweeps_; ++sw, cur ^= 1) {  // Chebyshev: x_prev, after the prolongation with its coarse value
    const double bytes = ncell * (2 * tsz + bsz + 1) + (cheb_ ? ncell * tsz + (sw == 1 ? ncoarse * tsz : 0.0) : 0.0);
    if (dots_here && sw + 1 == sweeps_) {  // + z' and the PCG dots (no xout)
      NB_LAUNCH(lc_, "smooth", s, bytes - ncell * tsz + ncell * 24,
                (launch_pdl(pdl_, kd, dim3(grid), dim3(tpb_), 0, s, L, b, plain(cur), z_, rnew_, r_, rb_, S_, flags_,
                            maxit_, static_cast<T>(cheb_c2_[sw]), static_cast<T>(cheb_c1_[sw]), cheb_ ? 1 : 0,
                            sw == 1 ? prolonged : plain(cur ^ 1))));
      continue;
    }
    MG_EMIT("smooth", bytes,
            smooth_phase(plain(cur), buf[cur ^ 1], mean[cur ^ 1], cheb_c2_[sw], cheb_c1_[sw], cheb_ ? 1 : 0,
                         sw == 1 ? prolonged : plain(cur ^ 1)),
            (launch_pdl(pdl_, ks, dim3(grid), dim3(tpb_), 0, s, L, b, bmean, plain(cur), buf[cur ^ 1], rb_,
                        mean[cur ^ 1], inv_nf, flags_, maxit_, static_cast<T>(cheb_c2_[sw]),
                        static_cast<T>(cheb_c1_[sw]), cheb_ ? 1 : 0, sw == 1 ? prolonged : plain(cur ^ 1), b16)));
  }
#undef MG_EMIT
  *out_x = buf[cur];
  *out_mean_slot = sing ? lvl_slot(lvl, cur) : -1;
}

// Records the V-cycle from the first level (>= 1, above the coarsest) of at
// most tail_bricks_ bricks as one cluster program, with the levels' vectors
// placed in the CTAs' shared-memory arenas, when the device can hold the
// cluster; otherwise leaves the per-sweep launches in place.
void MgSolver::build_tail() {
  tail_lvl_ = -1;
  const int last = static_cast<int>(lv_.size()) - 1;
  if (tail_bricks_ <= 0) return;
  int t = -1;
  for (int l = 1; l < last; ++l)
    if (lv_[l].h.nbrick <= tail_bricks_) {
      t = l;
      break;
    }
  if (t < 0 || last - t + 1 > MAX_TAIL_LEV) return;
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  const size_t tsz = mixed ? sizeof(float) : sizeof(double);
  const size_t nco = static_cast<size_t>(lv_[last].v.nx) * lv_[last].v.ny * lv_[last].v.nz;
  const size_t scratch = dense_ ? sizeof(double) * dense_nf_ : coarse_smem(nco);
  const void* fn = mixed ? reinterpret_cast<const void*>(k_vtail<float>) : reinterpret_cast<const void*>(k_vtail<double>);
  int dev = 0, optin = 0;
  NB_CUDA(cudaGetDevice(&dev));
  NB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  NB_CUDA(cudaFuncGetAttributes(&fa, fn));
  // The dynamic shared-memory limit is a property of the kernel, shared by all
  // solvers: set it to the device maximum once rather than to this solver's need.
  const int dyn_max = optin - static_cast<int>(fa.sharedSizeBytes);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  // Arena of cluster size cs: b, x0, x1 of every tail level, ceil(nbrick / cs)
  // bricks each, 128-byte aligned.
  const auto arena_of = [&](int cs, std::vector<size_t>* offs) {
    size_t off = 0;
    for (int l = t; l <= last; ++l) {
      const size_t slots = static_cast<size_t>((lv_[l].h.nbrick + cs - 1) / cs);
      for (int v = 0; v < 3; ++v) {
        if (offs) offs->push_back(off);
        off += (slots * BR3 * tsz + 127) / 128 * 128;
      }
    }
    return off;
  };
  int lcs = 4;
  while (lcs > 1 && (1 << lcs) > lv_[t].h.nbrick) --lcs;
  size_t smem = 0;
  for (; lcs >= 1; --lcs) {  // largest power-of-two cluster the device schedules
    const int cs = 1 << lcs;
    smem = arena_of(cs, nullptr) + scratch;
    if (smem > static_cast<size_t>(dyn_max)) continue;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) == cudaSuccess && nclusters > 0) break;
    (void)cudaGetLastError();
  }
  if (lcs < 1) return;
  const int cs = 1 << lcs;
  std::vector<size_t> offs;
  const size_t arena = arena_of(cs, &offs);
  std::vector<TailPhase> ph;
  tail_lvl_ = t;
  tail_bytes_ = 0.0;
  const int bslot = (singular_ && lv_[t].h.nfluid > 0) ? lvl_slot(t, 2) : -1;
  if (mixed) vcycle<float>(nullptr, t, lv_[t].b, bslot, nullptr, &tail_slot_, &tail_x_, &ph);
  else vcycle<double>(nullptr, t, lv_[t].b, bslot, nullptr, &tail_slot_, &tail_x_, &ph);
  tail_lvl_ = -1;
  if (ph.size() > static_cast<size_t>(MAX_TAIL_PH)) return;
  // global vector -> arena encoding
  bool ok = true;
  const auto enc = [&](const void* g) -> uintptr_t {
    if (!g) return 0;
    for (int l = t; l <= last; ++l) {
      const void* v[3] = {lv_[l].b, lv_[l].x0, lv_[l].x1};
      for (int k = 0; k < 3; ++k)
        if (v[k] == g) return offs[3 * (l - t) + k] + kArenaBias;
    }
    ok = false;
    return 0;
  };
  const auto encp = [&](const void* g) { return reinterpret_cast<void*>(enc(g)); };
  for (TailPhase& q : ph) {
    q.b = encp(q.b);
    q.out = encp(q.out);
    for (TailFetch* f : {&q.X, &q.P}) {
      f->x = encp(f->x);
      f->ec = encp(f->ec);
    }
  }
  TailProg h{};
  h.nlev = last - t + 1;
  h.nphase = static_cast<int>(ph.size());
  h.singular = singular_ ? 1 : 0;
  h.nf = dense_ ? dense_nf_ : 0;
  h.lcs = lcs;
  h.nbrick = lv_[t].h.nbrick;
  h.arena_bytes = arena;
  h.b_in = lv_[t].b;
  h.b_enc = enc(lv_[t].b);
  h.x_out = tail_x_;
  h.x_enc = enc(tail_x_);
  if (!ok) return;
  h.inv = dense_inv_;
  h.fmap = dense_fmap_;
  h.lexpos = dense_lexpos_;
  h.lexcell = dense_lexcell_;
  h.xs = dense_ ? static_cast<double*>(alloc(sizeof(double) * std::max(dense_nf_, 1))) : nullptr;
  for (int l = 0; l < h.nlev; ++l) h.lv[l] = lv_[t + l].v;
  for (size_t i = 0; i < ph.size(); ++i) h.ph[i] = ph[i];
  tail_prog_ = static_cast<TailProg*>(alloc(sizeof(TailProg)));
  NB_CUDA(cudaMemcpy(tail_prog_, &h, sizeof(TailProg), cudaMemcpyHostToDevice));
  tail_lvl_ = t;
  tail_cs_ = cs;
  tail_smem_ = smem;
}

void MgSolver::launch_tail(cudaStream_t s) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(tail_cs_);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = tail_smem_;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = tail_cs_;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_ ? 2 : 1;
  const TailProg* prog = tail_prog_;
  if (precision_ == NB_PRECISION_MIXED)
    NB_LAUNCH(lc_, "vtail", s, tail_bytes_, NB_CUDA(cudaLaunchKernelEx(&cfg, k_vtail<float>, prog, flags_, maxit_)));
  else
    NB_LAUNCH(lc_, "vtail", s, tail_bytes_, NB_CUDA(cudaLaunchKernelEx(&cfg, k_vtail<double>, prog, flags_, maxit_)));
}

// BF16 residual storage: the levels below the finest and above the cluster
// tail (and above the coarsest level), per-sweep launches only.
void MgSolver::mark_bf16() {
  const int last = static_cast<int>(lv_.size()) - 1;
  for (int l = 0; l <= last; ++l)
    lv_[l].b16 = coarse_bf16_ && !grid_prog_ && l >= 1 && l < last && (tail_lvl_ < 0 || l < tail_lvl_);
}

// Records the whole V-cycle from level 0 (every level, the coarsest solve
// included) as one grid program when the device can hold a cooperative grid
// of the program's kernel; otherwise leaves the per-sweep launches in place.
void MgSolver::build_grid() {
  grid_prog_ = nullptr;
  if (!vgrid_) return;
  const int last = static_cast<int>(lv_.size()) - 1;
  if (last + 1 > MAX_GRID_LEV) return;
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  constexpr int GT = 256;  // threads per CTA: two cells per thread, four CTAs per SM
  const void* fn = mixed ? reinterpret_cast<const void*>(k_vgrid<float, GT>)
                         : reinterpret_cast<const void*>(k_vgrid<double, GT>);
  int dev = 0, nsm = 0, coop = 0;
  NB_CUDA(cudaGetDevice(&dev));
  NB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  NB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return;
  const size_t nco = static_cast<size_t>(lv_[last].v.nx) * lv_[last].v.ny * lv_[last].v.nz;
  // the phase count of a V-cycle over these levels (recorded below)
  std::vector<TailPhase> ph;
  {
    const int saved_tail = tail_lvl_;
    tail_lvl_ = 0;  // phases' levels relative to level 0; no cluster tail inside
    const double saved_bytes = tail_bytes_;
    tail_bytes_ = 0.0;
    if (mixed) vcycle<float>(nullptr, 0, rnew_f_, -1, nullptr, &grid_slot_, &grid_x_, &ph);
    else vcycle<double>(nullptr, 0, rnew_, -1, nullptr, &grid_slot_, &grid_x_, &ph);
    grid_bytes_ = tail_bytes_;
    tail_bytes_ = saved_bytes;
    tail_lvl_ = saved_tail;
  }
  if (ph.size() > static_cast<size_t>(MAX_GRID_PH)) return;
  static_assert(sizeof(LevelView) % 8 == 0 && sizeof(TailPhase) % 8 == 0, "program staged in 8-byte units");
  const size_t smem = sizeof(LevelView) * (last + 1) + sizeof(TailPhase) * ph.size() +
                      (dense_ ? sizeof(double) * dense_nf_ : coarse_smem(nco));
  int optin = 0;
  NB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  NB_CUDA(cudaFuncGetAttributes(&fa, fn));
  if (smem + fa.sharedSizeBytes > static_cast<size_t>(optin)) return;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - static_cast<int>(fa.sharedSizeBytes)) !=
          cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, GT, smem) != cudaSuccess || per_sm < 1) {
    (void)cudaGetLastError();
    return;
  }
  // no more CTAs than the largest level has bricks, and never more than can be resident
  int widest = 1;
  for (const DevLevel& D : lv_) widest = std::max(widest, D.h.nbrick);
  const int ctas = std::min(per_sm * nsm, std::min(widest, MAX_GRID));
  GridProg h{};
  h.nlev = last + 1;
  h.nphase = static_cast<int>(ph.size());
  h.singular = singular_ ? 1 : 0;
  h.nf = dense_ ? dense_nf_ : 0;
  h.inv = dense_inv_;
  h.fmap = dense_fmap_;
  h.lexpos = dense_lexpos_;
  h.lexcell = dense_lexcell_;
  h.xs = dense_ ? static_cast<double*>(alloc(sizeof(double) * dense_nf_)) : nullptr;
  grid_sync_ = static_cast<unsigned*>(alloc(2 * sizeof(unsigned)));
  NB_CUDA(cudaMemset(grid_sync_, 0, 2 * sizeof(unsigned)));
  h.sync = grid_sync_;
  h.partials = static_cast<double*>(alloc(2 * sizeof(double) * ctas));
  h.flags = flags_;
  for (int l = 0; l <= last; ++l) h.lv[l] = lv_[l].v;
  for (size_t q = 0; q < ph.size(); ++q) h.ph[q] = ph[q];
  GridProg* d = static_cast<GridProg*>(alloc(sizeof(GridProg)));
  NB_CUDA(cudaMemcpy(d, &h, sizeof(GridProg), cudaMemcpyHostToDevice));
  grid_b_ = mixed ? static_cast<const void*>(rnew_f_) : static_cast<const void*>(rnew_);
  grid_prog_alt_ = nullptr;
  if (!mixed) {
    // FP64: the V-cycle reads rnew in place and the PCG swaps r and rnew every
    // cycle, so a second program reads the other buffer
    for (int q = 0; q < h.nphase; ++q)
      if (h.ph[q].b == rnew_) h.ph[q].b = r_;
    grid_prog_alt_ = static_cast<GridProg*>(alloc(sizeof(GridProg)));
    NB_CUDA(cudaMemcpy(grid_prog_alt_, &h, sizeof(GridProg), cudaMemcpyHostToDevice));
  }
  grid_prog_ = d;
  grid_ctas_ = ctas;
  grid_smem_ = smem;
}

// One grid V-cycle: the barrier counters are zeroed by a memset node, then the
// cooperative launch (no programmatic overlap: its CTAs must all be resident).
void MgSolver::launch_grid(cudaStream_t s, const void* b) {
  NB_CUDA(cudaMemsetAsync(grid_sync_, 0, 2 * sizeof(unsigned), s));  // arrivals and the abort flag
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid_ctas_);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = grid_smem_;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  const GridProg* prog = (mixed || b == grid_b_) ? grid_prog_ : grid_prog_alt_;
  if (mixed)
    NB_LAUNCH(lc_, "vgrid", s, grid_bytes_, NB_CUDA(cudaLaunchKernelEx(&cfg, k_vgrid<float, 256>, prog, flags_, maxit_)));
  else
    NB_LAUNCH(lc_, "vgrid", s, grid_bytes_, NB_CUDA(cudaLaunchKernelEx(&cfg, k_vgrid<double, 256>, prog, flags_, maxit_)));
}

// Minv: z = V-cycle(r) (+ Minv's removeMean), then either p = z, rz = r.z
// (first) or the flexible-beta dots, then p = z + beta p.
void MgSolver::iterate(cudaStream_t s, double tol, int maxit, int count) {
  const LevelView& L = lv_[0].v;
  const int grid = grid_of(L.nbrick);
  const double inv_nf = lv_[0].h.nfluid ? 1.0 / lv_[0].wfluid : 0.0;
  const bool sing = singular_ && lv_[0].h.nfluid > 0;
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  const double n = lv_[0].ncell;
  const double zsz = mixed ? 4.0 : 8.0;
  const auto km = tpb_ == 128 ? k_pcg_matvec<128> : (tpb_ == 256 ? k_pcg_matvec<256> : k_pcg_matvec<512>);
  for (int k = 0; k < count; ++k) {
    // p_ holds the last direction, p2_ receives this cycle's (swapped below)
    NB_LAUNCH(lc_, "pcg_matvec", s, n * 33,
              launch_pdl(pdl_, km, dim3(grid), dim3(tpb_), 0, s, L, z_, p_, p2_, Ap_, rb_, S_, flags_, maxit));
    // non-singular systems whose level 0 smooths by launches: the update also
    // writes level 0's first sweep (the V-cycle then starts at its second)
    const bool first0 = !sing && !grid_prog_ && lv_.size() > 1 && tail_lvl_ != 0;
    NB_LAUNCH(lc_, "pcg_update", s, n * (48 + (sing ? 1 : 0) + (mixed && !sing ? 4 : 0) + (first0 ? zsz + 2 : 0)),
              (launch_pdl(pdl_, k_pcg_update, dim3(grid), dim3(NT), 0, s, L, x_, p2_, r_, Ap_, rnew_,
                          mixed ? rnew_f_ : nullptr, sing ? 1 : 0, inv_nf, rb_, S_, flags_, maxit, tol,
                          first0 ? lv_[0].x0 : nullptr, cheb_c2_[0])));
    if (sing) {
      NB_LAUNCH(lc_, "pcg_center", s, n * (17 + (mixed ? 4 : 0)),
                (launch_pdl(pdl_, k_pcg_center, dim3(grid), dim3(NT), 0, s, L, rnew_, mixed ? rnew_f_ : nullptr, rb_, S_, flags_, maxit,
                                                  tol)));
    }
    void* zx = nullptr;
    int zslot = -1;
    const bool fused = !sing && !grid_prog_;
    if (grid_prog_) {
      launch_grid(s, mixed ? static_cast<const void*>(rnew_f_) : static_cast<const void*>(rnew_));
      zx = grid_x_;
      zslot = grid_slot_;
    } else {
      // non-singular: the V-cycle's last sweep also forms z' and the dots
      fuse_dots_ = !sing;
      if (mixed) vcycle<float>(s, 0, rnew_f_, -1, nullptr, &zslot, &zx, nullptr, first0);
      else vcycle<double>(s, 0, rnew_, -1, nullptr, &zslot, &zx, nullptr, first0);
      fuse_dots_ = false;
    }
    std::swap(p_, p2_);
    if (fused) {
      std::swap(r_, rnew_);
      continue;
    }
    const double* m1 = (sing && zslot >= 0) ? S_ + zslot : nullptr;
    const double* m2 = sing ? S_ + S_ZMEAN2 : nullptr;
    if (sing) {
      if (mixed)
        NB_LAUNCH(lc_, "pcg_mean", s, n * (zsz + 1),
                  (launch_pdl(pdl_, k_fluid_mean_f, dim3(grid), dim3(NT), 0, s,L, static_cast<const float*>(zx), m1, rb_, S_ + S_ZMEAN2,
                                                      inv_nf, flags_, maxit)));
      else
        NB_LAUNCH(lc_, "pcg_mean", s, n * (zsz + 1),
                  (launch_pdl(pdl_, k_fluid_mean, dim3(grid), dim3(NT), 0, s,L, static_cast<const double*>(zx), m1, rb_, S_ + S_ZMEAN2,
                                                    inv_nf, flags_, maxit)));
    }
    if (mixed)
      NB_LAUNCH(lc_, "pcg_dots", s, n * (zsz + 8 * 3 + 1),
                (launch_pdl(pdl_, k_pcg_dots<float>, dim3(grid), dim3(NT), 0, s,L, static_cast<const float*>(zx), m1, m2, z_, p_, rnew_,
                                                       r_, 0, rb_, S_, flags_, maxit)));
    else
      NB_LAUNCH(lc_, "pcg_dots", s, n * (zsz + 8 * 3 + 1),
                (launch_pdl(pdl_, k_pcg_dots<double>, dim3(grid), dim3(NT), 0, s,L, static_cast<const double*>(zx), m1, m2, z_, p_,
                                                        rnew_, r_, 0, rb_, S_, flags_, maxit)));
    std::swap(r_, rnew_);
  }
  NB_CUDA(cudaGetLastError());
}

void MgSolver::solve_async(cudaStream_t s, const double* b, double tol, int maxit, double* report,
                           const WarmStart* ws) {
  setup(s, b, tol, maxit, ws);
  // Iterate in batches; every kernel returns at once after convergence, so
  // over-issuing costs only launch latency. The batch grows geometrically.
  // The mixed form then checks the true residual and may restart (outer
  // iterative refinement, at most kMaxRefine times).
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  const LevelView& L = lv_[0].v;
  const int grid = grid_of(L.nbrick);
  const bool sing = singular_ && lv_[0].h.nfluid > 0;
  const double inv_nf = lv_[0].h.nfluid ? 1.0 / lv_[0].wfluid : 0.0;
  int issued = 0, batch = 4;
  for (int round = 0;; ++round) {
    while (issued < maxit) {
      const int cnt = std::min(batch, maxit - issued + (maxit - issued) % 2);
      iterate(s, tol, maxit, cnt);
      issued += cnt;
      NB_CUDA(cudaMemcpyAsync(h_flags_, flags_, sizeof(SolveFlags), cudaMemcpyDeviceToHost, s));
      NB_CUDA(cudaStreamSynchronize(s));
      if (h_flags_->stop != 0 || h_flags_->iters >= maxit) break;
      batch = std::min(batch * 2, 16);
    }
    if (!mixed || round >= kMaxRefine) break;
    NB_LAUNCH(lc_, "ir_residual", s, lv_[0].ncell * 27,
              (k_ir_residual<<<grid, NT, 0, s>>>(L, x_, rhs_, rnew_, rb_, S_, flags_, tol, maxit, inv_nf, 0, 0, 0)));
    NB_CUDA(cudaMemcpyAsync(h_flags_, flags_, sizeof(SolveFlags), cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaStreamSynchronize(s));
    if (h_flags_->stop != 0 || h_flags_->iters >= maxit) break;  // no restart (converged on the true residual too)
    k_ir_restart<<<grid, NT, 0, s>>>(L, rnew_, r_, rnew_f_, S_, flags_, sing ? 1 : 0, maxit);
    lc_.add();
    first_direction(s);
  }
  finish(s, report);
}

// Graph form: the cycle loop is a conditional WHILE node whose body runs two
// cycles (so the r/rnew buffers return to their captured roles) and then sets
// the loop condition on the device. Must be called while `s` is capturing.
void MgSolver::capture_solve(cudaStream_t s, const double* b, double tol, int maxit, double* report,
                             uint64_t* body_kernels, const WarmStart* ws) {
  setup(s, b, tol, maxit, ws);
  cudaStreamCaptureStatus st;
  cudaGraph_t g;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  NB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  cudaGraphConditionalHandle h;
  NB_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  NB_LAUNCH(lc_, "set_cond", s, 0, (k_set_cond<<<1, 1, 0, s>>>(h, flags_, maxit, nullptr)));
  NB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  NB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  cudaGraph_t body = p.conditional.phGraph_out[0];
  if (!side_) NB_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  std::atomic<uint64_t>* saved = lc_.count;
  std::atomic<uint64_t> nbody{0};
  lc_.count = &nbody;
  NB_CUDA(cudaStreamBeginCaptureToGraph(side_, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  iterate(side_, tol, maxit, 2);
  NB_LAUNCH(lc_, "set_cond", side_, 0, (k_set_cond<<<1, 1, 0, side_>>>(h, flags_, maxit, body_execs_)));
  cudaGraph_t body_out = nullptr;
  NB_CUDA(cudaStreamEndCapture(side_, &body_out));
  lc_.count = saved;
  if (body_kernels) *body_kernels = nbody.load();
  NB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  if (precision_ == NB_PRECISION_MIXED)
    for (int k = 0; k < kMaxRefine; ++k) capture_refinement(s, tol, maxit);
  finish(s, report);
}

// Outer iterative refinement inside the captured solve (mixed form): the true
// residual decides (k_ir_residual), an IF node holds the restart (residual,
// first direction) and a second WHILE node the cycles after it. Their bodies'
// kernels run only after a restart and are not counted as launches of a
// normal solve.
void MgSolver::capture_refinement(cudaStream_t s, double tol, int maxit) {
  const LevelView& L = lv_[0].v;
  const int grid = grid_of(L.nbrick);
  const bool sing = singular_ && lv_[0].h.nfluid > 0;
  const double inv_nf = lv_[0].h.nfluid ? 1.0 / lv_[0].wfluid : 0.0;
  cudaStreamCaptureStatus st;
  cudaGraph_t g;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  NB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  cudaGraphConditionalHandle h_if, h_loop;
  NB_CUDA(cudaGraphConditionalHandleCreate(&h_if, g, 0, cudaGraphCondAssignDefault));
  NB_CUDA(cudaGraphConditionalHandleCreate(&h_loop, g, 0, cudaGraphCondAssignDefault));
  NB_LAUNCH(lc_, "ir_residual", s, lv_[0].ncell * 27,
            (k_ir_residual<<<grid, NT, 0, s>>>(L, x_, rhs_, rnew_, rb_, S_, flags_, tol, maxit, inv_nf, 1, h_if,
                                                h_loop)));
  std::atomic<uint64_t>* saved = lc_.count;
  std::atomic<uint64_t> rare{0};
  // IF: the restart
  NB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams pi{};
  pi.type = cudaGraphNodeTypeConditional;
  pi.conditional.handle = h_if;
  pi.conditional.type = cudaGraphCondTypeIf;
  pi.conditional.size = 1;
  cudaGraphNode_t if_node;
  NB_CUDA(cudaGraphAddNode(&if_node, g, deps, nd, &pi));
  lc_.count = &rare;
  NB_CUDA(cudaStreamBeginCaptureToGraph(side_, pi.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeRelaxed));
  k_ir_restart<<<grid, NT, 0, side_>>>(L, rnew_, r_, rnew_f_, S_, flags_, sing ? 1 : 0, maxit);
  first_direction(side_);
  cudaGraph_t out = nullptr;
  NB_CUDA(cudaStreamEndCapture(side_, &out));
  // WHILE: the cycles after a restart
  cudaGraphNodeParams pw{};
  pw.type = cudaGraphNodeTypeConditional;
  pw.conditional.handle = h_loop;
  pw.conditional.type = cudaGraphCondTypeWhile;
  pw.conditional.size = 1;
  cudaGraphNode_t loop_node;
  NB_CUDA(cudaGraphAddNode(&loop_node, g, &if_node, 1, &pw));
  NB_CUDA(cudaStreamBeginCaptureToGraph(side_, pw.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeRelaxed));
  iterate(side_, tol, maxit, 2);
  k_set_cond<<<1, 1, 0, side_>>>(h_loop, flags_, maxit, nullptr);
  NB_CUDA(cudaStreamEndCapture(side_, &out));
  lc_.count = saved;
  NB_CUDA(cudaStreamUpdateCaptureDependencies(s, &loop_node, 1, cudaStreamSetCaptureDependencies));
}

void MgSolver::finish(cudaStream_t s, double* report) {
  const LevelView& L = lv_[0].v;
  const int grid = grid_of(L.nbrick);
  const double inv_nf = lv_[0].h.nfluid ? 1.0 / lv_[0].wfluid : 0.0;
  const bool sing = singular_ && lv_[0].h.nfluid > 0;
  // final removeMean(x) + true residual (multigrid.cpp:341-353)
  if (sing) {
    k_fluid_mean<<<grid, NT, 0, s>>>(L, x_, nullptr, rb_, S_ + S_XMEAN, inv_nf, nullptr, maxit_);
    lc_.add();
  }
  k_true_residual<<<grid, NT, 0, s>>>(L, x_, sing ? S_ + S_XMEAN : nullptr, rhs_, xfin_, rb_, S_);
  lc_.add();
  if (report) {
    k_report<<<1, 1, 0, s>>>(flags_, S_, report);
    lc_.add();
  }
  NB_CUDA(cudaGetLastError());
}

nb_poisson_report MgSolver::report_from(const double* r, double tol) {
  nb_poisson_report rep{};
  const double bnorm = std::sqrt(r[3]) + 1e-300;
  if (r[2] != 0.0) {  // early exit: rhs already below tolerance
    rep.iterations = 0;
    rep.residual = std::sqrt(r[3]) / bnorm;
    rep.converged = 1;
    return rep;
  }
  rep.iterations = static_cast<int>(r[0]);
  rep.residual = std::sqrt(r[4]) / bnorm;
  rep.converged = (r[1] == 1.0 || rep.residual <= tol) ? 1 : 0;
  return rep;
}

void MgSolver::setup(cudaStream_t s, const double* b, double tol, int maxit, const WarmStart* ws) {
  tol_ = tol;
  maxit_ = maxit;
  const LevelView& L = lv_[0].v;
  const int grid = grid_of(L.nbrick);
  const double inv_nf = lv_[0].h.nfluid ? 1.0 / lv_[0].wfluid : 0.0;
  const bool sing = singular_ && lv_[0].h.nfluid > 0;
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  // rhs = b masked (+ mean removal), r = rhs, x = 0, bnorm, early exit
  if (sing) {
    k_fluid_mean<<<grid, NT, 0, s>>>(L, b, nullptr, rb_, S_ + S_BSUM, inv_nf, nullptr, maxit);
    lc_.add();
  }
  if (ws)
    k_pcg_setup_warm<<<grid, NT, 0, s>>>(L, b, sing ? S_ + S_BSUM : nullptr, ws->guess, ws->dt, ws->alpha, ws->h1,
                                         ws->h2, ws->h3, ws->k2, ws->k3, ws->nhist, rhs_, r_, x_, mixed ? rnew_f_ : nullptr, rb_, S_, flags_,
                                         tol);
  else
    k_pcg_setup<<<grid, NT, 0, s>>>(L, b, sing ? S_ + S_BSUM : nullptr, rhs_, r_, x_,
                                    mixed ? rnew_f_ : nullptr, rb_, S_, flags_, tol);
  lc_.add();
  first_direction(s);
}

// z = Minv(r) ; p = z ; rz = r.z (the first cycle, and every refinement restart)
void MgSolver::first_direction(cudaStream_t s) {
  const LevelView& L = lv_[0].v;
  const int grid = grid_of(L.nbrick);
  const double inv_nf = lv_[0].h.nfluid ? 1.0 / lv_[0].wfluid : 0.0;
  const bool sing = singular_ && lv_[0].h.nfluid > 0;
  const bool mixed = precision_ == NB_PRECISION_MIXED;
  const int maxit = maxit_;
  void* zx = nullptr;
  int zslot = -1;
  if (grid_prog_) {
    launch_grid(s, mixed ? static_cast<const void*>(rnew_f_) : static_cast<const void*>(r_));
    zx = grid_x_;
    zslot = grid_slot_;
  } else if (mixed) {
    vcycle<float>(s, 0, rnew_f_, -1, nullptr, &zslot, &zx);
  } else {
    vcycle<double>(s, 0, r_, -1, nullptr, &zslot, &zx);
  }
  const double* m1 = (sing && zslot >= 0) ? S_ + zslot : nullptr;
  const double* m2 = sing ? S_ + S_ZMEAN2 : nullptr;
  if (sing) {
    if (mixed)
      k_fluid_mean_f<<<grid, NT, 0, s>>>(L, static_cast<const float*>(zx), m1, rb_, S_ + S_ZMEAN2, inv_nf,
                                         flags_, maxit);
    else
      k_fluid_mean<<<grid, NT, 0, s>>>(L, static_cast<const double*>(zx), m1, rb_, S_ + S_ZMEAN2, inv_nf,
                                       flags_, maxit);
    lc_.add();
  }
  if (mixed)
    k_pcg_dots<float><<<grid, NT, 0, s>>>(L, static_cast<const float*>(zx), m1, m2, z_, p_, r_, r_, 1, rb_,
                                          S_, flags_, maxit);
  else
    k_pcg_dots<double><<<grid, NT, 0, s>>>(L, static_cast<const double*>(zx), m1, m2, z_, p_, r_, r_, 1,
                                           rb_, S_, flags_, maxit);
  lc_.add();
  NB_CUDA(cudaGetLastError());
}

bool MgSolver::timed_out() const { return h_flags_ && h_flags_->stop == STOP_TIMEOUT; }

nb_poisson_report MgSolver::fetch_report(cudaStream_t s) {
  NB_CUDA(cudaMemcpyAsync(h_flags_, flags_, sizeof(SolveFlags), cudaMemcpyDeviceToHost, s));
  NB_CUDA(cudaMemcpyAsync(h_S_, S_, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, s));
  NB_CUDA(cudaStreamSynchronize(s));
  const double r[6] = {static_cast<double>(h_flags_->iters), static_cast<double>(h_flags_->stop),
                       static_cast<double>(h_flags_->early), h_S_[S_BNORM2], h_S_[S_TRUERES2],
                       static_cast<double>(h_flags_->nan)};
  return report_from(r, tol_);
}

void MgSolver::solve(cudaStream_t s, const double* b, double tol, int maxit) {
  solve_async(s, b, tol, maxit);
}

template void MgSolver::vcycle<double>(cudaStream_t, int, const void*, int, void*, int*, void**,
                                       std::vector<TailPhase>*, bool);
template void MgSolver::vcycle<float>(cudaStream_t, int, const void*, int, void*, int*, void**,
                                      std::vector<TailPhase>*, bool);

}  // namespace nb
