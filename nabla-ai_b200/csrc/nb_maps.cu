// nb_maps.cu — the integer maps of octree brick meshes, built on the device
// and exported from the host tree, for bit-exact comparison with the
// reference's Octree.
//
// Device builder (nb_amr_build_maps), for a leaf list in any order:
//   1. k_keys: the Morton key of every leaf's anchor on the finest level
//      (core/include/nabla/mesh/morton.hpp:19-48, through nb_morton.h),
//      paired with its input position; coordinates are range-checked.
//   2. a bitonic sort of the (key, position) pairs over the next power of two
//      (padding keys are all ones): the rank order of the mesh.
//   3. k_unique: two leaves with one anchor are an error.
//   4. k_face_nbrs: per (rank, face) the rule of Octree::faceNeighborsOf
//      (core/src/mesh/octree.cpp:229-277) at brick granularity: the coarser-
//      or-equal leaf that holds the brick across the face, else the 2x2 leaves
//      one level finer on the touching side, listed k1 over axis (a+1)%3
//      outer, k2 over axis (a+2)%3 inner as the reference lists them. Lookups
//      are binary searches in the sorted keys (a key matches only at its own
//      level), where the reference uses a hash map. Periodic axes wrap; a face
//      on a non-periodic domain boundary has no neighbour.
// Host export (nb_amr_mesh_maps): the same table from a mesh's own tree, its
// rank order and per-level lookup tables (the maps the flow and multigrid
// kernels are built from), so the two routes check each other.
// Device refinement (nb_amr_refine_device, nb_amr_case_refine): split marks by
// rank, rounds of 26-neighbour 2:1 balance through the same binary searches,
// a one-CTA scan of the output counts, the children emitted, then ranked by
// the same sort.
#include <algorithm>
#include <string>
#include <vector>

#include "nb_amr.h"
#include "nb_amr_level.h"
#include "nb_amr_mesh.h"
#include "nb_ctx.h"
#include "nb_maps.h"
#include "nb_morton.h"

using namespace nb;

namespace {

struct MapGeom {
  int nb0[3];
  int lmax;
  int per[3];
};

constexpr unsigned long long kPadKey = ~0ull;

__global__ void k_keys(int n, int npad, const int4* __restrict__ leaves, MapGeom g, unsigned long long* keys,
                       int* pos, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npad) return;
  if (i >= n) {
    keys[i] = kPadKey;
    pos[i] = -1;
    return;
  }
  const int4 f = leaves[i];
  const int L = f.x;
  bool ok = L >= 0 && L <= g.lmax;
  const int b[3] = {f.y, f.z, f.w};
  for (int a = 0; a < 3 && ok; ++a) ok = b[a] >= 0 && b[a] < (g.nb0[a] << L);
  if (!ok) {
    atomicExch(err, 2);
    keys[i] = kPadKey;
    pos[i] = i;
    return;
  }
  const int s = g.lmax - L;
  keys[i] = morton_encode(static_cast<uint32_t>(b[0]) << s, static_cast<uint32_t>(b[1]) << s,
                          static_cast<uint32_t>(b[2]) << s);
  pos[i] = i;
}

// One compare-exchange stage (j, k) of the bitonic network over npad pairs.
__global__ void k_bitonic(int npad, int j, int k, unsigned long long* keys, int* pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npad) return;
  const int l = i ^ j;
  if (l <= i) return;
  const bool up = (i & k) == 0;
  const unsigned long long a = keys[i], b = keys[l];
  if ((a > b) == up) {
    keys[i] = b;
    keys[l] = a;
    const int t = pos[i];
    pos[i] = pos[l];
    pos[l] = t;
  }
}

__global__ void k_unique(int n, const unsigned long long* keys, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 1 && i < n && keys[i] == keys[i - 1]) atomicExch(err, 1);
}

// Rank of the leaf at `level` whose anchor key is `key`, or -1.
__device__ int find_leaf(const unsigned long long* keys, const int* lev, int n, unsigned long long key, int level) {
  int lo = 0, hi = n;
  while (lo < hi) {  // lower bound: at most log2(n) + 1 rounds
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return (lo < n && keys[lo] == key && lev[lo] == level) ? lo : -1;
}

__global__ void k_ranked(int n, const int* pos, const int4* __restrict__ leaves, int4* ranked, int* lev) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int4 f = leaves[pos[r]];
  ranked[r] = f;
  lev[r] = f.x;
}

__global__ void k_face_nbrs(int n, const unsigned long long* keys, const int4* ranked, const int* lev, MapGeom g,
                            int* nbr, int* nnbr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * n) return;
  const int r = t / 6, d = t % 6, a = d >> 1, sgn = (d & 1) ? 1 : -1;
  const int4 f = ranked[r];
  const int L = f.x;
  int c[3] = {f.y, f.z, f.w};
  c[a] += sgn;
  int cnt = 0;
  int out[4] = {-1, -1, -1, -1};
  const int ext = g.nb0[a] << L;
  bool inside = true;
  if (c[a] < 0 || c[a] >= ext) {
    if (g.per[a]) c[a] = (c[a] + ext) % ext;
    else inside = false;
  }
  if (inside) {
    for (int l = L; l >= 0 && cnt == 0; --l) {
      const int s = L - l, u = g.lmax - l;
      const unsigned long long key =
          morton_encode(static_cast<uint32_t>(c[0] >> s) << u, static_cast<uint32_t>(c[1] >> s) << u,
                        static_cast<uint32_t>(c[2] >> s) << u);
      const int q = find_leaf(keys, lev, n, key, l);
      if (q >= 0) out[cnt++] = q;
    }
    if (cnt == 0 && L + 1 <= g.lmax) {
      const int t1 = (a + 1) % 3, t2 = (a + 2) % 3, u = g.lmax - L - 1;
      for (int k1 = 0; k1 < 2; ++k1)
        for (int k2 = 0; k2 < 2; ++k2) {
          int ch[3];
          ch[a] = sgn > 0 ? 2 * c[a] : 2 * c[a] + 1;
          ch[t1] = 2 * c[t1] + k1;
          ch[t2] = 2 * c[t2] + k2;
          const unsigned long long key =
              morton_encode(static_cast<uint32_t>(ch[0]) << u, static_cast<uint32_t>(ch[1]) << u,
                            static_cast<uint32_t>(ch[2]) << u);
          const int q = find_leaf(keys, lev, n, key, L + 1);
          if (q >= 0) out[cnt++] = q;
        }
    }
  }
  nnbr[t] = cnt;
  for (int q = 0; q < 4; ++q) nbr[4 * t + q] = out[q];
}

// ---- refinement on the device ----------------------------------------------
// The leaf of level <= L holding level-L brick c (coarser-or-equal search),
// or -1 when finer leaves cover it.
__device__ int holder(const unsigned long long* keys, const int* lev, int n, const MapGeom& g, int L, const int c[3]) {
  for (int l = L; l >= 0; --l) {
    const int s = L - l, u = g.lmax - l;
    const unsigned long long key = morton_encode(static_cast<uint32_t>(c[0] >> s) << u,
                                                 static_cast<uint32_t>(c[1] >> s) << u,
                                                 static_cast<uint32_t>(c[2] >> s) << u);
    const int q = find_leaf(keys, lev, n, key, l);
    if (q >= 0) return q;
  }
  return -1;
}

// Split marks by rank: mark[r] = flag of the input leaf, below lmax only.
__global__ void k_rank_marks(int n, const int* pos, const uint8_t* flags, const int* lev, int lmax, uint8_t* mark) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) mark[r] = (flags[pos[r]] != 0 && lev[r] < lmax) ? 1 : 0;
}

// One round of 26-neighbour 2:1 balance: a leaf that splits (children at
// L+1) forces every touching leaf of level <= L-1 to split too (the closure
// nb_amr_refine's host balance reaches; Octree::refineByMorton's rule,
// core/src/mesh/octree.cpp:325-356, over faces, edges and corners).
__global__ void k_balance_round(int n, const unsigned long long* keys, const int4* ranked, const int* lev, MapGeom g,
                                uint8_t* mark, int* changed) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || !mark[r]) return;
  const int4 f = ranked[r];
  const int L = f.x;
  if (L == 0) return;
  for (int d = 0; d < 27; ++d) {
    if (d == 13) continue;
    int c[3] = {f.y + d % 3 - 1, f.z + (d / 3) % 3 - 1, f.w + d / 9 - 1};
    bool inside = true;
    for (int a = 0; a < 3; ++a) {
      const int ext = g.nb0[a] << L;
      if (c[a] < 0 || c[a] >= ext) {
        if (g.per[a]) c[a] = (c[a] + ext) % ext;
        else inside = false;
      }
    }
    if (!inside) continue;
    const int q = holder(keys, lev, n, g, L, c);
    if (q >= 0 && lev[q] <= L - 1 && !mark[q]) {
      mark[q] = 1;
      *changed = 1;
    }
  }
}

// Exclusive scan of the output counts (8 for a split leaf, 1 otherwise) in
// one CTA: each thread sums a contiguous run of ranks, the CTA scans the run
// sums, each thread writes its run's offsets. total[0] = the new leaf count.
__global__ void __launch_bounds__(1024) k_emit_offsets(int n, const uint8_t* mark, int* off, int* total) {
  __shared__ int sums[1024];
  const int t = threadIdx.x, per = (n + 1023) / 1024;
  const int lo = min(n, t * per), hi = min(n, lo + per);
  int acc = 0;
  for (int r = lo; r < hi; ++r) acc += mark[r] ? 8 : 1;
  sums[t] = acc;
  __syncthreads();
  for (int w = 1; w < 1024; w <<= 1) {  // inclusive Hillis-Steele scan
    const int v = t >= w ? sums[t - w] : 0;
    __syncthreads();
    sums[t] += v;
    __syncthreads();
  }
  int run = t ? sums[t - 1] : 0;
  for (int r = lo; r < hi; ++r) {
    off[r] = run;
    run += mark[r] ? 8 : 1;
  }
  if (t == 1023) *total = sums[1023];
}

__global__ void k_emit_leaves(int n, const int4* ranked, const uint8_t* mark, const int* off, int4* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int4 f = ranked[r];
  if (!mark[r]) {
    out[off[r]] = f;
    return;
  }
  for (int o = 0; o < 8; ++o)
    out[off[r] + o] = make_int4(f.x + 1, 2 * f.y + (o & 1), 2 * f.z + ((o >> 1) & 1), 2 * f.w + (o >> 2));
}

// Marks from a per-leaf sensor array (4 values per leaf in rank order).
__global__ void k_sensor_marks(int n, const double* sensors, int which, double above, const int4* ranked, int lmax,
                               uint8_t* flags) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) flags[r] = (sensors[4 * r + which] > above && ranked[r].x < lmax) ? 1 : 0;
}

MapGeom map_geom(const nb_amr_geom& g) {
  MapGeom m{};
  for (int a = 0; a < 3; ++a) {
    m.nb0[a] = g.nb0[a];
    m.per[a] = g.face[2 * a].type == NB_BC_PERIODIC;
  }
  m.lmax = g.lmax;
  return m;
}

bool map_geom_ok(const nb_amr_geom* g) {
  if (!g || g->lmax < 0 || g->lmax >= AMR_MAXLEV) return false;
  for (int a = 0; a < 3; ++a)
    if (g->nb0[a] < 1 || (static_cast<long long>(g->nb0[a]) << g->lmax) > (1 << 17)) return false;
  return true;
}

// The host tree's table: the same rule through the per-level lookup tables.
void host_face_nbrs(const AmrTree& t, int r, int d, int out[4], int& cnt) {
  const AmrLeaf& f = t.leaves[r];
  const int a = d >> 1, sgn = (d & 1) ? 1 : -1, L = f.level;
  int c[3] = {f.b[0], f.b[1], f.b[2]};
  c[a] += sgn;
  cnt = 0;
  for (int q = 0; q < 4; ++q) out[q] = -1;
  const int ext = t.lnb(L, a);
  if (c[a] < 0 || c[a] >= ext) {
    if (t.geom.bc[2 * a] != NB_BC_PERIODIC) return;
    c[a] = (c[a] + ext) % ext;
  }
  for (int l = L; l >= 0; --l) {
    const int s = L - l;
    const int q = t.find(l, c[0] >> s, c[1] >> s, c[2] >> s);
    if (q >= 0 && t.leaves[q].level == l) {
      out[cnt++] = q;
      return;
    }
  }
  if (L + 1 >= t.nlev) return;
  const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
  for (int k1 = 0; k1 < 2; ++k1)
    for (int k2 = 0; k2 < 2; ++k2) {
      int ch[3];
      ch[a] = sgn > 0 ? 2 * c[a] : 2 * c[a] + 1;
      ch[t1] = 2 * c[t1] + k1;
      ch[t2] = 2 * c[t2] + k2;
      const int q = t.find(L + 1, ch[0], ch[1], ch[2]);
      if (q >= 0) out[cnt++] = q;
    }
}

// Keys, ranked leaves (optional) and the face-neighbour table of a host tree.
void export_tree_maps(const AmrTree& t, uint64_t* keys, int32_t* ranked, int32_t* nbr, int32_t* nnbr) {
  const int lmax = t.geom.lmax;
  for (size_t r = 0; r < t.leaves.size(); ++r) {
    const AmrLeaf& f = t.leaves[r];
    const int s = lmax - f.level;
    keys[r] = morton_encode(static_cast<uint32_t>(f.b[0]) << s, static_cast<uint32_t>(f.b[1]) << s,
                            static_cast<uint32_t>(f.b[2]) << s);
    if (ranked) {
      ranked[4 * r] = f.level;
      for (int a = 0; a < 3; ++a) ranked[4 * r + 1 + a] = f.b[a];
    }
    for (int d = 0; d < 6; ++d) {
      int out[4], cnt = 0;
      host_face_nbrs(t, static_cast<int>(r), d, out, cnt);
      nnbr[6 * r + d] = cnt;
      for (int q = 0; q < 4; ++q) nbr[24 * r + 4 * d + q] = out[q];
    }
  }
}

// Device buffers of one call, freed after the stream has drained.
class DevArena {
 public:
  explicit DevArena(cudaStream_t s) : s_(s) {}
  ~DevArena() {
    cudaStreamSynchronize(s_);
    for (void* q : bufs_) cudaFree(q);
  }
  template <typename T>
  T* get(size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, count ? count * sizeof(T) : 16) != cudaSuccess) {
      (void)cudaGetLastError();
      throw ApiError{NB_ERR_OOM, "octree maps: device allocation failed"};
    }
    bufs_.push_back(p);
    return static_cast<T*>(p);
  }

 private:
  cudaStream_t s_;
  std::vector<void*> bufs_;
};

struct Sorted {
  unsigned long long* keys;  // [npad], ascending; the first n are the leaves' keys
  int* pos;                  // [npad] input position of rank r
  int4* ranked;              // [n] leaves in rank order
  int* lev;                  // [n] their levels
};

unsigned blocks_of(long long m) { return static_cast<unsigned>((m + 255) / 256); }

// Keys, the bitonic rank sort, the unique-anchor check and the ranked leaves.
Sorted sort_leaves(nb_ctx* ctx, cudaStream_t s, const MapGeom& g, const int4* d_leaves, int n, int* d_err,
                   DevArena& A) {
  int npad = 1;
  while (npad < n) npad <<= 1;
  Sorted S{A.get<unsigned long long>(npad), A.get<int>(npad), A.get<int4>(n), A.get<int>(n)};
  k_keys<<<blocks_of(npad), 256, 0, s>>>(n, npad, d_leaves, g, S.keys, S.pos, d_err);
  ctx->launches++;
  for (int k = 2; k <= npad; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      k_bitonic<<<blocks_of(npad), 256, 0, s>>>(npad, j, k, S.keys, S.pos);
      ctx->launches++;
    }
  k_unique<<<blocks_of(n), 256, 0, s>>>(n, S.keys, d_err);
  k_ranked<<<blocks_of(n), 256, 0, s>>>(n, S.pos, d_leaves, S.ranked, S.lev);
  ctx->launches += 2;
  NB_CUDA(cudaGetLastError());
  return S;
}

void face_table(nb_ctx* ctx, cudaStream_t s, const MapGeom& g, const Sorted& S, int n, int* d_nbr, int* d_nnbr) {
  k_face_nbrs<<<blocks_of(6LL * n), 256, 0, s>>>(n, S.keys, S.ranked, S.lev, g, d_nbr, d_nnbr);
  ctx->launches++;
  NB_CUDA(cudaGetLastError());
}

void check_err(int h_err, const char* who) {
  if (h_err == 2) throw ApiError{NB_ERR_BAD_ARG, std::string(who) + ": a leaf lies outside the geometry"};
  if (h_err == 1) throw ApiError{NB_ERR_BAD_ARG, std::string(who) + ": two leaves share an anchor"};
}

// Splits the flagged leaves and restores 26-neighbour 2:1 balance on the
// device, then ranks the new leaves; writes them to the host array `out` in
// rank order. `flags_ranked`: the flags are per rank of the input (already
// sorted) instead of per input position.
void refine_on_device(nb_ctx* ctx, cudaStream_t s, const MapGeom& g, const int4* d_leaves, int n,
                      const uint8_t* d_flags, bool flags_ranked, int* d_err, DevArena& A, int32_t* out, int64_t cap,
                      int64_t* n_out) {
  const Sorted S = sort_leaves(ctx, s, g, d_leaves, n, d_err, A);
  uint8_t* mark = A.get<uint8_t>(n);
  if (flags_ranked) {
    NB_CUDA(cudaMemcpyAsync(mark, d_flags, n, cudaMemcpyDeviceToDevice, s));
  } else {
    k_rank_marks<<<blocks_of(n), 256, 0, s>>>(n, S.pos, d_flags, S.lev, g.lmax, mark);
    ctx->launches++;
  }
  int* changed = A.get<int>(1);
  int h_changed = 1;
  // every round moves the splits at least one level coarser: lmax rounds settle it
  for (int round = 0; h_changed && round <= g.lmax + 1; ++round) {
    NB_CUDA(cudaMemsetAsync(changed, 0, sizeof(int), s));
    k_balance_round<<<blocks_of(n), 256, 0, s>>>(n, S.keys, S.ranked, S.lev, g, mark, changed);
    ctx->launches++;
    NB_CUDA(cudaMemcpyAsync(&h_changed, changed, sizeof(int), cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaStreamSynchronize(s));
  }
  if (h_changed) throw ApiError{NB_ERR_BAD_ARG, "octree refinement: balance did not settle (unbalanced input)"};
  int* off = A.get<int>(n);
  int* total = A.get<int>(1);
  k_emit_offsets<<<1, 1024, 0, s>>>(n, mark, off, total);
  int m = 0;
  NB_CUDA(cudaMemcpyAsync(&m, total, sizeof(int), cudaMemcpyDeviceToHost, s));
  NB_CUDA(cudaStreamSynchronize(s));
  int4* fresh = A.get<int4>(m);
  k_emit_leaves<<<blocks_of(n), 256, 0, s>>>(n, S.ranked, mark, off, fresh);
  ctx->launches += 2;
  const Sorted R = sort_leaves(ctx, s, g, fresh, m, d_err, A);
  int h_err = 0;
  NB_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  NB_CUDA(cudaStreamSynchronize(s));
  check_err(h_err, "octree refinement");
  *n_out = m;
  if (!out || cap < m) throw ApiError{NB_ERR_BAD_ARG, "octree refinement: output capacity too small"};
  NB_CUDA(cudaMemcpyAsync(out, R.ranked, sizeof(int4) * m, cudaMemcpyDeviceToHost, s));
  NB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void nb::refine_from_sensors(nb_ctx* ctx, cudaStream_t s, const nb_amr_geom& g, const int32_t* leaves, int n,
                             const double* d_sensors, int which, double above, int32_t* out, int64_t cap,
                             int64_t* n_out) {
  const MapGeom mg = map_geom(g);
  DevArena A(s);
  int4* d_leaves = A.get<int4>(n);
  uint8_t* d_flags = A.get<uint8_t>(n);
  int* d_err = A.get<int>(1);
  NB_CUDA(cudaMemcpyAsync(d_leaves, leaves, sizeof(int4) * n, cudaMemcpyHostToDevice, s));
  NB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  k_sensor_marks<<<blocks_of(n), 256, 0, s>>>(n, d_sensors, which, above, d_leaves, mg.lmax, d_flags);
  ctx->launches++;
  // the mesh's leaves are already in rank order, so the flags are by rank
  refine_on_device(ctx, s, mg, d_leaves, n, d_flags, true, d_err, A, out, cap, n_out);
}

extern "C" {

uint64_t nb_morton_encode(uint32_t x, uint32_t y, uint32_t z) { return morton_encode(x, y, z); }

void nb_morton_decode(uint64_t key, uint32_t* x, uint32_t* y, uint32_t* z) {
  uint32_t a, b, c;
  morton_decode(key, a, b, c);
  if (x) *x = a;
  if (y) *y = b;
  if (z) *z = c;
}

nb_status nb_amr_build_maps(nb_ctx* ctx, const nb_amr_geom* g, const int32_t* leaves, int64_t n, uint64_t* keys,
                            int32_t* order, int32_t* nbr, int32_t* nnbr) {
  if (!ctx || !leaves || n <= 0 || n > (1 << 24) || !keys || !order || !nbr || !nnbr) return NB_ERR_BAD_ARG;
  if (!map_geom_ok(g)) return fail(ctx, NB_ERR_BAD_ARG, "nb_amr_build_maps: bad geometry");
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    const int nn = static_cast<int>(n);
    const MapGeom mg = map_geom(*g);
    cudaStream_t s = ctx->stream;
    DevArena A(s);
    int4* d_leaves = A.get<int4>(nn);
    int* d_nbr = A.get<int>(24 * static_cast<size_t>(nn));
    int* d_nnbr = A.get<int>(6 * static_cast<size_t>(nn));
    int* d_err = A.get<int>(1);
    NB_CUDA(cudaMemcpyAsync(d_leaves, leaves, sizeof(int4) * nn, cudaMemcpyHostToDevice, s));
    NB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    const Sorted S = sort_leaves(ctx, s, mg, d_leaves, nn, d_err, A);
    face_table(ctx, s, mg, S, nn, d_nbr, d_nnbr);
    int h_err = 0;
    NB_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaMemcpyAsync(keys, S.keys, sizeof(uint64_t) * nn, cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaMemcpyAsync(order, S.pos, sizeof(int) * nn, cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaMemcpyAsync(nbr, d_nbr, sizeof(int) * 24 * static_cast<size_t>(nn), cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaMemcpyAsync(nnbr, d_nnbr, sizeof(int) * 6 * static_cast<size_t>(nn), cudaMemcpyDeviceToHost, s));
    NB_CUDA(cudaStreamSynchronize(s));
    check_err(h_err, "nb_amr_build_maps");
    return NB_OK;
  });
}

nb_status nb_amr_refine_device(nb_ctx* ctx, const nb_amr_geom* g, const int32_t* leaves, int64_t n,
                               const uint8_t* flags, int32_t* out, int64_t cap, int64_t* n_out) {
  if (!ctx || !leaves || n <= 0 || n > (1 << 22) || !flags || !n_out) return NB_ERR_BAD_ARG;
  if (!map_geom_ok(g)) return fail(ctx, NB_ERR_BAD_ARG, "nb_amr_refine_device: bad geometry");
  return guarded(ctx, [&] {
    NB_CUDA(cudaSetDevice(ctx->device));
    const int nn = static_cast<int>(n);
    cudaStream_t s = ctx->stream;
    DevArena A(s);
    int4* d_leaves = A.get<int4>(nn);
    uint8_t* d_flags = A.get<uint8_t>(nn);
    int* d_err = A.get<int>(1);
    NB_CUDA(cudaMemcpyAsync(d_leaves, leaves, sizeof(int4) * nn, cudaMemcpyHostToDevice, s));
    NB_CUDA(cudaMemcpyAsync(d_flags, flags, nn, cudaMemcpyHostToDevice, s));
    NB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    refine_on_device(ctx, s, map_geom(*g), d_leaves, nn, d_flags, false, d_err, A, out, cap, n_out);
    return NB_OK;
  });
}

nb_status nb_amr_mesh_maps(const nb_amr_mesh* m, uint64_t* keys, int32_t* nbr, int32_t* nnbr) {
  if (!m || !keys || !nbr || !nnbr) return NB_ERR_BAD_ARG;
  export_tree_maps(m->lvl.tree, keys, nullptr, nbr, nnbr);
  return NB_OK;
}

nb_status nb_amr_tree_maps(const nb_amr_geom* g, const int32_t* leaves, int64_t n, uint64_t* keys, int32_t* ranked,
                           int32_t* nbr, int32_t* nnbr) {
  if (!map_geom_ok(g) || !leaves || n <= 0 || !keys || !ranked || !nbr || !nnbr) return NB_ERR_BAD_ARG;
  for (int f = 0; f < 6; ++f)
    if (g->face[f].type < NB_BC_WALL || g->face[f].type > NB_BC_PERIODIC) return NB_ERR_BAD_ARG;
  try {
    AmrGeom ag{};
    for (int a = 0; a < 3; ++a) {
      ag.nb0[a] = g->nb0[a];
      ag.h0[a] = g->h0[a];
      ag.origin[a] = g->origin[a];
    }
    for (int f = 0; f < 6; ++f) ag.bc[f] = g->face[f].type;
    ag.lmax = g->lmax;
    std::vector<AmrLeaf> in(static_cast<size_t>(n));
    for (int64_t q = 0; q < n; ++q)
      in[q] = AmrLeaf{leaves[4 * q], {leaves[4 * q + 1], leaves[4 * q + 2], leaves[4 * q + 3]}};
    std::string err;
    const AmrTree t = tree_from_leaves(ag, in, err);
    if (!err.empty()) return NB_ERR_BAD_ARG;
    export_tree_maps(t, keys, ranked, nbr, nnbr);
    return NB_OK;
  } catch (const std::exception&) {
    return NB_ERR_BAD_ARG;
  }
}

nb_status nb_amr_mesh_couplings(const nb_amr_mesh* m, int64_t* count, int32_t* off, int32_t* nbr, double* coef,
                                int64_t cap) {
  if (!m || !count) return NB_ERR_BAD_ARG;
  const AmrLevelHost& A = m->lvl;
  *count = static_cast<int64_t>(A.cf_nbr.size());
  if (!off && !nbr && !coef) return NB_OK;
  if (!off || !nbr || !coef || cap < *count) return NB_ERR_BAD_ARG;
  std::copy(A.cf_off.begin(), A.cf_off.end(), off);
  std::copy(A.cf_nbr.begin(), A.cf_nbr.end(), nbr);
  std::copy(A.cf_coef.begin(), A.cf_coef.end(), coef);
  return NB_OK;
}

}  // extern "C"
