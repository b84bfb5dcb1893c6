// nb_checkpoint.cpp — checkpoint files of a case (exact bit-for-bit restart).
//
// Uniform cases use the reference's NBFCK01 layout (core/src/flow/case.cpp:
// 244-319): 8 magic bytes "NBFCK01\0", int32 nx, ny, nz, int32 step, FP64 t,
// FP64 dt, then u, v, w, p each as a uint64 count followed by that many FP64
// values in the reference's lexicographic MAC layout, all in host byte order.
// A file written here is read by the reference's readCheckpoint and the other
// way round. Octree cases (no reference counterpart) use NBFAMR1: magic, int32
// leaf count, the leaves (level, bx, by, bz as int32, rank order), int32 step,
// FP64 t, FP64 dt, then the u, v, w face arrays in the library's storage
// order and p, with the same uint64 count prefix.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "nb_ctx.h"

using namespace nb;

namespace {

constexpr char kUniformMagic[8] = {'N', 'B', 'F', 'C', 'K', '0', '1', '\0'};
constexpr char kOctreeMagic[8] = {'N', 'B', 'F', 'A', 'M', 'R', '1', '\0'};

struct File {
  std::FILE* f = nullptr;
  explicit File(std::FILE* h) : f(h) {}
  ~File() {
    if (f) std::fclose(f);
  }
  File(const File&) = delete;
  File& operator=(const File&) = delete;
};

template <class T>
bool put(std::FILE* f, const T& v) {
  return std::fwrite(&v, sizeof(T), 1, f) == 1;
}
template <class T>
bool get(std::FILE* f, T& v) {
  return std::fread(&v, sizeof(T), 1, f) == 1;
}
bool put_vec(std::FILE* f, const std::vector<double>& a) {
  const uint64_t n = a.size();
  return put(f, n) && (n == 0 || std::fwrite(a.data(), 8, n, f) == n);
}
// Reads a counted FP64 array that must hold exactly `want` values.
bool get_vec(std::FILE* f, std::vector<double>& a, uint64_t want) {
  uint64_t n = 0;
  if (!get(f, n) || n != want) return false;
  a.resize(n);
  return n == 0 || std::fread(a.data(), 8, n, f) == n;
}

struct Header {
  int kind = -1;  // 0 NBFCK01 (uniform), 1 NBFAMR1 (octree)
  int32_t dims[3] = {0, 0, 0};
  std::vector<int32_t> leaves;  // octree: 4 per leaf
  int32_t step = 0;
  double t = 0.0, dt = 0.0;
};

// Reads the magic, the geometry and the clock; std::string error on failure.
std::string read_header(std::FILE* f, Header& h) {
  char magic[8];
  if (std::fread(magic, 1, 8, f) != 8) return "truncated file";
  if (std::memcmp(magic, kUniformMagic, 8) == 0) {
    h.kind = 0;
    if (!get(f, h.dims[0]) || !get(f, h.dims[1]) || !get(f, h.dims[2])) return "truncated header";
  } else if (std::memcmp(magic, kOctreeMagic, 8) == 0) {
    h.kind = 1;
    int32_t n = 0;
    if (!get(f, n) || n <= 0 || n > (1 << 26)) return "bad leaf count";
    h.leaves.resize(static_cast<size_t>(n) * 4);
    if (std::fread(h.leaves.data(), 4, h.leaves.size(), f) != h.leaves.size()) return "truncated leaf list";
  } else {
    return "bad magic";
  }
  if (!get(f, h.step) || !get(f, h.t) || !get(f, h.dt)) return "truncated header";
  return "";
}

}  // namespace

extern "C" {

nb_status nb_case_write_checkpoint(nb_case* c, const char* path) {
  if (!c || !path) return NB_ERR_BAD_ARG;
  nb_ctx* ctx = case_ctx(c);
  int step = 0;
  double t = 0.0, dt = 0.0;
  nb_status st = nb_case_get_clock(c, &step, &t, &dt);
  if (st != NB_OK) return st;
  std::vector<double> f[4];
  nb_amr_mesh* mesh = case_mesh(c);
  std::vector<int32_t> leaves;
  int dims[3] = {0, 0, 0};
  if (mesh) {
    int64_t sz[4];
    if ((st = nb_amr_case_sizes(c, sz)) != NB_OK) return st;
    for (int q = 0; q < 4; ++q) f[q].resize(static_cast<size_t>(sz[q]));
    if ((st = nb_amr_case_get_state(c, f[0].data(), f[1].data(), f[2].data(), f[3].data())) != NB_OK) return st;
    leaves.resize(static_cast<size_t>(nb_amr_mesh_leaf_count(mesh)) * 4);
    if ((st = nb_amr_mesh_leaves(mesh, leaves.data())) != NB_OK) return st;
  } else {
    case_dims(c, dims);
    const size_t nx = dims[0], ny = dims[1], nz = dims[2];
    f[0].resize((nx + 1) * ny * nz);
    f[1].resize(nx * (ny + 1) * nz);
    f[2].resize(nx * ny * (nz + 1));
    f[3].resize(nx * ny * nz);
    if ((st = nb_case_get_state(c, f[0].data(), f[1].data(), f[2].data(), f[3].data())) != NB_OK) return st;
  }
  File file(std::fopen(path, "wb"));
  if (!file.f) return fail(ctx, NB_ERR_BAD_ARG, std::string("nb_case_write_checkpoint: cannot open ") + path);
  bool ok;
  if (mesh) {
    ok = std::fwrite(kOctreeMagic, 1, 8, file.f) == 8 && put(file.f, static_cast<int32_t>(leaves.size() / 4)) &&
         std::fwrite(leaves.data(), 4, leaves.size(), file.f) == leaves.size();
  } else {
    ok = std::fwrite(kUniformMagic, 1, 8, file.f) == 8 && put(file.f, static_cast<int32_t>(dims[0])) &&
         put(file.f, static_cast<int32_t>(dims[1])) && put(file.f, static_cast<int32_t>(dims[2]));
  }
  ok = ok && put(file.f, static_cast<int32_t>(step)) && put(file.f, t) && put(file.f, dt);
  for (int q = 0; q < 4 && ok; ++q) ok = put_vec(file.f, f[q]);
  ok = ok && std::fflush(file.f) == 0;
  if (!ok) return fail(ctx, NB_ERR_BAD_ARG, std::string("nb_case_write_checkpoint: write failed on ") + path);
  return NB_OK;
}

nb_status nb_case_read_checkpoint(nb_case* c, const char* path) {
  if (!c || !path) return NB_ERR_BAD_ARG;
  nb_ctx* ctx = case_ctx(c);
  const std::string who = std::string("nb_case_read_checkpoint: ") + path + ": ";
  File file(std::fopen(path, "rb"));
  if (!file.f) return fail(ctx, NB_ERR_BAD_ARG, who + "cannot open");
  Header h;
  const std::string err = read_header(file.f, h);
  if (!err.empty()) return fail(ctx, NB_ERR_BAD_ARG, who + err);
  nb_amr_mesh* mesh = case_mesh(c);
  std::vector<double> f[4];
  uint64_t want[4];
  if (mesh) {
    if (h.kind != 1) return fail(ctx, NB_ERR_BAD_ARG, who + "not an octree checkpoint");
    std::vector<int32_t> leaves(static_cast<size_t>(nb_amr_mesh_leaf_count(mesh)) * 4);
    nb_amr_mesh_leaves(mesh, leaves.data());
    if (leaves != h.leaves) return fail(ctx, NB_ERR_BAD_ARG, who + "leaf list differs from the case's mesh");
    int64_t sz[4];
    nb_status st = nb_amr_case_sizes(c, sz);
    if (st != NB_OK) return st;
    for (int q = 0; q < 4; ++q) want[q] = static_cast<uint64_t>(sz[q]);
  } else {
    if (h.kind != 0) return fail(ctx, NB_ERR_BAD_ARG, who + "not a uniform-grid checkpoint");
    int dims[3];
    case_dims(c, dims);
    if (h.dims[0] != dims[0] || h.dims[1] != dims[1] || h.dims[2] != dims[2])
      return fail(ctx, NB_ERR_BAD_ARG, who + "grid dimension mismatch");
    const uint64_t nx = dims[0], ny = dims[1], nz = dims[2];
    want[0] = (nx + 1) * ny * nz;
    want[1] = nx * (ny + 1) * nz;
    want[2] = nx * ny * (nz + 1);
    want[3] = nx * ny * nz;
  }
  for (int q = 0; q < 4; ++q)
    if (!get_vec(file.f, f[q], want[q])) return fail(ctx, NB_ERR_BAD_ARG, who + "field size mismatch or truncated");
  if (mesh) {
    nb_status st = nb_amr_case_set_state(c, f[0].data(), f[1].data(), f[2].data(), f[3].data());
    if (st != NB_OK) return st;
    case_set_clock(c, h.step, h.t, h.dt);
    return NB_OK;
  }
  return nb_case_set_state(c, f[0].data(), f[1].data(), f[2].data(), f[3].data(), h.step, h.t, h.dt);
}

int nb_checkpoint_info(const char* path, int32_t* kind, int32_t dims[3], int64_t* nleaf, int32_t* step,
                       double* t, double* dt) {
  if (!path) return -1;
  File file(std::fopen(path, "rb"));
  if (!file.f) return -1;
  Header h;
  if (!read_header(file.f, h).empty()) return -1;
  if (kind) *kind = h.kind;
  if (dims)
    for (int a = 0; a < 3; ++a) dims[a] = h.dims[a];
  if (nleaf) *nleaf = static_cast<int64_t>(h.leaves.size() / 4);
  if (step) *step = h.step;
  if (t) *t = h.t;
  if (dt) *dt = h.dt;
  return 0;
}

}  // extern "C"
