// nb_bricks.cpp — host construction of the brick layout and the MG hierarchy.
//
// Integer maps only (bit-exact work): Morton ranking of bricks, the dense
// brick lookup table, per-cell type codes and the coarsening hierarchy.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "nb_internal.h"
#include "nb_morton.h"

namespace nb {

CudaError::CudaError(cudaError_t e, const char* call, const char* file, int line) : err(e) {
  what = std::string(cudaGetErrorString(e)) + " in " + call + " (" + file + ":" +
         std::to_string(line) + ")";
}

void build_level(HostLevel& L, int nx, int ny, int nz, double dx, double dy, double dz,
                 const uint8_t* solid) {
  L.nx = nx;
  L.ny = ny;
  L.nz = nz;
  L.dx = dx;
  L.dy = dy;
  L.dz = dz;
  L.nbx = (nx + BR - 1) / BR;
  L.nby = (ny + BR - 1) / BR;
  L.nbz = (nz + BR - 1) / BR;
  L.nbrick = L.nbx * L.nby * L.nbz;
  // Rank bricks by Morton key of their coordinates.
  std::vector<std::pair<uint64_t, int>> keys;
  keys.reserve(L.nbrick);
  for (int bz = 0; bz < L.nbz; ++bz)
    for (int by = 0; by < L.nby; ++by)
      for (int bx = 0; bx < L.nbx; ++bx)
        keys.emplace_back(morton_encode(bx, by, bz), (bz * L.nby + by) * L.nbx + bx);
  std::sort(keys.begin(), keys.end());
  L.lut.assign(L.nbrick, -1);
  L.bcoord.assign(3 * L.nbrick, 0);
  for (int r = 0; r < L.nbrick; ++r) {
    const int lin = keys[r].second;
    L.lut[lin] = r;
    L.bcoord[3 * r] = lin % L.nbx;
    L.bcoord[3 * r + 1] = (lin / L.nbx) % L.nby;
    L.bcoord[3 * r + 2] = lin / (L.nbx * L.nby);
  }
  const size_t ncell = static_cast<size_t>(nx) * ny * nz;
  L.solid.assign(ncell, 0);
  if (solid) std::memcpy(L.solid.data(), solid, ncell);
  L.type.assign(static_cast<size_t>(L.nbrick) * BR3, CELL_VOID);
  L.nfluid = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int b = L.lut[((k / BR) * L.nby + j / BR) * L.nbx + i / BR];
        const size_t idx = static_cast<size_t>(b) * BR3 + ((k & 7) << 6) + ((j & 7) << 3) + (i & 7);
        const bool s = L.solid[static_cast<size_t>(i) + static_cast<size_t>(nx) * (j + static_cast<size_t>(ny) * k)] != 0;
        L.type[idx] = s ? CELL_SOLID : CELL_FLUID;
        if (!s) ++L.nfluid;
      }
}

void build_codes(HostLevel& L, const int bc[6]) {
  L.code.assign(L.type.size(), static_cast<uint16_t>(CELL_VOID << CODE_TYPE));
  const int dims[3] = {L.nx, L.ny, L.nz};
  auto lex = [&](int i, int j, int k) {
    return static_cast<size_t>(i) + static_cast<size_t>(L.nx) * (j + static_cast<size_t>(L.ny) * k);
  };
  for (int k = 0; k < L.nz; ++k)
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i) {
        const int b = L.lut[((k / BR) * L.nby + j / BR) * L.nbx + i / BR];
        const size_t idx = static_cast<size_t>(b) * BR3 + ((k & 7) << 6) + ((j & 7) << 3) + (i & 7);
        const bool solid = L.solid[lex(i, j, k)] != 0;
        uint16_t code = static_cast<uint16_t>((solid ? CELL_SOLID : CELL_FLUID) << CODE_TYPE);
        for (int axis = 0; axis < 3 && !solid; ++axis) {
          if (axis == 2 && L.nz == 1) continue;  // 2-D: no z coupling
          for (int side = 0; side < 2; ++side) {
            int c[3] = {i, j, k};
            c[axis] += side ? 1 : -1;
            const int f = 2 * axis + side;
            if (c[axis] < 0 || c[axis] >= dims[axis]) {
              const int bt = bc[f];
              if (bt == NB_BC_OUTLET) {
                code |= static_cast<uint16_t>(1u << (CODE_DIRICHLET + f));
                continue;
              }
              if (bt != NB_BC_PERIODIC) continue;  // wall / inlet: Neumann
              c[axis] = (c[axis] + dims[axis]) % dims[axis];
            }
            if (!L.solid[lex(c[0], c[1], c[2])]) code |= static_cast<uint16_t>(1u << f);
          }
        }
        L.code[idx] = code;
      }
}

// MgPoisson hierarchy construction (core/src/flow/multigrid.cpp:211-266):
// halve an axis only if its length is >= 4, stop at <= 2048 cells or 8 levels;
// a coarse cell is fluid if any child is fluid.
std::vector<HostLevel> build_hierarchy(const nb_grid_desc& g, size_t coarsest_max) {
  constexpr int kMaxLevels = 8;
  const size_t kCoarsestMax = coarsest_max;
  constexpr int kMinCoarsen = 4;
  std::vector<HostLevel> H;
  H.reserve(kMaxLevels);
  H.emplace_back();
  build_level(H.back(), g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.solid);
  while (static_cast<int>(H.size()) < kMaxLevels) {
    const HostLevel& f = H.back();
    const int fx = f.nx >= kMinCoarsen ? 2 : 1;
    const int fy = f.ny >= kMinCoarsen ? 2 : 1;
    const int fz = f.nz >= kMinCoarsen ? 2 : 1;
    if (fx == 1 && fy == 1 && fz == 1) break;
    const int cnx = (f.nx + fx - 1) / fx, cny = (f.ny + fy - 1) / fy, cnz = (f.nz + fz - 1) / fz;
    const double cdx = f.dx * static_cast<double>(f.nx) / static_cast<double>(cnx);
    const double cdy = f.dy * static_cast<double>(f.ny) / static_cast<double>(cny);
    const double cdz = f.dz * static_cast<double>(f.nz) / static_cast<double>(cnz);
    std::vector<uint8_t> csolid(static_cast<size_t>(cnx) * cny * cnz, 1);
    for (int k = 0; k < f.nz; ++k)
      for (int j = 0; j < f.ny; ++j)
        for (int i = 0; i < f.nx; ++i)
          if (!f.solid[static_cast<size_t>(i) + static_cast<size_t>(f.nx) * (j + static_cast<size_t>(f.ny) * k)])
            csolid[static_cast<size_t>(i / fx) + static_cast<size_t>(cnx) * (j / fy + static_cast<size_t>(cny) * (k / fz))] = 0;
    HostLevel c;
    c.fx = fx;
    c.fy = fy;
    c.fz = fz;
    build_level(c, cnx, cny, cnz, cdx, cdy, cdz, csolid.data());
    H.push_back(std::move(c));
    if (static_cast<size_t>(cnx) * cny * cnz <= kCoarsestMax) break;
  }
  return H;
}

// FNV-1a over dims, BC types and solid cells (core/src/flow/multigrid.cpp:43-61),
// extended with the spacing bits because the device hierarchy also caches h.
uint64_t grid_signature(const nb_grid_desc& g) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    h ^= v;
    h *= 1099511628211ull;
  };
  mix(static_cast<uint64_t>(g.nx));
  mix(static_cast<uint64_t>(g.ny));
  mix(static_cast<uint64_t>(g.nz));
  for (int f = 0; f < 6; ++f) mix(static_cast<uint64_t>(g.face[f].type));
  const size_t n = static_cast<size_t>(g.nx) * g.ny * g.nz;
  if (g.solid)
    for (size_t i = 0; i < n; ++i)
      if (g.solid[i]) mix(i);
  uint64_t bits[3];
  std::memcpy(&bits[0], &g.dx, 8);
  std::memcpy(&bits[1], &g.dy, 8);
  std::memcpy(&bits[2], &g.dz, 8);
  for (uint64_t b : bits) mix(b);
  return h;
}

}  // namespace nb
