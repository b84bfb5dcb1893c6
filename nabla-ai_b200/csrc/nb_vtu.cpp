// nb_vtu.cpp — VTK XML unstructured-grid output of a case's cell-centred state.
//
// Uniform cases follow writeGridVtu (core/src/flow/case.cpp:175-241): one
// hexahedron per cell with its 8 corners in VTK order, cells in the
// reference's lexicographic order, ASCII values at 8 significant digits, and
// the cell data u, v, w (NSSolver::cellVelocity), p, speed and solid. Octree
// cases write every leaf cell the same way (leaves in rank order, cells
// x-fastest inside a brick) with an Int32 `level` array first, as the octree
// writer does (core/src/io/vtu_writer.cpp:8-80). The cell-centred values come
// from the device sampler (nb_case_sample) at the cell centres.
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "nb_amr_mesh.h"
#include "nb_ctx.h"

using namespace nb;

namespace {

struct Cells {
  std::vector<double> lo, hi;  // corners, 3 per cell
  std::vector<double> centre;  // 3 per cell
  std::vector<int> level;      // octree only
};

Cells uniform_cells(const nb_grid_desc& g) {
  Cells c;
  const size_t n = static_cast<size_t>(g.nx) * g.ny * g.nz;
  c.lo.reserve(3 * n);
  c.hi.reserve(3 * n);
  c.centre.reserve(3 * n);
  const double d[3] = {g.dx, g.dy, g.dz};
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        const int ijk[3] = {i, j, k};
        for (int a = 0; a < 3; ++a) {
          const double x0 = g.origin[a] + ijk[a] * d[a];
          c.lo.push_back(x0);
          c.hi.push_back(x0 + d[a]);
          c.centre.push_back(x0 + 0.5 * d[a]);
        }
      }
  return c;
}

Cells octree_cells(const nb_amr_geom& g, const std::vector<int32_t>& leaves) {
  Cells c;
  const size_t nl = leaves.size() / 4;
  for (size_t r = 0; r < nl; ++r) {
    const int L = leaves[4 * r];
    for (int l = 0; l < 512; ++l) {
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      for (int a = 0; a < 3; ++a) {
        const double h = g.h0[a] / static_cast<double>(1 << L);
        const double x0 = g.origin[a] + (leaves[4 * r + 1 + a] * 8 + loc[a]) * h;
        c.lo.push_back(x0);
        c.hi.push_back(x0 + h);
        c.centre.push_back(x0 + 0.5 * h);
      }
      c.level.push_back(L);
    }
  }
  return c;
}

}  // namespace

extern "C" {

nb_status nb_case_write_vtu(nb_case* c, const char* path) {
  if (!c || !path) return NB_ERR_BAD_ARG;
  nb_ctx* ctx = case_ctx(c);
  nb_amr_mesh* mesh = case_mesh(c);
  Cells cells;
  if (mesh) {
    std::vector<int32_t> leaves(static_cast<size_t>(nb_amr_mesh_leaf_count(mesh)) * 4);
    nb_status st = nb_amr_mesh_leaves(mesh, leaves.data());
    if (st != NB_OK) return st;
    cells = octree_cells(mesh->geom, leaves);
  } else {
    cells = uniform_cells(case_grid(c));
  }
  const size_t n = cells.centre.size() / 3;
  std::vector<double> f[4];
  for (int q = 0; q < 4; ++q) {
    f[q].resize(n);
    const nb_status st = nb_case_sample(c, q, static_cast<int64_t>(n), cells.centre.data(), f[q].data());
    if (st != NB_OK) return st;
  }
  std::vector<uint8_t> solid = case_solid(c);
  std::ofstream o(path);
  if (!o) return fail(ctx, NB_ERR_BAD_ARG, std::string("nb_case_write_vtu: cannot open ") + path);
  o.precision(8);
  const size_t npts = n * 8;
  o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" "
       "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n  <UnstructuredGrid>\n";
  o << "    <Piece NumberOfPoints=\"" << npts << "\" NumberOfCells=\"" << n << "\">\n";
  o << "      <Points>\n        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (size_t q = 0; q < n; ++q) {
    const double x0 = cells.lo[3 * q], y0 = cells.lo[3 * q + 1], z0 = cells.lo[3 * q + 2];
    const double x1 = cells.hi[3 * q], y1 = cells.hi[3 * q + 1], z1 = cells.hi[3 * q + 2];
    o << x0 << ' ' << y0 << ' ' << z0 << ' ' << x1 << ' ' << y0 << ' ' << z0 << ' ' << x1 << ' ' << y1 << ' '
      << z0 << ' ' << x0 << ' ' << y1 << ' ' << z0 << ' ' << x0 << ' ' << y0 << ' ' << z1 << ' ' << x1 << ' '
      << y0 << ' ' << z1 << ' ' << x1 << ' ' << y1 << ' ' << z1 << ' ' << x0 << ' ' << y1 << ' ' << z1 << '\n';
  }
  o << "        </DataArray>\n      </Points>\n      <Cells>\n";
  o << "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
  for (size_t i = 0; i < npts; ++i) o << i << ((i + 1) % 8 == 0 ? '\n' : ' ');
  o << "        </DataArray>\n        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
  for (size_t i = 1; i <= n; ++i) o << i * 8 << ' ';
  o << "\n        </DataArray>\n        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
  for (size_t i = 0; i < n; ++i) o << "12 ";
  o << "\n        </DataArray>\n      </Cells>\n      <CellData Scalars=\"speed\">\n";
  if (mesh) {
    o << "        <DataArray type=\"Int32\" Name=\"level\" format=\"ascii\">\n";
    for (int L : cells.level) o << L << ' ';
    o << "\n        </DataArray>\n";
  }
  const auto dump = [&](const char* name, const std::vector<double>& a) {
    o << "        <DataArray type=\"Float64\" Name=\"" << name << "\" format=\"ascii\">\n";
    for (double x : a) o << x << ' ';
    o << "\n        </DataArray>\n";
  };
  std::vector<double> speed(n), sol(n, 0.0);
  for (size_t q = 0; q < n; ++q) {
    speed[q] = std::sqrt(f[0][q] * f[0][q] + f[1][q] * f[1][q] + f[2][q] * f[2][q]);
    if (solid.size() == n) sol[q] = solid[q] ? 1.0 : 0.0;
  }
  dump("u", f[0]);
  dump("v", f[1]);
  dump("w", f[2]);
  dump("p", f[3]);
  dump("speed", speed);
  dump("solid", sol);
  o << "      </CellData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
  o.flush();
  if (!o) return fail(ctx, NB_ERR_BAD_ARG, std::string("nb_case_write_vtu: write failed on ") + path);
  return NB_OK;
}

}  // extern "C"
