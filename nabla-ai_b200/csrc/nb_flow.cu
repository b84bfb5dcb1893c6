// nb_flow.cu — sm_100a kernels of the MAC step: BC-aware halo staging, fused
// WENO-5 momentum RHS + SSP-RK3 combine, divergence, projection correction,
// step diagnostics and layout conversion.
//
// Reference arithmetic followed (paths within the reference project):
//   weno5 / reconstruct        core/src/flow/ns_solver.cpp:15-42
//   U / Vv / W ghost accessors core/src/flow/ns_solver.cpp:116-219
//   applyVelocityBC            core/src/flow/ns_solver.cpp:221-309
//   computeRhs                 core/src/flow/ns_solver.cpp:311-473
//   RK3 combine                core/src/flow/ns_solver.cpp:773-795
//   project (div, correction)  core/src/flow/ns_solver.cpp:475-579
//   computeDt                  core/src/flow/ns_solver.cpp:581-603
//   diagnostics                core/src/flow/ns_solver.cpp:605-763, :797-823
#include <algorithm>
#include <cmath>

#include "nb_flow.cuh"
#include "nb_momentum.cuh"
#include "nb_reduce.cuh"

namespace nb {

namespace {

constexpr int NT = 512;
constexpr int MAX_GRID = 148 * 4;
constexpr int RHS_NT = 256;
constexpr int TW = 14;  // brick + 3 ghost layers per side
constexpr int TN = TW * TW * TW;

inline int grid_for(int nbrick) { return nbrick < MAX_GRID ? nbrick : MAX_GRID; }

__device__ __forceinline__ bool is_solid_g(const LevelView& L, int i, int j, int k) {
  if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz) return false;
  return L.type[cell_index(L, i, j, k)] == CELL_SOLID;
}

// Storage index of a face (slab for the domain's high face).
__device__ __forceinline__ long long uidx(const FlowView& F, int i, int j, int k) {
  return i == F.L.nx ? F.nb + j + static_cast<long long>(F.L.ny) * k : cell_index(F.L, i, j, k);
}
__device__ __forceinline__ long long vidx(const FlowView& F, int i, int j, int k) {
  return j == F.L.ny ? F.nb + i + static_cast<long long>(F.L.nx) * k : cell_index(F.L, i, j, k);
}
__device__ __forceinline__ long long widx(const FlowView& F, int i, int j, int k) {
  return k == F.L.nz ? F.nb + i + static_cast<long long>(F.L.nx) * j : cell_index(F.L, i, j, k);
}

// inletVelocityAt(face, a, b) component `comp` (ns_solver.cpp:71-93); `a`
// plays the role of the reference's j argument in the parabolic profile.
__device__ __forceinline__ double inlet_vel(const FlowView& F, int face, int a, int comp) {
  double mag = F.inlet_speed[face];
  if (F.profile[face] == NB_PROFILE_PARABOLIC) {
    const double H = F.L.ny * F.L.dxyz[1];
    const double yc = F.origin[1] + 0.5 * H;
    const double y = F.origin[1] + (a + 0.5) * F.L.dxyz[1];
    const double r = (y - yc) / (0.5 * H);
    mag = 1.5 * F.inlet_speed[face] * (1.0 - r * r);
  }
  return F.inlet_axis[face] == comp ? mag : 0.0;
}

// The reference's recursive ghost accessors evaluate nested expressions
// c0 - (c1 - (c2 - ... - terminal)). Each walk records the constants and
// unwinds them innermost-first so the association is the same.
constexpr int ACC_MAX = 16;

__device__ double acc_u(const FlowView& F, const double* __restrict__ u, int i, int j, int k) {
  const int nx = F.L.nx, ny = F.L.ny, nz = F.L.nz;
  double cst[ACC_MAX];
  int d = 0;
  double term = __longlong_as_double(0x7ff8000000000000ll);
  for (int guard = 0; guard < ACC_MAX; ++guard) {
    if (k < 0 || k >= nz) {
      if (F.per[2]) { k = wrapi(k, nz); continue; }
      const int face = k < 0 ? 4 : 5;
      cst[d++] = 2.0 * F.wallv[face][0];
      k = k < 0 ? (-1 - k) : (2 * nz - 1 - k);
      continue;
    }
    if (j < 0 || j >= ny) {
      if (F.per[1]) { j = wrapi(j, ny); continue; }
      const int face = j < 0 ? 2 : 3;
      cst[d++] = 2.0 * F.wallv[face][0];
      j = j < 0 ? (-1 - j) : (2 * ny - 1 - j);
      continue;
    }
    if (i < 0 || i > nx) {
      if (F.per[0]) { i = wrapi(i, nx); continue; }
      const int ib = i < 0 ? 0 : nx;
      const int face = i < 0 ? 0 : 1;
      if (F.L.bc[face] == NB_BC_OUTLET) { term = u[uidx(F, ib, j, k)]; break; }
      cst[d++] = 2.0 * u[uidx(F, ib, j, k)];
      i = 2 * ib - i;
      continue;
    }
    term = u[uidx(F, i, j, k)];
    break;
  }
  for (int q = d - 1; q >= 0; --q) term = cst[q] - term;
  return term;
}

__device__ double acc_v(const FlowView& F, const double* __restrict__ v, int i, int j, int k) {
  const int nx = F.L.nx, ny = F.L.ny, nz = F.L.nz;
  double cst[ACC_MAX];
  int d = 0;
  double term = __longlong_as_double(0x7ff8000000000000ll);
  for (int guard = 0; guard < ACC_MAX; ++guard) {
    if (k < 0 || k >= nz) {
      if (F.per[2]) { k = wrapi(k, nz); continue; }
      const int face = k < 0 ? 4 : 5;
      cst[d++] = 2.0 * F.wallv[face][1];
      k = k < 0 ? (-1 - k) : (2 * nz - 1 - k);
      continue;
    }
    if (i < 0 || i >= nx) {
      if (F.per[0]) { i = wrapi(i, nx); continue; }
      const int im = i < 0 ? (-1 - i) : (2 * nx - 1 - i);
      const int face = i < 0 ? 0 : 1;
      if (F.L.bc[face] == NB_BC_INLET) {
        cst[d++] = 2.0 * inlet_vel(F, face, j, 1);
        i = im;
        continue;
      }
      if (F.L.bc[face] == NB_BC_OUTLET) {
        // j is still unresolved here; stencil points always have it in range,
        // the clamp only keeps unused corner halo points in bounds.
        term = v[vidx(F, i < 0 ? 0 : nx - 1, min(max(j, 0), ny), k)];
        break;
      }
      cst[d++] = 2.0 * F.wallv[face][1];
      i = im;
      continue;
    }
    if (j < 0 || j > ny) {
      if (F.per[1]) { j = wrapi(j, ny); continue; }
      const int jb = j < 0 ? 0 : ny;
      const int face = j < 0 ? 2 : 3;
      if (F.L.bc[face] == NB_BC_OUTLET) { term = v[vidx(F, i, jb, k)]; break; }
      cst[d++] = 2.0 * v[vidx(F, i, jb, k)];
      j = 2 * jb - j;
      continue;
    }
    term = v[vidx(F, i, j, k)];
    break;
  }
  for (int q = d - 1; q >= 0; --q) term = cst[q] - term;
  return term;
}

__device__ double acc_w(const FlowView& F, const double* __restrict__ w, int i, int j, int k) {
  const int nx = F.L.nx, ny = F.L.ny, nz = F.L.nz;
  double cst[ACC_MAX];
  int d = 0;
  double term = __longlong_as_double(0x7ff8000000000000ll);
  for (int guard = 0; guard < ACC_MAX; ++guard) {
    if (j < 0 || j >= ny) {
      if (F.per[1]) { j = wrapi(j, ny); continue; }
      const int face = j < 0 ? 2 : 3;
      cst[d++] = 2.0 * F.wallv[face][2];
      j = j < 0 ? (-1 - j) : (2 * ny - 1 - j);
      continue;
    }
    if (i < 0 || i >= nx) {
      if (F.per[0]) { i = wrapi(i, nx); continue; }
      const int im = i < 0 ? (-1 - i) : (2 * nx - 1 - i);
      const int face = i < 0 ? 0 : 1;
      if (F.L.bc[face] == NB_BC_OUTLET) {
        // k is still unresolved here (see acc_v).
        term = w[widx(F, i < 0 ? 0 : nx - 1, j, min(max(k, 0), nz))];
        break;
      }
      cst[d++] = 2.0 * F.wallv[face][2];
      i = im;
      continue;
    }
    if (k < 0 || k > nz) {
      if (F.per[2]) { k = wrapi(k, nz); continue; }
      const int kb = k < 0 ? 0 : nz;
      cst[d++] = 2.0 * w[widx(F, i, j, kb)];
      k = 2 * kb - k;
      continue;
    }
    term = w[widx(F, i, j, k)];
    break;
  }
  for (int q = d - 1; q >= 0; --q) term = cst[q] - term;
  return term;
}

__device__ __forceinline__ int tix(int a, int b, int c) { return ((c + 3) * TW + (b + 3)) * TW + (a + 3); }

// ---------------------------------------------------------------------------
// Fused momentum RHS + RK3 stage combine. One CTA per brick (grid-stride):
// stage the brick's u, v, w plus 3 ghost layers (BC-resolved exactly like the
// reference's accessors) in shared memory, then each thread forms the WENO-5
// divergence-form fluxes + central viscous term for its cells' low faces and
// writes the stage combination. Faces that the reference leaves without a RHS
// (domain-boundary faces, faces touching a solid) get R = 0.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(RHS_NT) k_rhs_rk(FlowView F, int stage, const double* __restrict__ dtp,
                                                   const double* __restrict__ u,
                                                   const double* __restrict__ v,
                                                   const double* __restrict__ w,
                                                   const double* __restrict__ u0,
                                                   const double* __restrict__ v0,
                                                   const double* __restrict__ w0, double* __restrict__ uo,
                                                   double* __restrict__ vo, double* __restrict__ wo) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tu = reinterpret_cast<T*>(smraw);
  T* tv = tu + TN;
  T* tw = tv + TN;
  const LevelView& L = F.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int twoD = L.twoD;
  const T dx = T(L.dxyz[0]), dy = T(L.dxyz[1]), dz = T(L.dxyz[2]);
  const T nu = T(F.nu);
  const double c1 = 1.0 / 3.0, c2 = 2.0 / 3.0;
  const double dt = *dtp;
  auto comb = [&](double a0, double a, double r) -> double {
    if (stage == 1) return a0 + dt * r;
    if (stage == 2) return 0.75 * a0 + 0.25 * (a + dt * r);
    return c1 * a0 + c2 * (a + dt * r);
  };
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int ox = L.bcoord[3 * brick] * BR, oy = L.bcoord[3 * brick + 1] * BR,
              oz = L.bcoord[3 * brick + 2] * BR;
    for (int p = threadIdx.x; p < TN; p += blockDim.x) {
      const int ti = p % TW, tj = (p / TW) % TW, tk = p / (TW * TW);
      const int far = (ti < 2 || ti > 11) + (tj < 2 || tj > 11) + (tk < 2 || tk > 11);
      if (far > 1) continue;  // never read by any stencil
      const int gi = ox + ti - 3, gj = oy + tj - 3, gk = oz + tk - 3;
      if (gi >= 0 && gj >= 0 && gk >= 0 && gi < nx && gj < ny && gk < nz) {
        // strictly inside the domain no ghost rule applies: every accessor
        // reads the cell's stored low face
        const long long c = cell_index(L, gi, gj, gk);
        tu[p] = static_cast<T>(u[c]);
        tv[p] = static_cast<T>(v[c]);
        tw[p] = static_cast<T>(w[c]);
      } else {
        tu[p] = static_cast<T>(acc_u(F, u, gi, gj, gk));
        tv[p] = static_cast<T>(acc_v(F, v, gi, gj, gk));
        tw[p] = static_cast<T>(acc_w(F, w, gi, gj, gk));
      }
    }
    __syncthreads();
    // Face jobs: component a's low face of every cell (one RHS call site).
    for (int job = threadIdx.x; job < 3 * BR3; job += blockDim.x) {
      const int a = job >> 9, l = job & (BR3 - 1);
      const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
      const int g[3] = {ox + loc[0], oy + loc[1], oz + loc[2]};
      if (g[0] >= nx || g[1] >= ny || g[2] >= nz) continue;  // void cell
      const int c = brick * BR3 + l;
      // faces touching a solid, the domain's low boundary faces and (2-D) w get R = 0
      double r = 0.0;
      if (g[a] >= 1 && !(a == 2 && twoD) && L.type[c] != CELL_SOLID &&
          !is_solid_g(L, g[0] - (a == 0), g[1] - (a == 1), g[2] - (a == 2)))
        r = static_cast<double>(rhs_face<T, TW, TW * TW>(tu, tv, tw, a, tix(loc[0], loc[1], loc[2]), F.weno, dx, dy,
                                                         dz, nu, T(F.bf[a]), twoD != 0));
      const double* f = a == 0 ? u : (a == 1 ? v : w);
      const double* f0 = a == 0 ? u0 : (a == 1 ? v0 : w0);
      double* o = a == 0 ? uo : (a == 1 ? vo : wo);
      o[c] = comb(f0[c], f[c], r);
      // the domain's high boundary face (no RHS)
      if (g[a] == (a == 0 ? nx : (a == 1 ? ny : nz)) - 1) {
        const long long s = a == 0 ? uidx(F, nx, g[1], g[2]) : (a == 1 ? vidx(F, g[0], ny, g[2]) : widx(F, g[0], g[1], nz));
        o[s] = comb(f0[s], f[s], 0.0);
      }
    }
    __syncthreads();
  }
}

// applyVelocityBC as a list of face actions (host-built, reference order).
__global__ void k_bc(const BcOp* __restrict__ ops, int n, int serial, double* u, double* v, double* w) {
  double* comp[3] = {u, v, w};
  if (serial) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      for (int m = 0; m < n; ++m) {
        const BcOp o = ops[m];
        comp[o.comp][o.idx] = o.action == 0 ? o.val : comp[o.comp][o.src];
      }
    return;
  }
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const BcOp o = ops[m];
    comp[o.comp][o.idx] = o.action == 0 ? o.val : comp[o.comp][o.src];
  }
}

__device__ __forceinline__ double div_at(const FlowView& F, const double* __restrict__ u,
                                         const double* __restrict__ v, const double* __restrict__ w,
                                         int c, int gi, int gj, int gk) {
  double d = (u[uidx(F, gi + 1, gj, gk)] - u[c]) / F.L.dxyz[0] +
             (v[vidx(F, gi, gj + 1, gk)] - v[c]) / F.L.dxyz[1];
  if (F.L.nz > 1) d += (w[widx(F, gi, gj, gk + 1)] - w[c]) / F.L.dxyz[2];
  return d;
}

// b = -div u* on fluid cells (ns_solver.cpp:482-498).
__global__ void __launch_bounds__(NT) k_div(FlowView F, const double* __restrict__ u,
                                            const double* __restrict__ v, const double* __restrict__ w,
                                            double* __restrict__ b) {
  const LevelView& L = F.L;
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    double o = 0.0;
    if (L.type[c] == CELL_FLUID) {
      int gi, gj, gk;
      cell_coords(L, c, gi, gj, gk);
      o = -div_at(F, u, v, w, c, gi, gj, gk);
    }
    b[c] = o;
  }
}

// phi with BC ghosts: Neumann at wall/inlet, Dirichlet-0 sign flip at the
// outlet, periodic wrap (ns_solver.cpp:508-526).
__device__ __forceinline__ double phi_at(const FlowView& F, const double* __restrict__ phi, int i,
                                         int j, int k) {
  const LevelView& L = F.L;
  int c[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  double sgn = 1.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double f = 1.0;
    if (c[a] < 0 || c[a] >= n[a]) {
      if (F.per[a]) {
        c[a] = wrapi(c[a], n[a]);
      } else {
        const int face = 2 * a + (c[a] < 0 ? 0 : 1);
        c[a] = c[a] < 0 ? 0 : n[a] - 1;
        f = L.bc[face] == NB_BC_OUTLET ? -1.0 : 1.0;
      }
    }
    sgn *= f;
  }
  return sgn * phi[cell_index(L, c[0], c[1], c[2])];
}

// u -= d(phi)/dn on every face not touching a solid, incl. boundary faces
// (ns_solver.cpp:528-562); p = phi / dt (ns_solver.cpp:575-578).
__global__ void __launch_bounds__(NT) k_correct(FlowView F, const double* __restrict__ phi,
                                                const double* __restrict__ dtp,
                                                double* __restrict__ u, double* __restrict__ v,
                                                double* __restrict__ w, double* __restrict__ p) {
  const LevelView& L = F.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const double dt = *dtp;
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    const uint8_t ty = L.type[c];
    if (ty == CELL_VOID) continue;
    int gi, gj, gk;
    cell_coords(L, c, gi, gj, gk);
    const bool sc = ty == CELL_SOLID;
    const double pc = phi_at(F, phi, gi, gj, gk);
    if (!sc && !is_solid_g(L, gi - 1, gj, gk))
      u[c] -= (pc - phi_at(F, phi, gi - 1, gj, gk)) / L.dxyz[0];
    if (gi == nx - 1 && !sc) {
      const long long s = uidx(F, nx, gj, gk);
      u[s] -= (phi_at(F, phi, nx, gj, gk) - pc) / L.dxyz[0];
    }
    if (!sc && !is_solid_g(L, gi, gj - 1, gk))
      v[c] -= (pc - phi_at(F, phi, gi, gj - 1, gk)) / L.dxyz[1];
    if (gj == ny - 1 && !sc) {
      const long long s = vidx(F, gi, ny, gk);
      v[s] -= (phi_at(F, phi, gi, ny, gk) - pc) / L.dxyz[1];
    }
    if (nz > 1) {
      if (!sc && !is_solid_g(L, gi, gj, gk - 1))
        w[c] -= (pc - phi_at(F, phi, gi, gj, gk - 1)) / L.dxyz[2];
      if (gk == nz - 1 && !sc) {
        const long long s = widx(F, gi, gj, nz);
        w[s] -= (phi_at(F, phi, gi, gj, nz) - pc) / L.dxyz[2];
      }
    }
    p[c] = phi[c] / dt;
  }
}

// Step diagnostics (ns_solver.cpp:605-763, :797-823) in one pass:
// [0] sum (u-u0)^2 over all faces, [1] sum div^2 (fluid), [2] max |div|,
// [3] fx, [4] fy, [5] net boundary mass flux.
__global__ void __launch_bounds__(NT) k_diag(FlowView F, const double* __restrict__ u,
                                             const double* __restrict__ v, const double* __restrict__ w,
                                             const double* __restrict__ u0, const double* __restrict__ v0,
                                             const double* __restrict__ w0, const double* __restrict__ p,
                                             RedBuf rb, StepScalars* out) {
  const LevelView& L = F.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const double dxv = L.dxyz[0], dyv = L.dxyz[1], dzv = L.dxyz[2];
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  auto sq = [](double a) { return a * a; };
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    const uint8_t ty = L.type[c];
    if (ty == CELL_VOID) continue;
    int gi, gj, gk;
    cell_coords(L, c, gi, gj, gk);
    acc[0] += sq(u[c] - u0[c]) + sq(v[c] - v0[c]) + sq(w[c] - w0[c]);
    if (gi == nx - 1) {
      const long long s = uidx(F, nx, gj, gk);
      acc[0] += sq(u[s] - u0[s]);
    }
    if (gj == ny - 1) {
      const long long s = vidx(F, gi, ny, gk);
      acc[0] += sq(v[s] - v0[s]);
    }
    if (gk == nz - 1) {
      const long long s = widx(F, gi, gj, nz);
      acc[0] += sq(w[s] - w0[s]);
    }
    if (ty == CELL_FLUID) {
      const double d = div_at(F, u, v, w, c, gi, gj, gk);
      acc[1] += d * d;
      acc[2] = fmax(acc[2], fabs(d));
    }
    // net boundary mass flux (ns_solver.cpp:651-675)
    if (gi == 0) acc[5] += (u[c] - u[uidx(F, nx, gj, gk)]) * (dyv * dzv);
    if (gj == 0) acc[5] += (v[c] - v[vidx(F, gi, ny, gk)]) * (dxv * dzv);
    if (nz > 1 && gk == 0) acc[5] += (w[c] - w[widx(F, gi, gj, nz)]) * (dxv * dyv);
    // forces on solid faces (ns_solver.cpp:703-763)
    if (F.has_solid && ty == CELL_FLUID) {
      const double mu = F.nu * F.density;
      const int nd = nz > 1 ? 6 : 4;
      const double uc = 0.5 * (u[c] + u[uidx(F, gi + 1, gj, gk)]);
      const double vc = 0.5 * (v[c] + v[vidx(F, gi, gj + 1, gk)]);
      for (int d = 0; d < nd; ++d) {
        const int axis = d >> 1;
        const int sgnd = (d & 1) ? 1 : -1;
        const int si = gi + (axis == 0 ? sgnd : 0), sj = gj + (axis == 1 ? sgnd : 0),
                  sk = gk + (axis == 2 ? sgnd : 0);
        if (!is_solid_g(L, si, sj, sk)) continue;
        const double area = axis == 0 ? dyv * dzv : (axis == 1 ? dxv * dzv : dxv * dyv);
        const double dn = L.dxyz[axis];
        const double nox = axis == 0 ? -static_cast<double>(sgnd) : 0.0;
        const double noy = axis == 1 ? -static_cast<double>(sgnd) : 0.0;
        const double pf = p[c];
        acc[3] += -pf * nox * area;
        acc[4] += -pf * noy * area;
        if (axis != 0) acc[3] += mu * uc / (0.5 * dn) * area;
        if (axis != 1) acc[4] += mu * vc / (0.5 * dn) * area;
      }
    }
  }
  grid_reduce<6, (1u << 2)>(acc, rb, [=] __device__(const double* t) {
    out->du2 = t[0];
    out->div2 = t[1];
    out->divmax = t[2] < 0.0 ? 0.0 : t[2];
    out->fx = t[3];
    out->fy = t[4];
    out->mass = t[5];
  });
}

// computeDt reduction (ns_solver.cpp:581-603).
__global__ void __launch_bounds__(NT) k_max_inv(FlowView F, const double* __restrict__ u,
                                                const double* __restrict__ v,
                                                const double* __restrict__ w, double visc, double cfl,
                                                double* dt_out, RedBuf rb,
                                                StepScalars* out) {
  const LevelView& L = F.L;
  const int twoD = L.twoD;
  double m[1] = {visc + 1e-300};
  for (int brick = blockIdx.x; brick < L.nbrick; brick += gridDim.x) {
    const int c = brick * BR3 + threadIdx.x;
    if (L.type[c] != CELL_FLUID) continue;
    int gi, gj, gk;
    cell_coords(L, c, gi, gj, gk);
    const double uc = fabs(0.5 * (u[c] + u[uidx(F, gi + 1, gj, gk)]));
    const double vc = fabs(0.5 * (v[c] + v[vidx(F, gi, gj + 1, gk)]));
    const double wc = twoD ? 0.0 : fabs(0.5 * (w[c] + w[widx(F, gi, gj, gk + 1)]));
    const double inv = uc / L.dxyz[0] + vc / L.dxyz[1] + (twoD ? 0.0 : wc / L.dxyz[2]) + visc;
    m[0] = fmax(m[0], inv);
  }
  grid_reduce<1, 1u>(m, rb, [=] __device__(const double* t) {
    out->maxinv = t[0];
    if (dt_out) *dt_out = cfl / t[0];  // ns_solver.cpp:602
  });
}

// lexicographic <-> brick conversion (one thread per lexicographic element)
__global__ void k_convert(FlowView F, int comp, int dir, const double* __restrict__ src,
                          double* __restrict__ dst, long long n) {
  const int nx = F.L.nx, ny = F.L.ny;
  const int ex = nx + (comp == 0), ey = ny + (comp == 1);
  for (long long m = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; m < n;
       m += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(m % ex);
    const int j = static_cast<int>((m / ex) % ey);
    const int k = static_cast<int>(m / (static_cast<long long>(ex) * ey));
    long long s;
    if (comp == 0) s = uidx(F, i, j, k);
    else if (comp == 1) s = vidx(F, i, j, k);
    else if (comp == 2) s = widx(F, i, j, k);
    else s = cell_index(F.L, i, j, k);
    if (dir == 0) dst[s] = src[m];
    else dst[m] = src[s];
  }
}

// Cell-centred values at points (BaselineBackend::sample,
// core/src/adaptive/run.cpp:49-62): the containing cell, indices truncated
// toward zero and clamped into the grid, then NSSolver::cellU/V/W
// (ns_solver.cpp:677-688) or the cell's pressure.
__global__ void k_sample(FlowView F, int comp, long long n, const double* __restrict__ xyz,
                         const double* __restrict__ u, const double* __restrict__ v,
                         const double* __restrict__ w, const double* __restrict__ p, double* __restrict__ out) {
  const LevelView& L = F.L;
  const int dims[3] = {L.nx, L.ny, L.nz};
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double d = fmin(fmax((xyz[3 * q + a] - F.origin[a]) / L.dxyz[a], -1.0), static_cast<double>(dims[a]));
      c[a] = min(max(static_cast<int>(d), 0), dims[a] - 1);
    }
    double val;
    if (comp == 0) val = 0.5 * (u[uidx(F, c[0], c[1], c[2])] + u[uidx(F, c[0] + 1, c[1], c[2])]);
    else if (comp == 1) val = 0.5 * (v[vidx(F, c[0], c[1], c[2])] + v[vidx(F, c[0], c[1] + 1, c[2])]);
    else if (comp == 2) val = 0.5 * (w[widx(F, c[0], c[1], c[2])] + w[widx(F, c[0], c[1], c[2] + 1)]);
    else val = p[cell_index(L, c[0], c[1], c[2])];
    out[q] = val;
  }
}

}  // namespace

long long lex_size(const FlowView& F, int comp) {
  const long long nx = F.L.nx, ny = F.L.ny, nz = F.L.nz;
  switch (comp) {
    case 0: return (nx + 1) * ny * nz;
    case 1: return nx * (ny + 1) * nz;
    case 2: return nx * ny * (nz + 1);
    default: return nx * ny * nz;
  }
}

long long store_size(const FlowView& F, int comp) {
  const long long nx = F.L.nx, ny = F.L.ny, nz = F.L.nz;
  switch (comp) {
    case 0: return F.nb + ny * nz;
    case 1: return F.nb + nx * nz;
    case 2: return F.nb + nx * ny;
    default: return F.nb;
  }
}

void flow_kernel_setup() {
  NB_CUDA(cudaFuncSetAttribute(k_rhs_rk<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               3 * TN * static_cast<int>(sizeof(double))));
  NB_CUDA(cudaFuncSetAttribute(k_rhs_rk<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               3 * TN * static_cast<int>(sizeof(float))));
}

void launch_bc(cudaStream_t s, const BcOp* ops, int n, int serial, double* u, double* v, double* w) {
  if (n <= 0) return;
  const int grid = serial ? 1 : std::min((n + 255) / 256, 1024);
  k_bc<<<grid, 256, 0, s>>>(ops, n, serial, u, v, w);
  NB_CUDA(cudaGetLastError());
}

void launch_rhs_rk(cudaStream_t s, const FlowView& F, int stage, const double* dtp, const double* u,
                   const double* v, const double* w, const double* u0, const double* v0,
                   const double* w0, double* uo, double* vo, double* wo, int mixed, int grid_cap) {
  const int grid = std::min(F.L.nbrick, std::max(grid_cap, 1));
  if (mixed)
    k_rhs_rk<float><<<grid, RHS_NT, 3 * TN * sizeof(float), s>>>(F, stage, dtp, u, v, w, u0, v0, w0, uo,
                                                                 vo, wo);
  else
    k_rhs_rk<double><<<grid, RHS_NT, 3 * TN * sizeof(double), s>>>(F, stage, dtp, u, v, w, u0, v0, w0,
                                                                   uo, vo, wo);
  NB_CUDA(cudaGetLastError());
}

void launch_div(cudaStream_t s, const FlowView& F, const double* u, const double* v, const double* w,
                double* b) {
  k_div<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, b);
  NB_CUDA(cudaGetLastError());
}

void launch_correct(cudaStream_t s, const FlowView& F, const double* phi, const double* dtp, double* u,
                    double* v, double* w, double* p) {
  k_correct<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, phi, dtp, u, v, w, p);
  NB_CUDA(cudaGetLastError());
}

void launch_diag(cudaStream_t s, const FlowView& F, const double* u, const double* v,
                 const double* w, const double* u0, const double* v0, const double* w0,
                 const double* p, RedBuf rb, StepScalars* out) {
  k_diag<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, u0, v0, w0, p, rb, out);
  NB_CUDA(cudaGetLastError());
}

void launch_sample(cudaStream_t s, const FlowView& F, int comp, long long n, const double* xyz, const double* u,
                   const double* v, const double* w, const double* p, double* out) {
  if (n <= 0) return;
  const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, 148 * 8));
  k_sample<<<grid, 256, 0, s>>>(F, comp, n, xyz, u, v, w, p, out);
  NB_CUDA(cudaGetLastError());
}

void launch_max_inv(cudaStream_t s, const FlowView& F, const double* u, const double* v,
                    const double* w, double visc, double cfl, double* dt_out, RedBuf rb,
                    StepScalars* out) {
  k_max_inv<<<grid_for(F.L.nbrick), NT, 0, s>>>(F, u, v, w, visc, cfl, dt_out, rb, out);
  NB_CUDA(cudaGetLastError());
}

void launch_convert(cudaStream_t s, const FlowView& F, int comp, int dir, const double* src,
                    double* dst) {
  const long long n = lex_size(F, comp);
  const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, 148 * 16));
  k_convert<<<grid, 256, 0, s>>>(F, comp, dir, src, dst, n);
  NB_CUDA(cudaGetLastError());
}

}  // namespace nb
