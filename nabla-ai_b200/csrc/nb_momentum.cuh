// nb_momentum.cuh — momentum right-hand sides of the staggered step on a
// staged tile: divergence-form WENO-5 (or central) convection with advecting
// velocity = average of the two neighbouring faces of the other component,
// plus the 7-point viscous Laplacian and the body force
// (core/src/flow/ns_solver.cpp:15-42, :311-473). `U(i,j,k)` etc. read the
// tile at brick-local offsets; dx, dy, dz are the cell sizes of the tile.
#pragma once

namespace nb {

template <typename T>
__device__ __forceinline__ T weno5_t(T v0, T v1, T v2, T v3, T v4) {
  const T eps = T(1e-12);
  const T c1312 = T(13.0 / 12.0), q = T(0.25);
  const T b0 = c1312 * (v0 - T(2) * v1 + v2) * (v0 - T(2) * v1 + v2) +
               q * (v0 - T(4) * v1 + T(3) * v2) * (v0 - T(4) * v1 + T(3) * v2);
  const T b1 = c1312 * (v1 - T(2) * v2 + v3) * (v1 - T(2) * v2 + v3) + q * (v1 - v3) * (v1 - v3);
  const T b2 = c1312 * (v2 - T(2) * v3 + v4) * (v2 - T(2) * v3 + v4) +
               q * (T(3) * v2 - T(4) * v3 + v4) * (T(3) * v2 - T(4) * v3 + v4);
  const T a0 = T(0.1) / ((eps + b0) * (eps + b0));
  const T a1 = T(0.6) / ((eps + b1) * (eps + b1));
  const T a2 = T(0.3) / ((eps + b2) * (eps + b2));
  const T s = a0 + a1 + a2;
  const T p0 = (T(2) * v0 - T(7) * v1 + T(11) * v2) / T(6.0);
  const T p1 = (-v1 + T(5) * v2 + T(2) * v3) / T(6.0);
  const T p2 = (T(2) * v2 + T(5) * v3 - v4) / T(6.0);
  return (a0 * p0 + a1 * p1 + a2 * p2) / s;
}

// Upwind-biased face value: the stencil is mirrored for a negative advecting
// velocity. The five inputs are selected first so that one WENO evaluation is
// emitted per call site (same value as evaluating the chosen branch).
template <typename T>
__device__ __forceinline__ T recon_t(int weno, T adv, T qm2, T qm1, T q0, T qp1, T qp2, T qp3) {
  if (!weno) return T(0.5) * (q0 + qp1);
  const bool up = adv >= T(0);
  return weno5_t<T>(up ? qm2 : qp3, up ? qm1 : qp2, up ? q0 : qp1, up ? qp1 : q0, up ? qp2 : qm1);
}

// Momentum RHS of component a at the a-face (i,j,k) of a staged tile, for any
// a: the normal direction convects component a with its own face average, each
// transverse direction d with the average of component d's two faces on
// either side of the a-face (ns_solver.cpp:322-472 written once for all three
// components). Component tiles t0, t1, t2 are indexed base + n*stride, with
// strides 1, SY, SZ along x, y, z; the flux and Laplacian terms are summed in
// x, y, z order as in rhs_u/v/w. With two_d the z terms are absent (the
// reference's nz == 1 branches).
template <typename T, int SY, int SZ>
__device__ __forceinline__ T rhs_face(const T* t0, const T* t1, const T* t2, int a, int c, int weno, T hx, T hy,
                                      T hz, T nu, T bf, bool two_d = false) {
  const T half = T(0.5);
  const T* A = a == 0 ? t0 : (a == 1 ? t1 : t2);
  const int sa = a == 0 ? 1 : (a == 1 ? SY : SZ);
  T dF[3], lap[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == 2 && two_d) {
      dF[d] = lap[d] = T(0);
      continue;
    }
    const int sd = d == 0 ? 1 : (d == 1 ? SY : SZ);
    const T hd = d == 0 ? hx : (d == 1 ? hy : hz);
    T advB, advT;
    if (d == a) {
      advB = half * (A[c - sa] + A[c]);
      advT = half * (A[c] + A[c + sa]);
    } else {
      const T* D = d == 0 ? t0 : (d == 1 ? t1 : t2);
      advT = half * (D[c - sa + sd] + D[c + sd]);
      advB = half * (D[c - sa] + D[c]);
    }
    const T qB = recon_t<T>(weno, advB, A[c - 3 * sd], A[c - 2 * sd], A[c - sd], A[c], A[c + sd], A[c + 2 * sd]);
    const T qT = recon_t<T>(weno, advT, A[c - 2 * sd], A[c - sd], A[c], A[c + sd], A[c + 2 * sd], A[c + 3 * sd]);
    dF[d] = (advT * qT - advB * qB) / hd;
    lap[d] = (A[c + sd] - T(2) * A[c] + A[c - sd]) / (hd * hd);
  }
  return -(dF[0] + dF[1] + dF[2]) + nu * ((lap[0] + lap[1]) + lap[2]) + bf;
}

// u-momentum at the x-face (i,j,k) (ns_solver.cpp:322-374).
template <typename T, class FU, class FV, class FW>
__device__ __forceinline__ T rhs_u(const FU& U, const FV& V, const FW& W, int i, int j, int k, int weno,
                                   T dx, T dy, T dz, T nu, T bf) {
  const T h = T(0.5);
  const T ucL = h * (U(i - 1, j, k) + U(i, j, k));
  const T ucR = h * (U(i, j, k) + U(i + 1, j, k));
  const T uxL = recon_t<T>(weno, ucL, U(i - 3, j, k), U(i - 2, j, k), U(i - 1, j, k), U(i, j, k), U(i + 1, j, k),
                           U(i + 2, j, k));
  const T uxR = recon_t<T>(weno, ucR, U(i - 2, j, k), U(i - 1, j, k), U(i, j, k), U(i + 1, j, k), U(i + 2, j, k),
                           U(i + 3, j, k));
  const T dFx = (ucR * uxR - ucL * uxL) / dx;
  const T vT = h * (V(i - 1, j + 1, k) + V(i, j + 1, k));
  const T vB = h * (V(i - 1, j, k) + V(i, j, k));
  const T uyT = recon_t<T>(weno, vT, U(i, j - 2, k), U(i, j - 1, k), U(i, j, k), U(i, j + 1, k), U(i, j + 2, k),
                           U(i, j + 3, k));
  const T uyB = recon_t<T>(weno, vB, U(i, j - 3, k), U(i, j - 2, k), U(i, j - 1, k), U(i, j, k), U(i, j + 1, k),
                           U(i, j + 2, k));
  const T dFy = (vT * uyT - vB * uyB) / dy;
  const T wT = h * (W(i - 1, j, k + 1) + W(i, j, k + 1));
  const T wB = h * (W(i - 1, j, k) + W(i, j, k));
  const T uzT = recon_t<T>(weno, wT, U(i, j, k - 2), U(i, j, k - 1), U(i, j, k), U(i, j, k + 1), U(i, j, k + 2),
                           U(i, j, k + 3));
  const T uzB = recon_t<T>(weno, wB, U(i, j, k - 3), U(i, j, k - 2), U(i, j, k - 1), U(i, j, k), U(i, j, k + 1),
                           U(i, j, k + 2));
  const T dFz = (wT * uzT - wB * uzB) / dz;
  T lap = (U(i + 1, j, k) - T(2) * U(i, j, k) + U(i - 1, j, k)) / (dx * dx) +
          (U(i, j + 1, k) - T(2) * U(i, j, k) + U(i, j - 1, k)) / (dy * dy);
  lap += (U(i, j, k + 1) - T(2) * U(i, j, k) + U(i, j, k - 1)) / (dz * dz);
  return -(dFx + dFy + dFz) + nu * lap + bf;
}

// v-momentum at the y-face (i,j,k) (ns_solver.cpp:376-424).
template <typename T, class FU, class FV, class FW>
__device__ __forceinline__ T rhs_v(const FU& U, const FV& V, const FW& W, int i, int j, int k, int weno,
                                   T dx, T dy, T dz, T nu, T bf) {
  const T h = T(0.5);
  const T vcB = h * (V(i, j - 1, k) + V(i, j, k));
  const T vcT = h * (V(i, j, k) + V(i, j + 1, k));
  const T vyB = recon_t<T>(weno, vcB, V(i, j - 3, k), V(i, j - 2, k), V(i, j - 1, k), V(i, j, k), V(i, j + 1, k),
                           V(i, j + 2, k));
  const T vyT = recon_t<T>(weno, vcT, V(i, j - 2, k), V(i, j - 1, k), V(i, j, k), V(i, j + 1, k), V(i, j + 2, k),
                           V(i, j + 3, k));
  const T dFy = (vcT * vyT - vcB * vyB) / dy;
  const T uR = h * (U(i + 1, j - 1, k) + U(i + 1, j, k));
  const T uL = h * (U(i, j - 1, k) + U(i, j, k));
  const T vxR = recon_t<T>(weno, uR, V(i - 2, j, k), V(i - 1, j, k), V(i, j, k), V(i + 1, j, k), V(i + 2, j, k),
                           V(i + 3, j, k));
  const T vxL = recon_t<T>(weno, uL, V(i - 3, j, k), V(i - 2, j, k), V(i - 1, j, k), V(i, j, k), V(i + 1, j, k),
                           V(i + 2, j, k));
  const T dFx = (uR * vxR - uL * vxL) / dx;
  const T wR = h * (W(i, j - 1, k + 1) + W(i, j, k + 1));
  const T wL = h * (W(i, j - 1, k) + W(i, j, k));
  const T vzR = recon_t<T>(weno, wR, V(i, j, k - 2), V(i, j, k - 1), V(i, j, k), V(i, j, k + 1), V(i, j, k + 2),
                           V(i, j, k + 3));
  const T vzL = recon_t<T>(weno, wL, V(i, j, k - 3), V(i, j, k - 2), V(i, j, k - 1), V(i, j, k), V(i, j, k + 1),
                           V(i, j, k + 2));
  const T dFz = (wR * vzR - wL * vzL) / dz;
  T lap = (V(i + 1, j, k) - T(2) * V(i, j, k) + V(i - 1, j, k)) / (dx * dx) +
          (V(i, j + 1, k) - T(2) * V(i, j, k) + V(i, j - 1, k)) / (dy * dy);
  lap += (V(i, j, k + 1) - T(2) * V(i, j, k) + V(i, j, k - 1)) / (dz * dz);
  return -(dFx + dFy + dFz) + nu * lap + bf;
}

// w-momentum at the z-face (i,j,k) (ns_solver.cpp:426-472).
template <typename T, class FU, class FV, class FW>
__device__ __forceinline__ T rhs_w(const FU& U, const FV& V, const FW& W, int i, int j, int k, int weno,
                                   T dx, T dy, T dz, T nu, T bf) {
  const T h = T(0.5);
  const T wcB = h * (W(i, j, k - 1) + W(i, j, k));
  const T wcT = h * (W(i, j, k) + W(i, j, k + 1));
  const T wzB = recon_t<T>(weno, wcB, W(i, j, k - 3), W(i, j, k - 2), W(i, j, k - 1), W(i, j, k), W(i, j, k + 1),
                           W(i, j, k + 2));
  const T wzT = recon_t<T>(weno, wcT, W(i, j, k - 2), W(i, j, k - 1), W(i, j, k), W(i, j, k + 1), W(i, j, k + 2),
                           W(i, j, k + 3));
  const T dFz = (wcT * wzT - wcB * wzB) / dz;
  const T uR = h * (U(i + 1, j, k - 1) + U(i + 1, j, k));
  const T uL = h * (U(i, j, k - 1) + U(i, j, k));
  const T wxR = recon_t<T>(weno, uR, W(i - 2, j, k), W(i - 1, j, k), W(i, j, k), W(i + 1, j, k), W(i + 2, j, k),
                           W(i + 3, j, k));
  const T wxL = recon_t<T>(weno, uL, W(i - 3, j, k), W(i - 2, j, k), W(i - 1, j, k), W(i, j, k), W(i + 1, j, k),
                           W(i + 2, j, k));
  const T dFx = (uR * wxR - uL * wxL) / dx;
  const T vR = h * (V(i, j + 1, k - 1) + V(i, j + 1, k));
  const T vL = h * (V(i, j, k - 1) + V(i, j, k));
  const T wyR = recon_t<T>(weno, vR, W(i, j - 2, k), W(i, j - 1, k), W(i, j, k), W(i, j + 1, k), W(i, j + 2, k),
                           W(i, j + 3, k));
  const T wyL = recon_t<T>(weno, vL, W(i, j - 3, k), W(i, j - 2, k), W(i, j - 1, k), W(i, j, k), W(i, j + 1, k),
                           W(i, j + 2, k));
  const T dFy = (vR * wyR - vL * wyL) / dy;
  const T lap = (W(i + 1, j, k) - T(2) * W(i, j, k) + W(i - 1, j, k)) / (dx * dx) +
                (W(i, j + 1, k) - T(2) * W(i, j, k) + W(i, j - 1, k)) / (dy * dy) +
                (W(i, j, k + 1) - T(2) * W(i, j, k) + W(i, j, k - 1)) / (dz * dz);
  return -(dFx + dFy + dFz) + nu * lap + bf;
}

}  // namespace nb
