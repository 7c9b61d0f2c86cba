// C3D10 element geometry on the device: natural derivatives at the Hammer 4-point rule,
// Jacobian, inverse and Cartesian derivatives.  Restates wnfea/elements/c3d10.py:21-137
// (and the matching constants of wnfea/solver/native/kernels.cpp:212-240).
#pragma once

#include <cuda_runtime.h>

namespace wn {

// Hammer rule: alpha = (5 - sqrt 5) / 20, beta = (5 + 3 sqrt 5) / 20, weight 1/24.
// Point g has volume coordinates (L2, L3, L4) = GP[g] (c3d10.py:25-30 arrays).
constexpr double kAlpha = 0.1381966011250105151795413165634361882280;
constexpr double kBeta = 0.5854101966249684544613760503096914353161;
constexpr double kWeight = 1.0 / 24.0;

__device__ __forceinline__ void gauss_point(int g, double& xi, double& eta, double& zeta) {
  xi = (g == 1) ? kBeta : kAlpha;
  eta = (g == 2) ? kBeta : kAlpha;
  zeta = (g == 3) ? kBeta : kAlpha;
}

// dN/dxi (3 x 10) at natural point (xi, eta, zeta): chain rule through the volume
// coordinates L1 = 1 - xi - eta - zeta, L2 = xi, L3 = eta, L4 = zeta (c3d10.py:84-104).
__device__ __forceinline__ void natural_derivs(double xi, double eta, double zeta, double dn[3][10]) {
  const double L1 = 1.0 - xi - eta - zeta, L2 = xi, L3 = eta, L4 = zeta;
  // dN/dL columns per node: d1 = dN/dL1, ...
  double d1[10] = {4 * L1 - 1, 0, 0, 0, 4 * L2, 0, 4 * L3, 4 * L4, 0, 0};
  double d2[10] = {0, 4 * L2 - 1, 0, 0, 4 * L1, 4 * L3, 0, 0, 4 * L4, 0};
  double d3[10] = {0, 0, 4 * L3 - 1, 0, 0, 4 * L2, 4 * L1, 0, 0, 4 * L4};
  double d4[10] = {0, 0, 0, 4 * L4 - 1, 0, 0, 0, 4 * L1, 4 * L2, 4 * L3};
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    dn[0][a] = d2[a] - d1[a];
    dn[1][a] = d3[a] - d1[a];
    dn[2][a] = d4[a] - d1[a];
  }
}

// Cartesian derivatives dN/dx (3 x 10) and det J at Gauss point g for element coordinates
// X[10][3].  Returns det J (the caller rejects det J <= 0 like c3d10.py:129-134).
__device__ __forceinline__ double gp_cartesian(int g, const double X[10][3], double dndx[3][10]) {
  double xi, eta, zeta;
  gauss_point(g, xi, eta, zeta);
  double dn[3][10];
  natural_derivs(xi, eta, zeta, dn);
  // J = dN/dxi X with X taken relative to node 0: the same matrix (the derivatives of the shape
  // functions sum to zero), without the cancellation of absolute coordinates -- an element 4 m
  // from the origin with 1 cm edges would lose about three digits of J (c3d10.py:109-137 uses
  // the absolute coordinates; its Ke there carries relative errors up to ~4e-13)
  double J[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
#pragma unroll
      for (int a = 1; a < 10; ++a) s = fma(dn[k][a], X[a][j] - X[0][j], s);
      J[k][j] = s;
    }
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  double inv[3][3];
  inv[0][0] = c00 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][0] = c01 * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][0] = c02 * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int a = 0; a < 10; ++a) dndx[i][a] = inv[i][0] * dn[0][a] + inv[i][1] * dn[1][a] + inv[i][2] * dn[2][a];
  return det;
}

// dN_a/dxi_k at Gauss point g: the value natural_derivs gives, as a constant expression (the
// same operations in the same order; 4 x is exact, so a contracted 4 x - 1 rounds alike), so
// that the terms of a zero derivative drop out of the sums below at compile time.
__host__ __device__ constexpr double nat_deriv(int g, int k, int a) {
  const double xi = (g == 1) ? kBeta : kAlpha, eta = (g == 2) ? kBeta : kAlpha, zeta = (g == 3) ? kBeta : kAlpha;
  const double L1 = 1.0 - xi - eta - zeta, L2 = xi, L3 = eta, L4 = zeta;
  const double d1[10] = {4 * L1 - 1, 0, 0, 0, 4 * L2, 0, 4 * L3, 4 * L4, 0, 0};
  const double d2[10] = {0, 4 * L2 - 1, 0, 0, 4 * L1, 4 * L3, 0, 0, 4 * L4, 0};
  const double d3[10] = {0, 0, 4 * L3 - 1, 0, 0, 4 * L2, 4 * L1, 0, 0, 4 * L4};
  const double d4[10] = {0, 0, 0, 4 * L4 - 1, 0, 0, 0, 4 * L1, 4 * L2, 4 * L3};
  return (k == 0 ? d2[a] : (k == 1 ? d3[a] : d4[a])) - d1[a];
}

// J[K][j] = sum over a = A..9 of dN_a/dxi_K (X_a - X_0)_j, zero derivatives skipped (fma with a
// zero factor would return the running sum unchanged).
template <int G, int K, int A = 1>
__device__ __forceinline__ double jac_entry(const double Xr[10][3], int j, double s = 0.0) {
  if constexpr (A == 10) {
    return s;
  } else {
    constexpr double c = nat_deriv(G, K, A);
    if constexpr (c != 0.0) s = fma(c, Xr[A][j], s);
    return jac_entry<G, K, A + 1>(Xr, j, s);
  }
}

// dN_A/dx_i = sum_k inv[i][k] dN_A/dxi_k, zero derivatives skipped.
template <int G, int A>
__device__ __forceinline__ double cart_entry(const double inv_i[3]) {
  constexpr double c0 = nat_deriv(G, 0, A), c1 = nat_deriv(G, 1, A), c2 = nat_deriv(G, 2, A);
  double s = 0.0;
  if constexpr (c0 != 0.0) s = fma(inv_i[0], c0, s);
  if constexpr (c1 != 0.0) s = fma(inv_i[1], c1, s);
  if constexpr (c2 != 0.0) s = fma(inv_i[2], c2, s);
  return s;
}

template <int G, int A = 0>
__device__ __forceinline__ void cart_row(const double inv_i[3], double* out) {
  if constexpr (A < 10) {
    out[A] = cart_entry<G, A>(inv_i);
    cart_row<G, A + 1>(inv_i, out);
  }
}

// gp_cartesian at a Gauss point known at compile time, from coordinates already taken relative
// to node 0 (Xr[a] = X_a - X_0; Xr[0] unused): the same J, det J and inverse, with the zero
// natural derivatives (8 of 30 in each of J's rows and dN/dx's sums) dropped.
template <int G>
__device__ __forceinline__ double gp_cartesian_rel(const double Xr[10][3], double dndx[3][10]) {
  double J[3][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    J[0][j] = jac_entry<G, 0>(Xr, j);
    J[1][j] = jac_entry<G, 1>(Xr, j);
    J[2][j] = jac_entry<G, 2>(Xr, j);
  }
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  double inv[3][3];
  inv[0][0] = c00 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][0] = c01 * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][0] = c02 * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
#pragma unroll
  for (int i = 0; i < 3; ++i) cart_row<G>(inv[i], dndx[i]);
  return det;
}

// Lame constants of the isotropic C of c3d10.py:192-216: C11 = lam + 2 mu, C12 = lam,
// shear diagonal G = mu.
__device__ __forceinline__ void lame(double E, double nu, double& lam, double& mu) {
  const double f = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  lam = f * nu;
  mu = E / (2.0 * (1.0 + nu));
}

}  // namespace wn
