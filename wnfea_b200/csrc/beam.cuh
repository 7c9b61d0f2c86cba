// Co-rotational 3D beam element on the device: internal force, written once for a scalar
// type S so that the same code evaluates f (S = double) and, with S = Dual, the exact
// directional derivative of f -- the consistent tangent of this formulation.
//
// Kinematics and forces restate the reference's live path (the NumPy branch of
// compute_internal_forces_fast, wnfea/solver/fast_kernels.py:451-537, identical in
// arithmetic to compute_beam_internal_forces_native, wnfea/solver/native/kernels.cpp:19-204):
// Rodrigues rotation of the reference triad onto the current chord, average nodal twist,
// Gram-Schmidt, local deformations [u_l, th_y1, th_z1, th_x, th_y2, th_z2], local forces
// q = [N, My1, Mz1, Tx, My2, Mz2] and f = B^T q at 6 DOFs per node.
#pragma once

#include <cuda_runtime.h>

namespace wn {

// Forward-mode dual number: value and one directional derivative.
struct Dual {
  double v, d;
  __device__ __forceinline__ Dual() : v(0.0), d(0.0) {}
  __device__ __forceinline__ Dual(double a) : v(a), d(0.0) {}
  __device__ __forceinline__ Dual(double a, double b) : v(a), d(b) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
__device__ __forceinline__ Dual wsqrt(Dual a) {
  const double s = ::sqrt(a.v);
  return Dual(s, s > 0.0 ? 0.5 * a.d / s : 0.0);
}
__device__ __forceinline__ Dual wsin(Dual a) { return Dual(::sin(a.v), ::cos(a.v) * a.d); }
__device__ __forceinline__ Dual wcos(Dual a) { return Dual(::cos(a.v), -::sin(a.v) * a.d); }
__device__ __forceinline__ Dual watan2(Dual y, Dual x) {
  const double r2 = x.v * x.v + y.v * y.v;
  return Dual(::atan2(y.v, x.v), r2 > 0.0 ? (x.v * y.d - y.v * x.d) / r2 : 0.0);
}
// the same four functions for S = double
__device__ __forceinline__ double wsqrt(double a) { return ::sqrt(a); }
__device__ __forceinline__ double wsin(double a) { return ::sin(a); }
__device__ __forceinline__ double wcos(double a) { return ::cos(a); }
__device__ __forceinline__ double watan2(double y, double x) { return ::atan2(y, x); }
__device__ __forceinline__ double value(double a) { return a; }
__device__ __forceinline__ double value(Dual a) { return a.v; }

template <typename S>
__device__ __forceinline__ S dot3(const S a[3], const S b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
template <typename S>
__device__ __forceinline__ void cross3(const S a[3], const S b[3], S c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Element internal force f (12: node 1 forces, node 1 moments, node 2 forces, node 2
// moments) for displacements/rotations u1, th1, u2, th2.  x1, x2: undeformed node
// coordinates; e: reference triad rows e1_0, e2_0, e3_0; L0: undeformed length;
// p = [E, G, A, Iy, Iz, J].
template <typename S>
__device__ void beam_internal_force(const double x1[3], const double x2[3], const double e[9], double L0,
                                    const double p[6], const S u1[3], const S th1[3], const S u2[3], const S th2[3],
                                    S f[12]) {
  const double v0[3] = {x2[0] - x1[0], x2[1] - x1[1], x2[2] - x1[2]};
  const S du[3] = {u2[0] - u1[0], u2[1] - u1[1], u2[2] - u1[2]};
  const S v[3] = {v0[0] + du[0], v0[1] + du[1], v0[2] + du[2]};
  const S L = wsqrt(dot3(v, v));
  const S inv_L = 1.0 / L;
  const S r1[3] = {v[0] * inv_L, v[1] * inv_L, v[2] * inv_L};
  const S e1[3] = {S(e[0]), S(e[1]), S(e[2])};
  S cr[3];
  cross3(e1, r1, cr);
  const S sin_phi = wsqrt(dot3(cr, cr));
  const S cos_phi = dot3(e1, r1);
  S r2[3] = {S(e[3]), S(e[4]), S(e[5])};
  S r3[3] = {S(e[6]), S(e[7]), S(e[8])};
  if (value(sin_phi) > 1e-12) {  // Rodrigues rotation of e2_0, e3_0 by phi about ax
    const S inv_s = 1.0 / sin_phi;
    const S ax[3] = {cr[0] * inv_s, cr[1] * inv_s, cr[2] * inv_s};
    const S phi = watan2(sin_phi, cos_phi);
    const S cp = wcos(phi), sp = wsin(phi);
    const S e2[3] = {S(e[3]), S(e[4]), S(e[5])};
    const S e3[3] = {S(e[6]), S(e[7]), S(e[8])};
    S a2[3], a3[3];
    cross3(ax, e2, a2);
    cross3(ax, e3, a3);
    const S ad2 = dot3(ax, e2), ad3 = dot3(ax, e3);
    for (int k = 0; k < 3; ++k) {
      r2[k] = e2[k] * cp + a2[k] * sp + ax[k] * ad2 * (1.0 - cp);
      r3[k] = e3[k] * cp + a3[k] * sp + ax[k] * ad3 * (1.0 - cp);
    }
  }
  // average nodal twist about the chord
  const S ths[3] = {th1[0] + th2[0], th1[1] + th2[1], th1[2] + th2[2]};
  const S tw = 0.5 * dot3(ths, r1);
  const S ct = wcos(tw), st = wsin(tw);
  S c12[3], c13[3];
  cross3(r1, r2, c12);
  cross3(r1, r3, c13);
  for (int k = 0; k < 3; ++k) {
    r2[k] = r2[k] * ct + c12[k] * st;
    r3[k] = r3[k] * ct + c13[k] * st;
  }
  // Gram-Schmidt
  const S d21 = dot3(r2, r1);
  for (int k = 0; k < 3; ++k) r2[k] = r2[k] - d21 * r1[k];
  const S n2 = 1.0 / wsqrt(dot3(r2, r2));
  for (int k = 0; k < 3; ++k) r2[k] = r2[k] * n2;
  cross3(r1, r2, r3);
  const S n3 = 1.0 / wsqrt(dot3(r3, r3));
  for (int k = 0; k < 3; ++k) r3[k] = r3[k] * n3;
  // local deformations
  const S v0du = v0[0] * du[0] + v0[1] * du[1] + v0[2] * du[2];
  const S u_l = (2.0 * v0du + dot3(du, du)) / (L + L0);
  const S r3du = dot3(r3, du), r2du = dot3(r2, du);
  const S dth[3] = {th2[0] - th1[0], th2[1] - th1[1], th2[2] - th1[2]};
  const S thy1 = dot3(r2, th1) + r3du * inv_L;
  const S thz1 = dot3(r3, th1) - r2du * inv_L;
  const S thx = dot3(r1, dth);
  const S thy2 = dot3(r2, th2) + r3du * inv_L;
  const S thz2 = dot3(r3, th2) - r2du * inv_L;
  // local forces q = [N, My1, Mz1, Tx, My2, Mz2]
  const double E = p[0], G = p[1], A = p[2], Iy = p[3], Iz = p[4], J = p[5];
  const S N = (E * A / L0) * u_l;
  const S My1 = (E * Iy / L0) * (4.0 * thy1 + 2.0 * thy2);
  const S My2 = (E * Iy / L0) * (2.0 * thy1 + 4.0 * thy2);
  const S Mz1 = (E * Iz / L0) * (4.0 * thz1 + 2.0 * thz2);
  const S Mz2 = (E * Iz / L0) * (2.0 * thz1 + 4.0 * thz2);
  const S Tx = (G * J / L0) * thx;
  const S shz = (My1 + My2) * inv_L;
  const S shy = (Mz1 + Mz2) * inv_L;
  for (int k = 0; k < 3; ++k) {
    const S f1 = -N * r1[k] - shz * r3[k] + shy * r2[k];
    f[k] = f1;
    f[3 + k] = -Tx * r1[k] + My1 * r2[k] + Mz1 * r3[k];
    f[6 + k] = -f1;
    f[9 + k] = Tx * r1[k] + My2 * r2[k] + Mz2 * r3[k];
  }
}

}  // namespace wn
