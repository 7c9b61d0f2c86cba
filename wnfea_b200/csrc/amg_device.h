// Device-side smoothed-aggregation setup (amg_device.cu).
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "amg.h"
#include "solid.h"

namespace wn {

// Build the hierarchy of the assembled matrix of s on the device (aggregation and the
// tentative QR on the host) into H: the device levels (A for levels >= 1, P, R in FP64 and FP32,
// 1/diag), rho, the coarsest inverse, and the host metadata of H.host (dinv, rho, agg, the dense
// coarsest matrix); the host copies of the level matrices are made on demand (amg_sync_host).
// Returns 0, a WN_E* / CUDA error, or 1 when a row exceeds the shared-memory capacities of the
// device products (the caller then runs the host builder).
int amg_build_device(Solid* s, const wn_amg_params& prm, AmgHierarchy& H);
// Block-Jacobi smoothing of the 6-DOF levels (l >= 1) by a change of basis per aggregate:
// with D_i = L_i L_i^T the diagonal 6 x 6 block of node i of A_l and T_l = diag(L_i^-T),
//   A^_l = T_l^T A_l T_l,  P^_l = T_l^-1 P_l T_(l+1),  R^_l = P^_l^T   (T_0 = T_coarsest = I),
// so A^_l has identity diagonal blocks and the point-Jacobi / Chebyshev smoother on A^_l is the
// block-Jacobi one on A_l (D^-1 A^ = T^T D_block^-1 A T^-T), while the V-cycle's coarse
// corrections, being Galerkin, are the same operators in the new basis.  Replaces the device
// levels' A, P, R (FP64 and FP32), 1/diag and rho(D^-1 A^) (host copies: dinv and rho; the
// matrices on demand through amg_sync_host).  No-op without a 6-DOF level.
int amg_coarse_block_basis(AmgHierarchy& H, const wn_amg_params& prm);
// Download the device level matrices into H.host when they are newer than the host copies
// (device-built levels, or levels moved to the block basis); no-op otherwise.
int amg_sync_host(AmgHierarchy& H);

// WN_AMG_TRACE=1 in the environment: phase times of a setup on stderr
struct PhaseClock {
  const char* who;
  bool on;
  std::chrono::steady_clock::time_point t;
  explicit PhaseClock(const char* w)
      : who(w), on(std::getenv("WN_AMG_TRACE") != nullptr), t(std::chrono::steady_clock::now()) {}
  void mark(const char* what, int lvl) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "%s: level %d %-12s %8.3f s\n", who, lvl, what,
                 std::chrono::duration<double>(now - t).count());
    t = now;
  }
};

}  // namespace wn
