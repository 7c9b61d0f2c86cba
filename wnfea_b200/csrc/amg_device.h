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
// Download the device-built level matrices into H.host (no-op for host-built hierarchies).
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
