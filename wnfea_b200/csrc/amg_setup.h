// Host-side smoothed-aggregation AMG setup for 3-DOF (C3D10) and 6-DOF block systems.
#pragma once

#include <stdint.h>

#include <vector>

#include "wnfea_cuda.h"

namespace wn {

struct HostBsr {
  int br = 0, bc = 0;
  int64_t n_rows = 0, n_cols = 0;  // block rows / block columns
  std::vector<int32_t> rp, ci;
  std::vector<double> v;           // nnzb * br * bc, row-major blocks
  int64_t nnzb() const { return (int64_t)ci.size(); }
};

struct HostLevel {
  HostBsr A;                 // empty for level 0 (the assembled matrix is used in place)
  int bs = 3;                // DOFs per node of this level
  int64_t n_nodes = 0;
  std::vector<double> dinv;  // 1 / diag(A), n_nodes * bs
  double rho = 0.0;          // spectral radius estimate of D^-1 A
  HostBsr P, R;              // prolongation (bs x 6 blocks) and restriction R = P^T (6 x bs)
  std::vector<int32_t> agg;  // node -> aggregate (-1 = not aggregated)
  int64_t n_agg = 0;
};

struct HostHierarchy {
  wn_amg_params params{};
  std::vector<HostLevel> levels;  // levels[0..L-1] have P/R; the coarsest matrix is dense
  int64_t n_coarse = 0;           // scalar DOFs of the coarsest level
  std::vector<double> coarse_A;   // dense coarsest matrix (row-major), FP64
  std::vector<double> coarse_inv; // A_c^-1 = L^-T L^-1 from its Cholesky factor, FP64
};

// Build the hierarchy from the fine BSR3 matrix (FP64), node coordinates (n x 3) and the
// Dirichlet mask (3n, may be null).  Returns WN_OK or a WN_E* code (message set).
int amg_build(const wn_amg_params& prm, int64_t n0, int bs0, const int32_t* rp0, const int32_t* ci0,
              const double* v0, const double* coords, const uint8_t* fixed, HostHierarchy& out);

wn_amg_params amg_default_params();

// Pieces shared by the host setup above and the device setup (amg_device.cu):
// greedy aggregation from block norms (-1 = unaggregated); the rigid-body near-null space of
// level 0; the tentative prolongator (per-aggregate QR: Qnode n x bs x 6, Bc n_agg x 36); the
// dense coarsest level (out.n_coarse, coarse_A, coarse_inv).
int64_t aggregate_norms(int64_t n, const int32_t* rp, const int32_t* ci, const double* nrm, double theta,
                        std::vector<int32_t>& agg);
void near_null_space(int64_t n0, int bs0, const double* coords, const uint8_t* fixed, std::vector<double>& B);
void tentative_prolongator(int64_t n, int bs, int64_t n_agg, const std::vector<int32_t>& agg,
                           const std::vector<double>& B, std::vector<double>& Qnode, std::vector<double>& Bc);
int dense_coarse(int64_t n, int bs, const int32_t* rp, const int32_t* ci, const double* v, HostHierarchy& out);

}  // namespace wn
