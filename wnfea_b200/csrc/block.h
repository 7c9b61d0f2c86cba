// Multi-right-hand-side (batched) PCG workspace: up to kBatch load cases solved together
// against one assembled matrix and one AMG hierarchy.
//
// Layout: a batched vector of n scalar DOFs is n x kBatch, DOF-major with the kBatch load
// cases of one DOF contiguous (element (i, j) at i * kBatch + j; 128 B per DOF in FP32, 256 B
// in FP64).  A block row of the matrix is handled by 8 lanes, each owning 4 consecutive load
// cases, so every matrix block is read once per product for all kBatch cases.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "amg.h"
#include "device_array.h"

namespace wn {

constexpr int kBatch = 32;

// per-load-case PCG state (device)
struct BlockScalars {
  double rz[kBatch];      // r . z of the current iteration
  double alpha[kBatch];   // step of the current iteration (0 for finished cases)
  double beta[kBatch];    // p = z + beta p of the next iteration (0 for finished cases)
  double bnorm2[kBatch];  // ||b_j||^2
  double tol2[kBatch];    // (rtol_j ||b_j||)^2
  double rr[kBatch];      // ||r_j||^2 of the last check
  int col_done[kBatch];
  int col_iters[kBatch];
  int col_status[kBatch];
  int done;      // every case finished (or the iteration limit reached)
  int iters;     // iterations of the batch
  int status;
  int max_iter;
};

template <typename T>
struct BatchLevelVecs {
  DArray<T> b, x, x2, r, d, d2, res;
  int alloc(int64_t n) {
    WN_CHECK(b.alloc(n));
    WN_CHECK(x.alloc(n));
    WN_CHECK(x2.alloc(n));
    WN_CHECK(r.alloc(n));
    WN_CHECK(d.alloc(n));
    WN_CHECK(d2.alloc(n));
    WN_CHECK(res.alloc(n));
    return 0;
  }
};

struct BlockWork {
  int64_t n = 0;  // scalar DOFs of the fine level
  static constexpr int kMaxParts = 148 * 16;
  int npA = 0, npB = 0, npC = 0;
  DArray<double> partA, partB, partC;  // kMaxParts x kBatch
  DArray<BlockScalars> scal;           // [0] inner PCG, [1] outer column norms
  DArray<double> rtol_cols;            // kBatch inner targets
  std::vector<double> h_rtol;
  // outer refinement: F, U = U + Ulo (double-double), R = F - K U
  DArray<double> F, U, Ulo, R;
  // Krylov vectors (FP64)
  DArray<double> x, r, p0, p1, q;
  // 1 / diag of the fine matrix (refreshed per solve)
  DArray<double> dinv64;
  DArray<float> dinv32;
  // preconditioner input / output in the V-cycle precision
  DArray<float> z32, r32;
  DArray<double> z64;
  // the fine V-cycle's first smoothing input dinv r / theta, written by the PCG update
  DArray<float> d0_32;
  DArray<double> d0_64;
  // V-cycle vectors per level and the coarsest right-hand side / solution
  std::vector<BatchLevelVecs<float>> lv32;
  std::vector<BatchLevelVecs<double>> lv64;
  DArray<float> cb32, cx32;
  DArray<double> cb64, cx64;
  uint64_t hierarchy_id = 0;        // the AmgHierarchy the level vectors were sized for
  // x-tiles of the fine level (block_solver.cu build_x_tiles): runs of rows whose blocks name at
  // most 256 columns; per tile its sorted columns, per block its column's index among them
  DArray<int32_t> xt_rows, xt_col_ptr, xt_cols;
  DArray<uint8_t> xt_lcol;
  int xt_n = 0;         // tiles (0: no plan)
  bool xt_tried = false;
  GraphCache graphs[2][3];          // [V-cycle precision 0 fp64 / 1 fp32][preconditioner]
  int64_t launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t own = nullptr;
  ~BlockWork() {
    for (auto& a : graphs)
      for (auto& g : a) g.reset();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own) cudaStreamDestroy(own);
  }
};

}  // namespace wn
