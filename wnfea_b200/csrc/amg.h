// Device-resident AMG hierarchy and solver workspace.
#pragma once

#include <string>

#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <vector>

#include "amg_setup.h"
#include "device_array.h"
#include "stream_mat.h"

namespace wn {

struct DevBsr {
  int br = 0, bc = 0;
  int64_t n_rows = 0, n_cols = 0, nnzb = 0;
  DArray<int32_t> rp, ci;
  DArray<double> v64;
  DArray<float> v32;
  int upload(const HostBsr& h);
};

// work vectors of one level in one precision
template <typename T>
struct LevelVecs {
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

struct DevLevel {
  int bs = 3;
  int64_t n_nodes = 0;
  // A: level 0 borrows the system's matrix; coarser levels own theirs
  const int32_t* a_rp = nullptr;
  const int32_t* a_ci = nullptr;
  const double* a64 = nullptr;
  const float* a32 = nullptr;
  DevBsr A;
  DArray<double> dinv64;
  DArray<float> dinv32;
  double rho = 0.0;
  double inv_theta = 0.0;
  std::vector<double> c1, c2;  // Chebyshev step coefficients k = 1..deg-1
  DevBsr P, R;
  // the same matrices prepared for the streamed kernels (those of at least
  // wn_amg_params.stream_min_mb in FP32; n_tiles == 0 otherwise)
  StreamMat As, Ps, Rs;
  LevelVecs<double> v64;
  LevelVecs<float> v32;
  // host row pointers of A (levels >= 1), P and R when the hierarchy was built on the device
  std::vector<int32_t> h_A_rp, h_P_rp, h_R_rp;
};

struct AmgHierarchy {
  HostHierarchy host;  // kept for export to tests / diagnostics
  std::vector<DevLevel> levels;
  int64_t n_coarse = 0;
  DArray<double> coarse_inv;
  DArray<double> cb64, cx64;  // coarsest rhs / solution (FP64 path)
  DArray<float> cb32, cx32;   // (FP32 path)
  int degree = 2;
  double setup_seconds = 0.0;
  bool device_built = false;  // levels made by amg_build_device (host.levels hold no matrices
  bool host_synced = false;   // until amg_sync_host copies them down)
  bool basis_changed = false;  // the 6-DOF levels were moved to the block-Jacobi basis on the
                               // device (amg_coarse_block_basis): host copies are stale too
  uint64_t id = 0;  // unique per setup (workspaces sized for a hierarchy compare it)
};

// PCG scalars shared between kernels (device)
struct PcgScalars {
  double rz[2];    // r.z of the last two iterations (parity-indexed)
  double bnorm2;   // ||b||^2
  double tol2;     // (rtol ||b||)^2
  double rr;       // ||r||^2 of the last check
  double alpha;
  int done;
  int iters;
  int status;
  int max_iter;
};

template <typename T>
struct PcgVecs {
  DArray<T> x, r, z, p0, p1, q;
  DArray<T> d0;  // D^-1 r / theta_0 of the fine level, written by the update for the next V-cycle
  int alloc(int64_t n) {
    WN_CHECK(d0.alloc(n));
    WN_CHECK(x.alloc(n));
    WN_CHECK(r.alloc(n));
    WN_CHECK(z.alloc(n));
    WN_CHECK(p0.alloc(n));
    WN_CHECK(p1.alloc(n));
    WN_CHECK(q.alloc(n));
    return 0;
  }
};

struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  int64_t key = -1;
  int64_t kernels = 0;  // kernels per replay
  uint64_t fine_epoch = 0;  // StreamMat::epoch of the fine matrix at capture
  ~GraphCache() {
    if (exec) cudaGraphExecDestroy(exec);
  }
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key = -1;
  }
};

struct SolverWork {
  int64_t n = 0;  // scalar DOFs
  static constexpr int kMaxParts = 148 * 16;
  // number of valid partials in partA / partB / partC: the grid of the kernel that last
  // wrote them (host-side bookkeeping, baked into captured graphs in launch order)
  int npA = 0, npB = 0, npC = 0;
  DArray<double> partA, partB, partC;
  DArray<PcgScalars> scal;   // [0] = FP64 / inner solve, [1] = outer refinement
  DArray<double> u64, ulo, r64;  // outer refinement: u = u64 + ulo (double-double), r = F - K u
  DArray<float> r32;
  DArray<double> dinv64;      // Jacobi (point) of the fine matrix
  DArray<float> dinv32;
  DArray<double> binv64;      // block-Jacobi: pseudo-inverses of the diagonal blocks (row-major per node)
  DArray<float> binv32;
  PcgVecs<double> p64;
  PcgVecs<float> p32;
  // the FP16 V-cycle (solve precision 3): set for the solve's duration; s = diag(K)^-1/2 of the
  // current matrix (FP64 for the FP16 pack, FP32 for the vectors) and q = 1 / s
  bool half = false;
  DArray<double> s64;
  DArray<float> s32, q32;
  // captured chunk graphs: [mode 0 fp64 / 1 mixed / 2 fp32 / 3 mixed with the FP16 V-cycle]
  //                        [preconditioner 0 none / 1 jacobi / 2 amg / 3 block jacobi]
  GraphCache graphs[4][4];
  int64_t launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t own = nullptr;  // used when the caller passes the legacy default stream
  // Launch accounting of the current solve.  bytes: algorithmic bytes (unique reads + writes)
  // of the kernels that did their work; the PCG iterations are counted from the device-side
  // iteration count, so kernels that returned early after convergence are not counted.
  double bytes = 0.0;
  double iter_core_bytes = 0.0, iter_prec_bytes = 0.0;  // one iteration: SpMV/update/check, M^-1
  // Profile mode (wn_solve_params.profile): graphs off, an event after every launch; each
  // launch's duration is the time between its event and the previous one
  struct Note {
    const char* kind;  // kernel class; with level >= 0 reported as "l<level>.<kind>"
    int level;
    double bytes;
    int iter;   // PCG iteration of the launch (-1: outside the iterations)
    bool prec;  // part of the iteration's preconditioner apply
    bool valid;
  };
  bool profile = false;
  int cur_iter = -1;
  bool cur_prec = false;
  std::vector<Note> notes;
  std::vector<cudaEvent_t> note_events;  // note_events[i]: after launch i; [0] is the start mark
  struct ProfileRow {
    std::string name;
    int64_t count = 0;
    double ms = 0.0, bytes = 0.0;
  };
  std::vector<ProfileRow> last_profile;  // aggregated per kernel class after a profiled solve
  ~SolverWork() {
    for (auto& a : graphs)
      for (auto& g : a) g.reset();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own) cudaStreamDestroy(own);
    for (cudaEvent_t e : note_events) cudaEventDestroy(e);
  }
};

}  // namespace wn
