// AMG V-cycle and PCG / mixed-precision iterative refinement on sm_100a.
//
// Reference template: the GPU-resident PCG of hip_amg_solve_pcg_device
// (wnfea/solver/native/hip_kernels.cpp:2384-2489) with its V-cycle
// (hip_amg_apply_pure_vcycle_device, :2080-2340), and the host PCG of
// solid_solver.py:197-308 / nonlinear_solver.py:51-156.  Here:
//   * every V-cycle stage is one fused warp-per-block-row kernel: Chebyshev step +
//     residual, restriction, prolongation, post-smoothing (the reference launches ~5
//     CSR kernels per level and round-trips the coarse solve through the host when it has
//     more than 128 unknowns);
//   * PCG dot products are FP64, two-stage and deterministic: each producing CTA writes
//     one partial, every consuming CTA reduces the partial array in the same fixed order
//     (no atomics, identical scalars in all CTAs); the p-update is fused into the SpMV
//     (p_j = z_j + beta p_j built on the fly);
//   * the iterations are captured once into a CUDA graph (a chunk of iterations whose
//     kernels return early once the device-side convergence flag is set); the host reads
//     the flag once per chunk instead of once per iteration (hip_kernels.cpp:2465-2476);
//   * precision modes: FP64 throughout; "mixed" = FP64 PCG (FP64 SpMV, x, r, q, dots; FP32
//     search directions p on the streamed fine level) with
//     an FP32 preconditioner (the V-cycle's values, vectors and accumulation in FP32, FP64
//     coarsest inverse); "fp32 IR" = FP32 PCG (FP32 SpMV) inside FP64 iterative refinement.
//     Every mode runs inside an FP64 refinement loop whose residual r = F - K u uses the FP64
//     matrix with compensated arithmetic.
#include <chrono>
#include <map>
#include <string>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "amg.h"
#include "amg_device.h"
#include "common.cuh"
#include "eft.cuh"
#include "kernels.h"
#include "solid.h"
#include "spmv.cuh"
#include "solver.h"

namespace wn {

// ---------------------------------------------------------------------------------------
// reductions shared by the PCG kernels
// ---------------------------------------------------------------------------------------
constexpr int kThreads = 256;
// Row kernels are register-limited: ask for 6 resident CTAs per SM (<= 42 registers).
constexpr int kMinBlocks = 6;

// all threads of the CTA get the fixed-order sum of part[0..n)
__device__ __forceinline__ double reduce_parts(const double* __restrict__ part, int n, double* sh) {
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) sh[0] = s;
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void write_part(double v, double* part, double* sh) {
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// ---------------------------------------------------------------------------------------
// functors building SpMV inputs on the fly
// ---------------------------------------------------------------------------------------
template <typename T>
struct XD0 {  // d0_j = dinv_j b_j / theta   (first Chebyshev step from a zero guess)
  const T* __restrict__ b;
  const T* __restrict__ dinv;
  T inv_theta;
  __device__ __forceinline__ T operator()(int64_t j) const { return dinv[j] * b[j] * inv_theta; }
};
template <typename T>
struct XD0U {  // the same with a unit diagonal (the FP16 V-cycle's equilibrated fine level)
  const T* __restrict__ b;
  T inv_theta;
  __device__ __forceinline__ T operator()(int64_t j) const { return b[j] * inv_theta; }
};
template <typename T>
struct XPNew {  // p_j = z_j + beta p_old_j
  const T* __restrict__ z;
  const T* __restrict__ p;
  T beta;
  __device__ __forceinline__ T operator()(int64_t j) const { return z[j] + beta * p[j]; }
};

// the fine level (3x3 blocks, the assembled matrix) is component-major; coarse levels are
// block-contiguous
template <int BS>
struct LayoutOf {
  static constexpr Layout value = (BS == 3) ? kSoA : kAoS;
};

// lanes per block row: 16 for the fine 3x3 level (rows of ~25 blocks: two rows per warp keep
// more loads in flight), a full warp for the 6x6 coarse levels
template <int BS>
struct GroupOf {
  static constexpr int value = (BS == 3) ? 16 : 32;
};

// Row loop for groups of G lanes: defines `lane` (index inside the group), `row` and needs
// `const bool active = row < n_rows;` in the body (all lanes stay in the loop for the
// group shuffles).
#define GROUP_ROW_LOOP(n_rows, G)                                                              \
  const int lane = (threadIdx.x & 31) % (G);                                                   \
  const int grp_ = (threadIdx.x & 31) / (G);                                                   \
  const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;                 \
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;                               \
  for (int64_t rb_ = warp0, row = warp0 * (32 / (G)) + grp_; rb_ * (32 / (G)) < (n_rows);      \
       rb_ += nwarps, row = rb_ * (32 / (G)) + grp_)

#define WARP_ROW_LOOP(n_rows)                                                   \
  const int lane = threadIdx.x & 31;                                            \
  const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;  \
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;                \
  for (int64_t row = warp0; row < (n_rows); row += nwarps)

template <int BS, typename T>
__device__ __forceinline__ T pick(const T (&acc)[BS], int lane) {
  T v = acc[0];
#pragma unroll
  for (int k = 1; k < BS; ++k)
    if (lane == k) v = acc[k];
  return v;
}

// ---------------------------------------------------------------------------------------
// V-cycle kernels (T = double or float, accumulation in T)
// ---------------------------------------------------------------------------------------

// First pre-smoothing step from x = 0.  deg == 1: x = d0, res = b - A x (fused residual).
// deg >= 2: second Chebyshev step: r1 = D^-1 (b - A d0), d1 = c1 d0 + c2 r1, x = d0 + d1.
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads, (BS == 3) ? kMinBlocks : 1) k_pre_first(int64_t n_rows, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const T* __restrict__ av, int64_t stride,
                                                        const T* __restrict__ b, const T* __restrict__ dinv,
                                                        T inv_theta, int deg, T c1, T c2, T* __restrict__ x,
                                                        T* __restrict__ r, T* __restrict__ d, T* __restrict__ res,
                                                        const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  if (S->done) return;
  GROUP_ROW_LOOP(n_rows, GroupOf<BS>::value) {
    const bool active = row < n_rows;
    T acc[BS];
    group_block_row<BS, BS, GroupOf<BS>::value, LayoutOf<BS>::value, T, T>(rp, ci, av, stride, row, active,
        XD0<T>{b, dinv, inv_theta}, acc, lane);
    if (active && lane < BS) {
      const int64_t i = row * BS + lane;
      const T t = pick<BS>(acc, lane);
      const T bi = b[i], di = dinv[i];
      const T d0 = di * bi * inv_theta;
      if (deg == 1) {
        x[i] = d0;
        res[i] = bi - t;
      } else {
        const T r1 = di * bi - di * t;
        const T d1 = c1 * d0 + c2 * r1;
        x[i] = d0 + d1;
        r[i] = r1;
        d[i] = d1;
      }
    }
  }
}

// Chebyshev step k >= 1: r -= D^-1 A d_in; d_out = c1 d_in + c2 r; x += d_out.
// If part != nullptr: also the partial of b . x (the PCG's r . z at the finest level).
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads, (BS == 3) ? kMinBlocks : 1) k_cheb_step(int64_t n_rows, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const T* __restrict__ av, int64_t stride,
                                                        const T* __restrict__ dinv, const T* __restrict__ d_in,
                                                        T* __restrict__ d_out, T* __restrict__ r, T* __restrict__ x,
                                                        T c1, T c2, const T* __restrict__ b, double* __restrict__ part,
                                                        const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double dot = 0.0;
  GROUP_ROW_LOOP(n_rows, GroupOf<BS>::value) {
    const bool active = row < n_rows;
    T acc[BS];
    group_block_row<BS, BS, GroupOf<BS>::value, LayoutOf<BS>::value, T, T>(rp, ci, av, stride, row, active,
        XLoad<T, T>{d_in}, acc, lane);
    if (active && lane < BS) {
      const int64_t i = row * BS + lane;
      const T ri = r[i] - dinv[i] * pick<BS>(acc, lane);
      const T dn = c1 * d_in[i] + c2 * ri;
      const T xn = x[i] + dn;
      r[i] = ri;
      d_out[i] = dn;
      x[i] = xn;
      if (part) dot += (double)b[i] * (double)xn;
    }
  }
  if (part) write_part(dot, part, sh);
}

// res = b - A x
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads, (BS == 3) ? kMinBlocks : 1) k_residual(int64_t n_rows, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci, const T* __restrict__ av, int64_t stride,
                                                       const T* __restrict__ b, const T* __restrict__ x,
                                                       T* __restrict__ res, const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  if (S->done) return;
  GROUP_ROW_LOOP(n_rows, GroupOf<BS>::value) {
    const bool active = row < n_rows;
    T acc[BS];
    group_block_row<BS, BS, GroupOf<BS>::value, LayoutOf<BS>::value, T, T>(rp, ci, av, stride, row, active,
        XLoad<T, T>{x}, acc, lane);
    if (active && lane < BS) {
      const int64_t i = row * BS + lane;
      res[i] = b[i] - pick<BS>(acc, lane);
    }
  }
}

// y = A x (accumulate = 0) or y += A x (accumulate = 1) for a BR x BC block-contiguous
// matrix, (A x)_i scaled by ys_i when ys is given; G lanes per block row (32 / G rows per
// warp) so that short rows (the prolongators) still fill the warp.
template <int BR, int BC, int G, typename T>
__global__ void __launch_bounds__(kThreads) k_level_spmv(int64_t n_rows, const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                         const T* __restrict__ x, T* __restrict__ y, int accumulate,
                                                         const PcgScalars* __restrict__ S,
                                                         const T* __restrict__ ys = nullptr) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  if (S->done) return;
  constexpr int RPW = 32 / G;
  const int lane = threadIdx.x & 31;
  const int gl = lane % G, grp = lane / G;
  const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t rb = warp0; rb * RPW < n_rows; rb += nwarps) {
    const int64_t row = rb * RPW + grp;
    const bool active = row < n_rows;
    T acc[BR];
    group_block_row<BR, BC, G, kAoS, T, T>(rp, ci, av, 0, row, active, XLoad<T, T>{x}, acc, gl);
    if (active && gl < BR) {
      const int64_t i = row * BR + gl;
      const T v = (ys ? ys[i] : T(1)) * pick<BR>(acc, gl);
      y[i] = accumulate ? y[i] + v : v;
    }
  }
}

// launch k_level_spmv with a group size matched to the mean row length
template <int BR, int BC, typename T>
static void level_spmv_rows(const DevBsr& M, const T* vals, const T* x, T* y, int accumulate, const PcgScalars* S,
                            cudaStream_t st, const T* ys = nullptr) {
  const double avg = M.n_rows ? (double)M.nnzb / (double)M.n_rows : 0.0;
  if (avg >= 24.0) {
    auto k = k_level_spmv<BR, BC, 32, T>;
    k<<<resident_grid(k, kThreads, (M.n_rows * 32 + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        M.n_rows, M.rp.p, M.ci.p, vals, x, y, accumulate, S, ys);
  } else if (avg >= 12.0) {
    auto k = k_level_spmv<BR, BC, 16, T>;
    k<<<resident_grid(k, kThreads, (M.n_rows * 16 + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        M.n_rows, M.rp.p, M.ci.p, vals, x, y, accumulate, S, ys);
  } else {
    auto k = k_level_spmv<BR, BC, 8, T>;
    k<<<resident_grid(k, kThreads, (M.n_rows * 8 + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        M.n_rows, M.rp.p, M.ci.p, vals, x, y, accumulate, S, ys);
  }
}

// First post-smoothing step from a nonzero x: r0 = D^-1 (b - A x), d0 = r0 / theta,
// x2 = x + d0 (x2 is a separate buffer: x is still read by neighbouring rows).
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads, (BS == 3) ? kMinBlocks : 1) k_post_first(int64_t n_rows, const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ ci, const T* __restrict__ av, int64_t stride,
                                                         const T* __restrict__ b, const T* __restrict__ dinv,
                                                         T inv_theta, const T* __restrict__ x, T* __restrict__ x2,
                                                         T* __restrict__ r, T* __restrict__ d, double* __restrict__ part,
                                                         const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double dot = 0.0;
  GROUP_ROW_LOOP(n_rows, GroupOf<BS>::value) {
    const bool active = row < n_rows;
    T acc[BS];
    group_block_row<BS, BS, GroupOf<BS>::value, LayoutOf<BS>::value, T, T>(rp, ci, av, stride, row, active,
        XLoad<T, T>{x}, acc, lane);
    if (active && lane < BS) {
      const int64_t i = row * BS + lane;
      const T r0 = dinv[i] * (b[i] - pick<BS>(acc, lane));
      const T d0 = r0 * inv_theta;
      const T xn = x[i] + d0;
      r[i] = r0;
      d[i] = d0;
      x2[i] = xn;
      if (part) dot += (double)b[i] * (double)xn;
    }
  }
  if (part) write_part(dot, part, sh);
}

// coarsest level: x = A_c^-1 b with the dense FP64 inverse.  Four warps per row (two rows per
// CTA), each lane with four independent partial sums over columns 128 apart, combined in a fixed
// order, so a 1,500-column row takes three dependent load rounds instead of ~47.
constexpr int kCoarseWarpsPerRow = 4;
template <typename T>
__global__ void __launch_bounds__(kThreads) k_coarse(int64_t n, const double* __restrict__ inv,
                                                     const T* __restrict__ b, T* __restrict__ x,
                                                     const PcgScalars* __restrict__ S) {
  __shared__ double part[kThreads / 32];
  if (S->done) return;
  constexpr int RPC = (kThreads / 32) / kCoarseWarpsPerRow;  // rows per CTA
  constexpr int STEP = 32 * kCoarseWarpsPerRow;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, q = w % kCoarseWarpsPerRow;
  for (int64_t row0 = (int64_t)blockIdx.x * RPC; row0 < n; row0 += (int64_t)gridDim.x * RPC) {
    const int64_t row = row0 + w / kCoarseWarpsPerRow;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    if (row < n) {
      const double* rowp = inv + row * n;
      int64_t j = q * 32 + lane;
      for (; j + 3 * STEP < n; j += 4 * STEP) {
        s0 += __ldg(rowp + j) * (double)b[j];
        s1 += __ldg(rowp + j + STEP) * (double)b[j + STEP];
        s2 += __ldg(rowp + j + 2 * STEP) * (double)b[j + 2 * STEP];
        s3 += __ldg(rowp + j + 3 * STEP) * (double)b[j + 3 * STEP];
      }
      for (; j < n; j += STEP) s0 += __ldg(rowp + j) * (double)b[j];
    }
    const double s = warp_sum((s0 + s1) + (s2 + s3));
    if (lane == 0) part[w] = s;
    __syncthreads();
    if (q == 0 && lane == 0 && row < n) x[row] = (T)((part[w] + part[w + 1]) + (part[w + 2] + part[w + 3]));
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// PCG kernels
// ---------------------------------------------------------------------------------------

// r = b, x = 0, rm = (TM) b (if rm != null; times rsc_i when rsc is given: the FP16 V-cycle's
// scaled input), partC = b . b (zero-RHS handling in k_init_scalars)
template <typename TK, typename TM>
__global__ void __launch_bounds__(kThreads) k_init_vecs(int64_t n, const TK* __restrict__ b, TK* __restrict__ x,
                                                        TK* __restrict__ r, TM* __restrict__ rm,
                                                        double* __restrict__ partC, const TM* __restrict__ rsc) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const TK v = b[i];
    r[i] = v;
    x[i] = TK(0);
    if (rm) rm[i] = rsc ? rsc[i] * (TM)v : (TM)v;
    s += (double)v * (double)v;
  }
  write_part(s, partC, sh);
}

// The equilibration of the FP16 V-cycle from the fine matrix's diagonal: s = diag(K)^-1/2
// (1 where the diagonal is not positive), q = 1 / s.
__global__ void k_fill_scale(int64_t n_rows, int64_t nnzb, const int32_t* __restrict__ diag_block,
                             const double* __restrict__ k64, double* __restrict__ s64, float* __restrict__ s32,
                             float* __restrict__ q32) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_rows * 3;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = t / 3;
    const int c = (int)(t - row * 3);
    const double dv = k64[(int64_t)(c * 4) * nnzb + diag_block[row]];
    const double q = dv > 0.0 ? sqrt(dv) : 1.0;
    s64[t] = 1.0 / q;
    s32[t] = (float)(1.0 / q);
    q32[t] = (float)q;
  }
}

__global__ void k_init_scalars(PcgScalars* S, const double* __restrict__ partC, int nparts, double rtol,
                               int max_iter) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  const double bb = reduce_parts(partC, nparts, sh);
  if (threadIdx.x == 0) {
    S->rz[0] = S->rz[1] = 0.0;
    S->bnorm2 = bb;
    S->tol2 = rtol * rtol * bb;
    S->rr = bb;
    S->alpha = 0.0;
    S->iters = 0;
    S->status = 0;
    S->max_iter = max_iter;
    S->done = (bb == 0.0 || !isfinite(bb)) ? 1 : 0;
    if (!isfinite(bb)) S->status = WN_EBREAKDOWN;
  }
}

// z = D^-1 r (jacobi = 1) or z = r (jacobi = 0); partA = r . z
template <typename T>
__global__ void __launch_bounds__(kThreads) k_prec_vec(int64_t n, const T* __restrict__ r, const T* __restrict__ dinv,
                                                       int jacobi, T* __restrict__ z, double* __restrict__ partA,
                                                       const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = r[i];
    const T zi = jacobi ? dinv[i] * ri : ri;
    z[i] = zi;
    s += (double)ri * (double)zi;
  }
  write_part(s, partA, sh);
}

// Block-Jacobi preconditioner (solid_solver.py:237-258): the pseudo-inverse of every BS x BS
// diagonal block, as the reference's numpy.linalg.pinv of the 3x3 node blocks.  The diagonal
// blocks of the assembled stiffness are symmetric (each entry and its transpose sum the same
// element contributions in the same order), so pinv = V diag(1 / lambda) V^T from a cyclic
// Jacobi eigen-decomposition (Golub & Van Loan, Matrix Computations, sec. 8.5), eigenvalues with
// |lambda| <= 1e-15 max |lambda| taken as zero (numpy's default cutoff relative to the largest
// singular value).  One thread per node in FP64; the FP32 copy serves the mixed modes.  Output
// row-major per node: b[(node * BS + i) * BS + j].
template <int BS>
__global__ void k_fill_block_pinv(int64_t n_nodes, int64_t nnzb, const int32_t* __restrict__ diag_block,
                                  const double* __restrict__ k64, double* __restrict__ b64,
                                  float* __restrict__ b32) {
  for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n_nodes;
       node += (int64_t)gridDim.x * blockDim.x) {
    const int64_t db = diag_block[node];
    double a[BS][BS], v[BS][BS];
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int j = 0; j < BS; ++j) {
        a[i][j] = (BS == 3) ? k64[(int64_t)(3 * i + j) * nnzb + db] : k64[db * BS * BS + i * BS + j];
        v[i][j] = (i == j) ? 1.0 : 0.0;
      }
    // fixed sweep count: the cyclic method converges quadratically; 12 sweeps reach the FP64
    // level for blocks of this size, rotations with a zero off-diagonal entry are skipped
    for (int sweep = 0; sweep < 12; ++sweep) {
#pragma unroll
      for (int p = 0; p < BS - 1; ++p)
#pragma unroll
        for (int q = p + 1; q < BS; ++q) {
          const double apq = a[p][q];
          if (apq == 0.0) continue;
          const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
          const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
          for (int k = 0; k < BS; ++k) {  // A <- A J (columns p, q)
            const double akp = a[k][p], akq = a[k][q];
            a[k][p] = c * akp - s * akq;
            a[k][q] = s * akp + c * akq;
          }
#pragma unroll
          for (int k = 0; k < BS; ++k) {  // A <- J^T A (rows p, q)
            const double apk = a[p][k], aqk = a[q][k];
            a[p][k] = c * apk - s * aqk;
            a[q][k] = s * apk + c * aqk;
          }
          a[p][q] = a[q][p] = 0.0;
#pragma unroll
          for (int k = 0; k < BS; ++k) {  // V <- V J
            const double vkp = v[k][p], vkq = v[k][q];
            v[k][p] = c * vkp - s * vkq;
            v[k][q] = s * vkp + c * vkq;
          }
        }
    }
    double lmax = 0.0;
#pragma unroll
    for (int i = 0; i < BS; ++i) lmax = fmax(lmax, fabs(a[i][i]));
    double inv[BS];
#pragma unroll
    for (int i = 0; i < BS; ++i) inv[i] = (fabs(a[i][i]) > 1e-15 * lmax) ? 1.0 / a[i][i] : 0.0;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int j = 0; j < BS; ++j) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < BS; ++k) s += v[i][k] * inv[k] * v[j][k];
        b64[(node * BS + i) * BS + j] = s;
        b32[(node * BS + i) * BS + j] = (float)s;
      }
  }
}

// z = B^-1 r per node with the block pseudo-inverses; partA = r . z
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) k_prec_block(int64_t n_nodes, const T* __restrict__ r,
                                                         const T* __restrict__ binv, T* __restrict__ z,
                                                         double* __restrict__ partA,
                                                         const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double s = 0.0;
  for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n_nodes;
       node += (int64_t)gridDim.x * blockDim.x) {
    T rv[BS];
#pragma unroll
    for (int j = 0; j < BS; ++j) rv[j] = r[node * BS + j];
    const T* b = binv + node * BS * BS;
#pragma unroll
    for (int i = 0; i < BS; ++i) {
      T zi = T(0);
#pragma unroll
      for (int j = 0; j < BS; ++j) zi += b[i * BS + j] * rv[j];
      z[node * BS + i] = zi;
      s += (double)rv[i] * (double)zi;
    }
  }
  write_part(s, partA, sh);
}

template <typename TK, typename TM>
struct XPNew2 {  // p_j = z_j + beta p_old_j, z in the preconditioner's precision
  const TM* __restrict__ z;
  const TK* __restrict__ p;
  TK beta;
  __device__ __forceinline__ TK operator()(int64_t j) const { return (TK)z[j] + beta * p[j]; }
};

// iteration k: rz = sum(partA); beta = rz / rz_prev (0 at k = 0); p_new = z + beta p_old;
// q = A p_new; partB = p_new . q.  Parity par = k & 1 selects the p buffers and rz slot.
// TK: Krylov vectors / matrix precision; TM: preconditioner output precision.
// The lane's own p_new entry is formed before the row product so that its loads overlap the
// matrix stream; the FP64 variant then needs up to 48 registers (5 resident CTAs per SM).
template <int BS, typename TK, typename TM>
__global__ void __launch_bounds__(kThreads, (BS == 3) ? (sizeof(TK) == 4 ? kMinBlocks : 5) : 1) k_spmv_dot(int64_t n_rows, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci, const TK* __restrict__ av, int64_t stride,
                                                       const TM* __restrict__ z, const TK* __restrict__ p_old,
                                                       TK* __restrict__ p_new, TK* __restrict__ q,
                                                       const double* __restrict__ partA, double* __restrict__ partB,
                                                       int nparts, int first, int par, PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  const double rz = reduce_parts(partA, nparts, sh);
  const double rz_prev = S->rz[par ^ 1];
  const TK beta = first ? TK(0) : (TK)(rz / rz_prev);
  double dot = 0.0;
  GROUP_ROW_LOOP(n_rows, GroupOf<BS>::value) {
    const bool active = row < n_rows;
    const bool own = active && lane < BS;
    const int64_t i = row * BS + lane;
    const TK pi = own ? (TK)z[i] + beta * p_old[i] : TK(0);
    TK acc[BS];
    group_block_row<BS, BS, GroupOf<BS>::value, LayoutOf<BS>::value, TK, TK>(rp, ci, av, stride, row, active,
        XPNew2<TK, TM>{z, p_old, beta}, acc, lane);
    if (own) {
      const TK qi = pick<BS>(acc, lane);
      p_new[i] = pi;
      q[i] = qi;
      dot += (double)pi * (double)qi;
    }
  }
  write_part(dot, partB, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0) S->rz[par] = rz;
}

// alpha = rz / (p . q); x += alpha p; r -= alpha q; rm = (TM) r (if rm != null); partC = r . r
template <typename TK, typename TM, typename TP = TK>
__global__ void __launch_bounds__(kThreads) k_update(int64_t n, TK* __restrict__ x, TK* __restrict__ r,
                                                     TM* __restrict__ rm, const TP* __restrict__ p,
                                                     const TK* __restrict__ q, const double* __restrict__ partB,
                                                     double* __restrict__ partC, int nparts, int par,
                                                     PcgScalars* __restrict__ S, TM* __restrict__ d0,
                                                     const TM* __restrict__ dinv, TM inv_theta,
                                                     const TM* __restrict__ rsc) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  const double gamma = reduce_parts(partB, nparts, sh);
  const double alpha = S->rz[par] / gamma;
  if (!(gamma > 0.0) || !isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->status = WN_EBREAKDOWN;
      S->done = 1;
    }
    return;
  }
  const TK a = (TK)alpha;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += a * (TK)p[i];
    const TK ri = r[i] - a * q[i];
    r[i] = ri;
    // rsc: the FP16 V-cycle's input is S r (and its first smoothing input S r / theta, dinv = S)
    if (rm) rm[i] = rsc ? rsc[i] * (TM)ri : (TM)ri;
    // the next V-cycle's first smoothing input (x_j = D^-1 b_j / theta with b = r in the
    // preconditioner's precision), so that its streamed kernel gathers one vector, not two
    if (d0) d0[i] = dinv[i] * (TM)ri * inv_theta;
    s += (double)ri * (double)ri;
  }
  write_part(s, partC, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0) S->alpha = alpha;
}

// convergence test after an iteration (one CTA); the iteration count lives on the device so
// that a captured chunk of iterations can be replayed any number of times
__global__ void k_check(PcgScalars* S, const double* __restrict__ partC, int nparts) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  const double rr = reduce_parts(partC, nparts, sh);
  if (threadIdx.x == 0) {
    const int it = S->iters + 1;
    S->rr = rr;
    S->iters = it;
    if (!isfinite(rr)) {
      S->status = WN_EBREAKDOWN;
      S->done = 1;
    } else if (rr <= S->tol2) {
      S->done = 1;
    } else if (it >= S->max_iter) {
      S->status = WN_ENOCONV;
      S->done = 1;
    }
  }
}

// S->rr = sum(partC) (one CTA)
__global__ void k_reduce_rr(PcgScalars* S, const double* __restrict__ partC, int nparts) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  const double rr = reduce_parts(partC, nparts, sh);
  if (threadIdx.x == 0) S->rr = rr;
}

// partials of a . b
template <typename T>
__global__ void __launch_bounds__(kThreads) k_dot_pair(int64_t n, const T* __restrict__ a, const T* __restrict__ b,
                                                       double* __restrict__ part, const PcgScalars* __restrict__ S) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  write_part(s, part, sh);
}

// partials of x . x
template <typename T>
__global__ void __launch_bounds__(kThreads) k_dot_self(int64_t n, const T* __restrict__ x, double* __restrict__ part) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  __shared__ double sh[kThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += (double)x[i] * (double)x[i];
  write_part(s, part, sh);
}

// ---------------------------------------------------------------------------------------
// mixed-precision refinement kernels (FP64)
// ---------------------------------------------------------------------------------------

// r64 = F - K64 (u + ulo) from compensated products and sums (Dot2), rounded to FP64 at the
// end; r32 = (float) r64; partC = r64 . r64.  A group of lanes per block row (16 for 3x3
// component-major blocks, 32 for 6x6 block-contiguous ones), each with a (sum, error) pair over
// its blocks, combined by a butterfly of TwoSums (the same order in every lane).
template <int BS>
__global__ void __launch_bounds__(kThreads) k_outer_residual_dd(int64_t n_rows, const int32_t* __restrict__ rp,
                                                                const int32_t* __restrict__ ci,
                                                                const double* __restrict__ av, int64_t stride,
                                                                const double* __restrict__ F,
                                                                const double* __restrict__ u,
                                                                const double* __restrict__ ulo,
                                                                double* __restrict__ r64, float* __restrict__ r32,
                                                                double* __restrict__ partC) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  constexpr int G = GroupOf<BS>::value;
  __shared__ double sh[kThreads / 32];
  double rr = 0.0;
  GROUP_ROW_LOOP(n_rows, G) {
    const bool active = row < n_rows;
    double s[BS], c[BS];
#pragma unroll
    for (int r = 0; r < BS; ++r) s[r] = c[r] = 0.0;
    if (active) {
      const int32_t q1 = __ldg(rp + row + 1);
      for (int32_t q = __ldg(rp + row) + lane; q < q1; q += G) {
        const int64_t col = __ldg(ci + q);
        double uh[BS], ul[BS];
#pragma unroll
        for (int k = 0; k < BS; ++k) {
          uh[k] = u[col * BS + k];
          ul[k] = ulo[col * BS + k];
        }
#pragma unroll
        for (int r = 0; r < BS; ++r)
#pragma unroll
          for (int k = 0; k < BS; ++k) {
            const double a = (LayoutOf<BS>::value == kSoA) ? __ldg(av + (int64_t)(r * BS + k) * stride + q)
                                                            : __ldg(av + (int64_t)q * BS * BS + r * BS + k);
            double p, ep, t, es;
            two_prod(a, uh[k], p, ep);
            two_sum(s[r], p, t, es);
            s[r] = t;
            c[r] += (ep + es) + a * ul[k];
          }
      }
    }
#pragma unroll
    for (int r = 0; r < BS; ++r)
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
        const double s2 = __shfl_xor_sync(0xffffffffu, s[r], o);
        const double c2 = __shfl_xor_sync(0xffffffffu, c[r], o);
        double t, e;
        two_sum(s[r], s2, t, e);
        s[r] = t;
        c[r] = (c[r] + c2) + e;
      }
    if (active && lane < BS) {
      const int64_t i = row * BS + lane;
      const double sv = pick<BS>(s, lane), cv = pick<BS>(c, lane);
      double t, e;
      two_sum(F[i], -sv, t, e);
      const double ri = t + (e - cv);
      r64[i] = ri;
      if (r32) r32[i] = (float)ri;
      rr += ri * ri;
    }
  }
  write_part(rr, partC, sh);
}

// (u, ulo) += dx as a double-double pair, renormalised so that u = fl(u + ulo)
template <typename T>
__global__ void k_accumulate(int64_t n, double* __restrict__ u, double* __restrict__ ulo, const T* __restrict__ dx) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s, e, h, g;
    two_sum(u[i], (double)dx[i], s, e);
    two_sum(s, __dadd_rn(ulo[i], e), h, g);
    u[i] = h;
    ulo[i] = g;
  }
}

// 1 / diag of the fine matrix: 3x3 component-major (stride nnzb) or 6x6 block-contiguous
__global__ void k_fill_dinv(int64_t n_rows, int bs, int64_t nnzb, const int32_t* __restrict__ diag_block,
                            const double* __restrict__ k64,
                            double* __restrict__ d64, float* __restrict__ d32) {
  pdl_trigger();  // dependents launched programmatically may start their prologue
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_rows * bs;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = t / bs;
    const int c = (int)(t - row * bs);
    const double dv = (bs == 3) ? k64[(int64_t)(c * 4) * nnzb + diag_block[row]]
                                : k64[(int64_t)diag_block[row] * 36 + c * 7];
    const double inv = (fabs(dv) > 1e-12) ? 1.0 / dv : 1.0;  // solid_solver.py:230
    d64[t] = inv;
    d32[t] = (float)inv;
  }
}

// ---------------------------------------------------------------------------------------
// streamed fine-level kernels: the arithmetic of k_pre_first / k_cheb_step / k_residual /
// k_post_first / k_spmv_dot on the 3x3 fine matrix, with the matrix streamed through shared
// memory by bulk async copies (stream.cuh).  Each epilogue loads the row's own operands
// before the row product (load) and writes its results after it (store).
// With SC (the FP16 V-cycle) the fine level runs on the equilibrated matrix S A S (unit
// diagonal: dinv is not read) with its vectors in the scaled space (x^ = S^-1 x, b^ = S b);
// the epilogues then map back where the fine level hands a vector on: the residual to the
// restriction (rs = S^-1), the V-cycle's output (os = S); a null scale pointer is 1.
// Without SC the scale pointers are not read.
// ---------------------------------------------------------------------------------------
template <bool SC, typename T>
__device__ __forceinline__ T scale_or_one(const T* __restrict__ s, int64_t i) {
  if constexpr (SC)
    return s ? s[i] : T(1);
  else
    return T(1);
}
template <bool SC, typename T>
__device__ __forceinline__ T diag_inv(const T* __restrict__ dinv, int64_t i) {
  if constexpr (SC)
    return T(1);
  else
    return dinv[i];
}

template <typename T, bool SC = false>
struct EpiPreFirst {
  const T* __restrict__ b;
  const T* __restrict__ dinv;
  T inv_theta;
  int deg;
  T c1, c2;
  T* __restrict__ x;
  T* __restrict__ r;
  T* __restrict__ d;
  T* __restrict__ res;
  const T* __restrict__ rs = nullptr;  // residual scale (deg 1)
  struct Pre {
    T bi, di, si;
  };
  __device__ __forceinline__ Pre load(int64_t i) const {
    return {b[i], diag_inv<SC>(dinv, i), scale_or_one<SC>(rs, i)};
  }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, T t) const {
    const T d0 = p.di * p.bi * inv_theta;
    if (deg == 1) {
      x[i] = d0;
      res[i] = SC ? p.si * (p.bi - t) : p.bi - t;
    } else {
      const T r1 = p.di * p.bi - p.di * t;
      const T d1 = c1 * d0 + c2 * r1;
      x[i] = d0 + d1;
      r[i] = r1;
      d[i] = d1;
    }
    return 0.0;
  }
};

template <typename T, bool SC = false>
struct EpiCheb {
  const T* __restrict__ dinv;
  const T* __restrict__ d_in;
  T* __restrict__ d_out;
  T* __restrict__ r;
  T* __restrict__ x;
  T c1, c2;
  const T* __restrict__ b;
  int want_dot;
  const T* __restrict__ os = nullptr;  // scale of the x written (the V-cycle's last step)
  struct Pre {
    T di, dd, ri, xi, bi, si;
  };
  // b_i (for the dot) is loaded with the other operands, before the row product
  __device__ __forceinline__ Pre load(int64_t i) const {
    return {diag_inv<SC>(dinv, i), d_in[i], r[i], x[i], want_dot ? b[i] : T(0), scale_or_one<SC>(os, i)};
  }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, T t) const {
    const T ri = p.ri - p.di * t;
    const T dn = c1 * p.dd + c2 * ri;
    const T xn = p.xi + dn;
    r[i] = ri;
    d_out[i] = dn;
    x[i] = SC ? p.si * xn : xn;
    return want_dot ? (double)p.bi * (double)xn : 0.0;  // b^ . x^ = b . x in the scaled space
  }
};

template <typename T, bool SC = false>
struct EpiResidual {
  const T* __restrict__ b;
  T* __restrict__ res;
  const T* __restrict__ rs = nullptr;  // residual scale
  struct Pre {
    T bi, si;
  };
  __device__ __forceinline__ Pre load(int64_t i) const { return {b[i], scale_or_one<SC>(rs, i)}; }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, T t) const {
    res[i] = SC ? p.si * (p.bi - t) : p.bi - t;
    return 0.0;
  }
};

template <typename T, bool SC = false>
struct EpiPostFirst {
  const T* __restrict__ b;
  const T* __restrict__ dinv;
  T inv_theta;
  const T* __restrict__ x;
  T* __restrict__ x2;
  T* __restrict__ r;
  T* __restrict__ d;
  int want_dot;
  const T* __restrict__ os = nullptr;  // scale of x2 (when this is the V-cycle's last step)
  struct Pre {
    T di, bi, xi, si;
  };
  __device__ __forceinline__ Pre load(int64_t i) const {
    return {diag_inv<SC>(dinv, i), b[i], x[i], scale_or_one<SC>(os, i)};
  }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, T t) const {
    const T r0 = p.di * (p.bi - t);
    const T d0 = r0 * inv_theta;
    const T xn = p.xi + d0;
    r[i] = r0;
    d[i] = d0;
    x2[i] = SC ? p.si * xn : xn;
    return want_dot ? (double)p.bi * (double)xn : 0.0;
  }
};

template <typename TK, typename TM>
struct EpiSpmvDot {
  const TM* __restrict__ z;
  const TK* __restrict__ p_old;
  TK beta;
  TK* __restrict__ p_new;
  TK* __restrict__ q;
  struct Pre {
    TK pi;
  };
  __device__ __forceinline__ Pre load(int64_t i) const { return {(TK)z[i] + beta * p_old[i]}; }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, TK t) const {
    p_new[i] = p.pi;
    q[i] = t;
    return (double)p.pi * (double)t;
  }
};

template <typename T, bool SC = false>
struct EpiLevel {  // y = A x (accumulate = 0) or y += A x (the transfer operators); SC: row scale ys
  T* __restrict__ y;
  int accumulate;
  const T* __restrict__ ys = nullptr;
  struct Pre {
    T yi, si;
  };
  __device__ __forceinline__ Pre load(int64_t i) const {
    return {accumulate ? y[i] : T(0), scale_or_one<SC>(ys, i)};
  }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, T t) const {
    const T v = SC ? p.si * t : t;
    y[i] = accumulate ? p.yi + v : v;
    return 0.0;
  }
};

// a matrix as the streamed kernels see it: the tile-major pack of one precision
struct StreamView {
  const PackTile* tiles;
  int n_tiles;
  const unsigned char* pack;
  StreamCtl ctl;
};

template <typename T>
static StreamView stream_view(const StreamMat& m) {
  if constexpr (std::is_same<T, __half>::value)
    return {m.d16.p, m.n_tiles, m.p16.p, m.ctl};
  else if constexpr (sizeof(T) == 4)
    return {m.d32.p, m.n_tiles, m.p32.p, m.ctl};
  else
    return {m.d64.p, m.n_tiles, m.p64.p, m.ctl};
}

// Launched with programmatic stream serialisation (launch_pdl): the first tiles of the matrix
// are in flight before the predecessor has finished.
template <typename T, int BR, int BC, typename XF, typename EPI, typename SHAPE = StreamDefault<T, BR, BC>>
__global__ void __launch_bounds__(kStreamThreads, (SHAPE::kCtasPerSm))
    k_stream_rows(StreamView m, XF xf, EPI epi, double* __restrict__ part, PcgScalars* __restrict__ S) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double sh[kStreamThreads / 32];
  pdl_trigger();
  bool skipped = false;
  const double dot = stream_rows_v<T, typename ShapeValue<SHAPE, T>::type, BR, BC, typename SHAPE::type>(
      m.tiles, m.n_tiles, m.pack, xf, epi, smem, &S->status, &S->done, m.ctl, &skipped);
  if (part && !skipped) write_part(dot, part, sh);
}

// rz = sum(partA) and beta = rz / rz_prev (0 on the first iteration), into shared memory
struct BetaHook {
  const double* partA;
  int nparts, first, par;
  const PcgScalars* S;
  double* sh;
  double* rz_beta;  // shared: [0] rz, [1] beta
  __device__ __forceinline__ void operator()() const {
    const double rz = reduce_parts(partA, nparts, sh);
    if (threadIdx.x == 0) {
      rz_beta[0] = rz;
      rz_beta[1] = first ? 0.0 : rz / S->rz[par ^ 1];
    }
    __syncthreads();
  }
};

// The streamed PCG product in two launches: k_pnew forms p_new = z + beta p_old once (beta from
// the partials of r . z, reduced by every CTA as BetaHook does; block 0 records rz for the next
// beta), then k_stream_spmv_dot_p gathers p_new like a plain SpMV -- one vector per gathered
// DOF instead of z and p_old, the same values.
template <typename TK, typename TM, typename TP = TK>
__global__ void __launch_bounds__(kThreads) k_pnew(int64_t n, const TM* __restrict__ z, const TP* __restrict__ p_old,
                                                   TP* __restrict__ p_new, const double* __restrict__ partA,
                                                   int nparts, int first, int par, PcgScalars* __restrict__ S) {
  __shared__ double sh[kThreads / 32];
  __shared__ double rz_beta[2];
  pdl_trigger();
  pdl_wait();
  if (*(volatile int*)&S->done) return;
  BetaHook{partA, nparts, first, par, S, sh, rz_beta}();
  const double* beta = rz_beta + 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p_new[i] = (TP)((TK)z[i] + (TK)*beta * (TK)p_old[i]);
  if (blockIdx.x == 0 && threadIdx.x == 0) S->rz[par] = rz_beta[0];
}

template <typename TK, typename TP = TK>
struct EpiSpmvDotP {  // q = A p_new; dot: p_new . q (p_new already written)
  const TP* __restrict__ p_new;
  TK* __restrict__ q;
  struct Pre {
    TK pi;
  };
  __device__ __forceinline__ Pre load(int64_t i) const { return {(TK)p_new[i]}; }
  __device__ __forceinline__ double store(int64_t i, const Pre& p, TK t) const {
    q[i] = t;
    return (double)p.pi * (double)t;
  }
};

template <int BS, typename TK, typename TP = TK>
__global__ void __launch_bounds__(kStreamThreads, (StreamDefault<TK, BS, BS>::kCtasPerSm))
    k_stream_spmv_dot_p(StreamView m, const TP* __restrict__ p_new, TK* __restrict__ q, double* __restrict__ partB,
                        PcgScalars* __restrict__ S) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double sh[kStreamThreads / 32];
  pdl_trigger();
  bool skipped = false;
  const double dot = stream_rows<TK, BS, BS, typename StreamDefault<TK, BS, BS>::type>(
      m.tiles, m.n_tiles, m.pack, XLoad<TP, TK>{p_new}, EpiSpmvDotP<TK, TP>{p_new, q}, smem, &S->status, &S->done,
      m.ctl, &skipped);
  if (skipped) return;
  write_part(dot, partB, sh);
}

// launch with programmatic stream serialisation: the kernel may begin (and start streaming its
// matrix) while its predecessor on the stream finishes; it waits (griddepcontrol) before
// reading anything the predecessor wrote
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), int grid, int threads, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// grid of a streamed kernel of shape CFG (one persistent wave), 0 if it cannot run on this device
template <typename T, int BR, int BC, typename CFG = typename StreamDefault<T, BR, BC>::type, typename K>
static int stream_grid(K kern, int n_tiles) {
  const int per_sm =
      stream_ctas_per_sm(reinterpret_cast<const void*>(kern), kStreamThreads, stream_smem_bytes<T, BR, BC, CFG>());
  if (per_sm < 1) return 0;
  return std::max(1, std::min(n_tiles, kNumSMs * per_sm));
}

// launch a streamed row kernel on matrix m (BR x BC blocks); false (nothing launched) when m
// has no current pack of that shape or the kernel cannot be configured.  A shape with FP16
// values streams the FP16 pack (its currency is the caller's to check).
template <typename T, int BR, int BC, typename XF, typename EPI, typename SHAPE = StreamDefault<T, BR, BC>>
static bool launch_stream_rows(const StreamMat& m, XF xf, EPI epi, double* part, PcgScalars* S, cudaStream_t st,
                               int* grid_out) {
  using TV = typename ShapeValue<SHAPE, T>::type;
  constexpr bool kHalf = std::is_same<TV, __half>::value;
  if (m.br != BR || m.bc != BC || (kHalf ? !m.p16.p : !m.packed)) return false;
  using CFG = typename SHAPE::type;
  auto kern = k_stream_rows<T, BR, BC, XF, EPI, SHAPE>;
  const int g = stream_grid<TV, BR, BC, CFG>(kern, m.n_tiles);
  if (g == 0) return false;
  if (launch_pdl(kern, g, kStreamThreads, stream_smem_bytes<TV, BR, BC, CFG>(), st, stream_view<TV>(m), xf, epi, part,
                 S) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (grid_out) *grid_out = g;
  return true;
}

// y = M x or y += M x for a transfer operator: streamed from its pack when it has one, else the
// register row kernel
// (SC: (M x)_i scaled by ys_i -- the FP16 V-cycle's prolongation into its scaled fine level)
template <int BR, int BC, typename T, bool SC = false>
static void level_spmv(const DevBsr& M, const StreamMat& Ms, const T* vals, const T* x, T* y, int accumulate,
                       PcgScalars* S, cudaStream_t st, const T* ys = nullptr) {
  if constexpr (BR == 6 && BC == 6) {  // short rows (the prolongations): 8 lanes per row
    if (M.nnzb < 16 * M.n_rows) {
      if (launch_stream_rows<T, 6, 6, XLoad<T, T>, EpiLevel<T, SC>, StreamShort66<T>>(
              Ms, XLoad<T, T>{x}, EpiLevel<T, SC>{y, accumulate, ys}, nullptr, S, st, nullptr))
        return;
      level_spmv_rows<BR, BC, T>(M, vals, x, y, accumulate, S, st, SC ? ys : nullptr);
      return;
    }
  }
  if (launch_stream_rows<T, BR, BC>(Ms, XLoad<T, T>{x}, EpiLevel<T, SC>{y, accumulate, ys}, nullptr, S, st, nullptr))
    return;
  level_spmv_rows<BR, BC, T>(M, vals, x, y, accumulate, S, st, SC ? ys : nullptr);
}

// ---------------------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------------------
static inline int rows_grid(int64_t n_rows) { return grid_for(n_rows, 32, kThreads, 8); }
static inline int vec_grid(int64_t n) { return grid_for(n, 1, kThreads, 8); }

// ---------------------------------------------------------------------------------------
// launch accounting: algorithmic bytes per launch (unique reads + writes of the kernel's
// arrays) and, in profile mode, an event after the launch
// ---------------------------------------------------------------------------------------
// one pass over a block matrix: values, column indices, row pointers
static double mat_bytes(int64_t nnzb, int br, int bc, int64_t n_rows, int value_bytes) {
  return (double)nnzb * (br * bc * value_bytes + 4) + 4.0 * (double)(n_rows + 1);
}

static void note(SolverWork& W, cudaStream_t st, const char* kind, int level, double bytes) {
  W.bytes += bytes;
  if (!W.profile) return;
  const size_t i = W.notes.size();
  while (W.note_events.size() < i + 2) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    W.note_events.push_back(e);
  }
  cudaEventRecord(W.note_events[i + 1], st);
  W.notes.push_back({kind, level, bytes, W.cur_iter, W.cur_prec, true});
}

template <typename T>
struct Prec;
template <>
struct Prec<double> {
  static const double* A0(Solid* s) { return s->k64.p; }
  static const double* Av(DevLevel& L) { return L.A.v64.p; }
  static const double* Pv(DevLevel& L) { return L.P.v64.p; }
  static const double* Rv(DevLevel& L) { return L.R.v64.p; }
  static const double* dinv(DevLevel& L) { return L.dinv64.p; }
  static LevelVecs<double>& vecs(DevLevel& L) { return L.v64; }
  static double* cb(AmgHierarchy& h) { return h.cb64.p; }
  static double* cx(AmgHierarchy& h) { return h.cx64.p; }
  static PcgVecs<double>& pcg(SolverWork& w) { return w.p64; }
  static const double* fine_dinv(SolverWork& w) { return w.dinv64.p; }
  static const double* fine_binv(SolverWork& w) { return w.binv64.p; }
};
template <>
struct Prec<float> {
  static const float* A0(Solid* s) { return s->k32.p; }
  static const float* Av(DevLevel& L) { return L.A.v32.p; }
  static const float* Pv(DevLevel& L) { return L.P.v32.p; }
  static const float* Rv(DevLevel& L) { return L.R.v32.p; }
  static const float* dinv(DevLevel& L) { return L.dinv32.p; }
  static LevelVecs<float>& vecs(DevLevel& L) { return L.v32; }
  static float* cb(AmgHierarchy& h) { return h.cb32.p; }
  static float* cx(AmgHierarchy& h) { return h.cx32.p; }
  static PcgVecs<float>& pcg(SolverWork& w) { return w.p32; }
  static const float* fine_dinv(SolverWork& w) { return w.dinv32.p; }
  static const float* fine_binv(SolverWork& w) { return w.binv32.p; }
};

template <int BS, typename T>
static void level_A(Solid* s, DevLevel& L, int lvl, const int32_t*& rp, const int32_t*& ci, const T*& av) {
  if (lvl == 0) {
    rp = s->row_ptr.p;
    ci = s->col_idx.p;
    av = Prec<T>::A0(s);
  } else {
    rp = L.A.rp.p;
    ci = L.A.ci.p;
    av = Prec<T>::Av(L);
  }
}

// One V-cycle at level lvl: x_out = V(b).  At level 0, b / out are the PCG's r / z and
// part (if not null) receives the partials of b . out.
template <typename T>
static int vcycle(Solid* s, AmgHierarchy& H, SolverWork& W, int lvl, const T* b, T* out, double* part,
                  PcgScalars* S, cudaStream_t st, const T* d0 = nullptr) {
  const int nlev = (int)H.levels.size();
  if (lvl == nlev) {  // coarsest
    constexpr int rows_per_cta = (kThreads / 32) / kCoarseWarpsPerRow;
    k_coarse<T><<<resident_grid(k_coarse<T>, kThreads, (H.n_coarse + rows_per_cta - 1) / rows_per_cta), kThreads, 0,
                  st>>>(H.n_coarse, H.coarse_inv.p, b, out, S);
    W.launches++;
    note(W, st, "coarse", -1, (double)H.n_coarse * H.n_coarse * 8 + 2.0 * H.n_coarse * sizeof(T));
    if (part) {  // a hierarchy without levels: the PCG's r . z comes from here
      const int g = resident_grid(k_dot_pair<T>, kThreads, (H.n_coarse + kThreads - 1) / kThreads);
      W.npA = g;
      k_dot_pair<T><<<g, kThreads, 0, st>>>(H.n_coarse, b, out, part, S);
      W.launches++;
      note(W, st, "dot", -1, 2.0 * H.n_coarse * sizeof(T));
    }
    WN_CUDA(cudaGetLastError());
    return 0;
  }
  DevLevel& L = H.levels[lvl];
  LevelVecs<T>& V = Prec<T>::vecs(L);
  const int64_t nr = L.n_nodes;
  // the FP16 V-cycle (W.half): level 0 streams the equilibrated matrix S A S from its FP16 pack
  // with the level's vectors in the scaled space (unit diagonal, no dinv); qs = S^-1 maps the
  // residual and the prolongated correction, os = S the output
  const bool half0 = lvl == 0 && W.half;
  const T* qs = nullptr;
  const T* os = nullptr;
  if constexpr (std::is_same<T, float>::value) {
    if (half0) {
      qs = W.q32.p;
      os = W.s32.p;
    }
  }
  // level 0: 1/diag of the current matrix (refreshed per solve), so a hierarchy kept across
  // re-assemblies still smooths with the right diagonal
  const T* dinv = half0 ? nullptr : (lvl == 0) ? Prec<T>::fine_dinv(W) : Prec<T>::dinv(L);
  const int deg = H.degree;
  const T it = (T)L.inv_theta;
  const int64_t sd = (lvl == 0) ? s->nnzb : 0;  // component stride of the fine matrix
  const int64_t work = (nr * 32 + kThreads - 1) / kThreads;
  // algorithmic bytes: the level matrix, one level vector, the transfer operators
  const double Vb = (double)nr * L.bs * sizeof(T);
  const double Ab = half0 ? mat_bytes(s->nnzb, 3, 3, nr, 2)
                          : mat_bytes(lvl == 0 ? s->nnzb : L.A.nnzb, L.bs, L.bs, nr, sizeof(T));
  const int64_t nc_dofs = (lvl + 1 < nlev) ? H.levels[lvl + 1].n_nodes * H.levels[lvl + 1].bs : H.n_coarse;
  const double Vc = (double)nc_dofs * sizeof(T);
  const double Rb = mat_bytes(L.R.nnzb, L.R.br, L.R.bc, L.R.n_rows, sizeof(T));
  const double Pb = mat_bytes(L.P.nnzb, L.P.br, L.P.bc, L.P.n_rows, sizeof(T));
  auto run = [&](auto bs_tag, auto sc_tag) -> int {
    constexpr int BS = decltype(bs_tag)::value;
    constexpr bool SC = decltype(sc_tag)::value;  // the FP16 V-cycle's level 0 (3x3, FP32 only)
    static_assert(!SC || (BS == 3 && std::is_same<T, float>::value), "FP16 level: 3x3 blocks, FP32 arithmetic");
    auto rg = [&](auto kern) { return resident_grid(kern, kThreads, work); };
    const int32_t* rp;
    const int32_t* ci;
    const T* av;
    level_A<BS, T>(s, L, lvl, rp, ci, av);
    // pre-smoothing (+ residual).  A level whose matrix has a current tile-major pack (the fine
    // level; coarse levels too large for L2) streams it through shared memory (stream.cuh);
    // the others use the register row kernels.  The FP16 level 0 has no register form: a
    // launch that fails there is an error.
    const StreamMat& Am = (lvl == 0) ? s->fine : L.As;
    const bool stream = Am.packed;
    bool half_failed = false;
    auto rows = [&](auto xf, auto epi, double* prt, int* gout) -> bool {
      if constexpr (SC) {
        const bool ok = launch_stream_rows<T, 3, 3, decltype(xf), decltype(epi), StreamHalf33>(Am, xf, epi, prt, S,
                                                                                               st, gout);
        half_failed = half_failed || !ok;
        return true;
      } else {
        return stream && launch_stream_rows<T, BS, BS>(Am, xf, epi, prt, S, st, gout);
      }
    };
    const T c1 = deg >= 2 ? (T)L.c1[0] : T(0), c2 = deg >= 2 ? (T)L.c2[0] : T(0);
    // d0 (level 0, from the PCG update): the first step's input D^-1 b / theta precomputed
    EpiPreFirst<T, SC> epi_pre{b, dinv, it, deg, c1, c2, V.x.p, V.r.p, V.d.p, V.res.p};
    epi_pre.rs = qs;
    bool pre_streamed;
    if (d0)
      pre_streamed = rows(XLoad<T, T>{d0}, epi_pre, nullptr, nullptr);
    else if constexpr (SC)
      pre_streamed = rows(XD0U<T>{b, it}, epi_pre, nullptr, nullptr);
    else
      pre_streamed = rows(XD0<T>{b, dinv, it}, epi_pre, nullptr, nullptr);
    if (!pre_streamed)
      k_pre_first<BS, T><<<rg(k_pre_first<BS, T>), kThreads, 0, st>>>(nr, rp, ci, av, sd, b, dinv, it, deg, c1, c2,
                                                                      V.x.p, V.r.p, V.d.p, V.res.p, S);
    W.launches++;
    note(W, st, "pre_smooth", lvl, Ab + (deg == 1 ? 4 : 5) * Vb);
    T* din = V.d.p;
    T* dout = V.d2.p;
    for (int k = 2; k < deg; ++k) {
      const T ck1 = (T)L.c1[k - 1], ck2 = (T)L.c2[k - 1];
      if (!rows(XLoad<T, T>{din}, EpiCheb<T, SC>{dinv, din, dout, V.r.p, V.x.p, ck1, ck2, b, 0}, nullptr, nullptr))
        k_cheb_step<BS, T><<<rg(k_cheb_step<BS, T>), kThreads, 0, st>>>(nr, rp, ci, av, sd, dinv, din, dout, V.r.p,
                                                                        V.x.p, ck1, ck2, b, nullptr, S);
      W.launches++;
      note(W, st, "pre_cheb", lvl, Ab + 7 * Vb);
      std::swap(din, dout);
    }
    if (deg >= 2) {
      EpiResidual<T, SC> epi_res{b, V.res.p};
      epi_res.rs = qs;
      if (!rows(XLoad<T, T>{V.x.p}, epi_res, nullptr, nullptr))
        k_residual<BS, T><<<rg(k_residual<BS, T>), kThreads, 0, st>>>(nr, rp, ci, av, sd, b, V.x.p, V.res.p, S);
      W.launches++;
      note(W, st, "residual", lvl, Ab + 3 * Vb);
    }
    // restriction b_c = R res
    DevLevel* Ln = lvl + 1 < nlev ? &H.levels[lvl + 1] : nullptr;
    T* bc = Ln ? Prec<T>::vecs(*Ln).b.p : Prec<T>::cb(H);
    T* xc = Ln ? Prec<T>::vecs(*Ln).x2.p : Prec<T>::cx(H);
    level_spmv<6, BS, T>(L.R, L.Rs, Prec<T>::Rv(L), V.res.p, bc, 0, S, st);
    W.launches++;
    note(W, st, "restrict", lvl, Rb + Vb + Vc);
    WN_CHECK(vcycle<T>(s, H, W, lvl + 1, bc, xc, nullptr, S, st));
    // prolongation x += P x_c (x^ += S^-1 P x_c in the scaled space)
    level_spmv<BS, 6, T, SC>(L.P, L.Ps, Prec<T>::Pv(L), xc, V.x.p, 1, S, st, qs);
    W.launches++;
    note(W, st, "prolong", lvl, Pb + Vc + 2 * Vb);
    // post-smoothing: result in `out`
    double* part_last = (deg == 1) ? part : nullptr;
    int gpf = 0;
    EpiPostFirst<T, SC> epi_post{b, dinv, it, V.x.p, out, V.r.p, V.d.p, part_last != nullptr};
    epi_post.os = deg == 1 ? os : nullptr;
    if (!rows(XLoad<T, T>{V.x.p}, epi_post, part_last, &gpf)) {
      gpf = rg(k_post_first<BS, T>);
      k_post_first<BS, T><<<gpf, kThreads, 0, st>>>(nr, rp, ci, av, sd, b, dinv, it, V.x.p, out, V.r.p, V.d.p,
                                                     part_last, S);
    }
    if (part_last) W.npA = gpf;
    W.launches++;
    note(W, st, "post_smooth", lvl, Ab + 6 * Vb);
    din = V.d.p;
    dout = V.d2.p;
    for (int k = 1; k < deg; ++k) {
      double* pk = (k == deg - 1) ? part : nullptr;
      const T ck1 = (T)L.c1[k - 1], ck2 = (T)L.c2[k - 1];
      int gcs = 0;
      EpiCheb<T, SC> epi_cheb{dinv, din, dout, V.r.p, out, ck1, ck2, b, pk != nullptr};
      epi_cheb.os = (k == deg - 1) ? os : nullptr;
      if (!rows(XLoad<T, T>{din}, epi_cheb, pk, &gcs)) {
        gcs = rg(k_cheb_step<BS, T>);
        k_cheb_step<BS, T><<<gcs, kThreads, 0, st>>>(nr, rp, ci, av, sd, dinv, din, dout, V.r.p, out, ck1, ck2, b, pk,
                                                     S);
      }
      if (pk) W.npA = gcs;
      W.launches++;
      note(W, st, "post_cheb", lvl, Ab + (pk ? 8 : 7) * Vb);
      std::swap(din, dout);
    }
    WN_REQUIRE(!half_failed, WN_ESTATE, "FP16 V-cycle: the streamed fine-level kernel could not be launched");
    return 0;
  };
  int rc;
  if (half0) {
    if constexpr (std::is_same<T, float>::value)
      rc = run(std::integral_constant<int, 3>{}, std::true_type{});
    else
      rc = WN_ESTATE;
  } else if (L.bs == 3) {
    rc = run(std::integral_constant<int, 3>{}, std::false_type{});
  } else {
    rc = run(std::integral_constant<int, 6>{}, std::false_type{});
  }
  WN_CHECK(rc);
  WN_CUDA(cudaGetLastError());
  return 0;
}

// z = M r with partials of r . z into partA
template <typename T>
static int apply_prec(Solid* s, SolverWork& W, int precond, const T* r, T* z, PcgScalars* S, cudaStream_t st,
                      const T* d0 = nullptr) {
  if (precond == 2) return vcycle<T>(s, *s->amg, W, 0, r, z, W.partA.p, S, st, d0);
  if (precond == 3) {
    auto launch = [&](auto kern) {
      const int g = resident_grid(kern, kThreads, (s->n_nodes + kThreads - 1) / kThreads);
      W.npA = g;
      kern<<<g, kThreads, 0, st>>>(s->n_nodes, r, Prec<T>::fine_binv(W), z, W.partA.p, S);
    };
    if (s->bs == 3)
      launch(k_prec_block<3, T>);
    else
      launch(k_prec_block<6, T>);
    W.launches++;
    note(W, st, "block_jacobi", -1, (2.0 + s->bs) * W.n * sizeof(T));
    WN_CUDA(cudaGetLastError());
    return 0;
  }
  const int gp = resident_grid(k_prec_vec<T>, kThreads, (W.n + kThreads - 1) / kThreads);
  W.npA = gp;
  k_prec_vec<T><<<gp, kThreads, 0, st>>>(W.n, r, Prec<T>::fine_dinv(W), precond == 1 ? 1 : 0, z,
                                                         W.partA.p, S);
  W.launches++;
  note(W, st, precond == 1 ? "jacobi" : "copy", -1, (precond == 1 ? 3.0 : 2.0) * W.n * sizeof(T));
  WN_CUDA(cudaGetLastError());
  return 0;
}

// the FP16 V-cycle's input scale S (null otherwise)
template <typename TM>
static const TM* half_scale(const SolverWork& W) {
  if constexpr (std::is_same<TM, float>::value)
    return W.half ? W.s32.p : nullptr;
  else
    return nullptr;
}

// PCG buffers of one precision pairing: Krylov vectors / matrix in TK, preconditioner in TM
template <typename TK, typename TM>
struct PcgBufs {
  TK *x, *r, *p0, *p1, *q;
  TM *z, *rm;  // rm: r in TM for the preconditioner (nullptr when TK == TM: r is used)
  const TK* A;
};

template <typename TK, typename TM>
static PcgBufs<TK, TM> pcg_bufs(Solid* s, SolverWork& W);
template <>
PcgBufs<double, double> pcg_bufs(Solid* s, SolverWork& W) {
  return {W.p64.x.p, W.p64.r.p, W.p64.p0.p, W.p64.p1.p, W.p64.q.p, W.p64.z.p, nullptr, s->k64.p};
}
template <>
PcgBufs<double, float> pcg_bufs(Solid* s, SolverWork& W) {
  return {W.p64.x.p, W.p64.r.p, W.p64.p0.p, W.p64.p1.p, W.p64.q.p, W.p32.z.p, W.p32.r.p, s->k64.p};
}
template <>
PcgBufs<float, float> pcg_bufs(Solid* s, SolverWork& W) {
  return {W.p32.x.p, W.p32.r.p, W.p32.p0.p, W.p32.p1.p, W.p32.q.p, W.p32.z.p, nullptr, s->k32.p};
}

template <typename TK, typename TM>
static const TM* prec_input(const PcgBufs<TK, TM>& B) {
  if constexpr (std::is_same<TK, TM>::value)
    return B.r;
  else
    return B.rm;
}

// one PCG iteration k (parity k & 1)
template <typename TK, typename TM>
static int pcg_iteration(Solid* s, SolverWork& W, int precond, int k, PcgScalars* S, cudaStream_t st) {
  PcgBufs<TK, TM> B = pcg_bufs<TK, TM>(s, W);
  const int par = k & 1;
  TK* p_new = par ? B.p1 : B.p0;
  TK* p_old = par ? B.p0 : B.p1;
  const int gup = resident_grid(k_update<TK, TM>, kThreads, (W.n + kThreads - 1) / kThreads);
  // The mixed modes on the streamed fine level keep the search directions in FP32: p = z + beta p
  // is formed in FP64 and rounded once, and the product and the update read that same rounded p,
  // so q = A p and r = b - A x stay consistent in FP64; the gathers and the vector passes move
  // half the bytes.  (FP64 everywhere else: the matrix, q, x, r and the dots.)
  constexpr bool kMixed = std::is_same<TK, double>::value && std::is_same<TM, float>::value;
  using TPf = typename std::conditional<kMixed, float, TK>::type;
  bool p32 = false;
  auto spmv_dot = [&](auto bs_tag) {
    constexpr int BS = decltype(bs_tag)::value;
    if (s->fine.packed && s->fine.br == BS) {  // the fine matrix streamed through shared memory
      auto kern = k_stream_spmv_dot_p<BS, TK, TPf>;
      const int g = stream_grid<TK, BS, BS>(kern, s->fine.n_tiles);
      const int gp = resident_grid(k_pnew<TK, TM, TPf>, kThreads, (W.n + kThreads - 1) / kThreads);
      if (g > 0) {
        p32 = kMixed;
        TPf* pn = reinterpret_cast<TPf*>(p_new);
        cudaError_t e = launch_pdl(k_pnew<TK, TM, TPf>, gp, kThreads, 0, st, W.n, (const TM*)B.z,
                                   (const TPf*)reinterpret_cast<TPf*>(p_old), pn, (const double*)W.partA.p, W.npA,
                                   (int)(k == 0), par, S);
        if (e == cudaSuccess) {
          note(W, st, "pcg_pnew", -1, (double)W.n * (sizeof(TM) + 2 * sizeof(TPf)));
          W.launches++;
          e = launch_pdl(kern, g, kStreamThreads, stream_smem_bytes<TK, BS, BS>(), st, stream_view<TK>(s->fine),
                         (const TPf*)pn, B.q, W.partB.p, S);
          if (e == cudaSuccess) return -g;  // negative: the product's bytes are those of a plain SpMV
        }
        return 0;  // a failed launch: reported by the error check below
      }
    }
    const int g = resident_grid(k_spmv_dot<BS, TK, TM>, kThreads, (s->n_nodes * 32 + kThreads - 1) / kThreads);
    k_spmv_dot<BS, TK, TM><<<g, kThreads, 0, st>>>(s->n_nodes, s->row_ptr.p, s->col_idx.p, B.A, s->nnzb, B.z, p_old,
                                                   p_new, B.q, W.partA.p, W.partB.p, W.npA, k == 0, par, S);
    return g;
  };
  const double b_start = W.bytes;
  int gsd = s->bs == 3 ? spmv_dot(std::integral_constant<int, 3>{}) : spmv_dot(std::integral_constant<int, 6>{});
  const double nK = (double)W.n * sizeof(TK), nM = (double)W.n * sizeof(TM);
  // the fused product reads z and p_old and writes p_new and q; the split one reads p_new and
  // writes q (k_pnew counted its own bytes)
  note(W, st, "pcg_spmv_dot", -1,
       mat_bytes(s->nnzb, s->bs, s->bs, s->n_nodes, sizeof(TK)) +
           (gsd < 0 ? (p32 ? nM + nK : 2 * nK) : nM + 3 * nK));
  gsd = gsd < 0 ? -gsd : gsd;
  WN_CUDA(cudaGetLastError());
  WN_REQUIRE(gsd > 0, WN_ESTATE, "PCG product: launch failed");
  W.npB = gsd;
  // with the AMG preconditioner, the update also writes the fine level's first smoothing input
  const bool pre_input = precond == 2 && !s->amg->levels.empty();
  TM* d0 = pre_input ? Prec<TM>::pcg(W).d0.p : nullptr;
  const TM it0 = pre_input ? (TM)s->amg->levels[0].inv_theta : TM(0);
  if (p32)
    k_update<TK, TM, TPf><<<gup, kThreads, 0, st>>>(W.n, B.x, B.r, B.rm, reinterpret_cast<const TPf*>(p_new), B.q,
                                                    W.partB.p, W.partC.p, W.npB, par, S, d0,
                                                    W.half ? half_scale<TM>(W) : Prec<TM>::fine_dinv(W), it0,
                                                    half_scale<TM>(W));
  else
    k_update<TK, TM><<<gup, kThreads, 0, st>>>(W.n, B.x, B.r, B.rm, p_new, B.q, W.partB.p, W.partC.p, W.npB, par, S,
                                               d0, W.half ? half_scale<TM>(W) : Prec<TM>::fine_dinv(W), it0,
                                               half_scale<TM>(W));
  note(W, st, "pcg_update", -1, (p32 ? 5 * nK + nM : 6 * nK) + (B.rm ? nM : 0.0) + (d0 ? 2 * nM : 0.0));
  W.npC = gup;
  k_check<<<1, kThreads, 0, st>>>(S, W.partC.p, W.npC);
  note(W, st, "pcg_check", -1, 0.0);
  W.launches += 3;
  WN_CUDA(cudaGetLastError());
  const double b_mid = W.bytes;
  W.cur_prec = true;
  const int rc = apply_prec<TM>(s, W, precond, prec_input(B), B.z, S, st, d0);
  W.cur_prec = false;
  W.iter_core_bytes = b_mid - b_start;
  W.iter_prec_bytes = W.bytes - b_mid;
  return rc;
}

// PCG on the fine matrix: solves A x = b from x = 0 to ||r|| <= rtol ||b||.  The first chunk
// of iterations is issued directly (iteration 0 forms p = z); later chunks replay one
// captured CUDA graph.  mode indexes the graph cache (0 fp64, 1 mixed, 2 fp32).
template <typename TK, typename TM>
static int pcg_solve(Solid* s, SolverWork& W, int mode, const TK* b, double rtol, int max_iter, int precond,
                     int chunk, int use_graph, PcgScalars* S, cudaStream_t st, PcgScalars* hS) {
  PcgBufs<TK, TM> B = pcg_bufs<TK, TM>(s, W);
  WN_CUDA(cudaMemsetAsync(B.p0, 0, W.n * sizeof(TK), st));  // iteration 0: p = z + 0 * p_old
  WN_CUDA(cudaMemsetAsync(B.p1, 0, W.n * sizeof(TK), st));
  const size_t note0 = W.notes.size();
  W.cur_iter = -1;
  W.npC = resident_grid(k_init_vecs<TK, TM>, kThreads, (W.n + kThreads - 1) / kThreads);
  k_init_vecs<TK, TM><<<W.npC, kThreads, 0, st>>>(W.n, b, B.x, B.r, B.rm, W.partC.p, half_scale<TM>(W));
  note(W, st, "pcg_init", -1, 3.0 * W.n * sizeof(TK) + (B.rm ? (double)W.n * sizeof(TM) : 0.0));
  k_init_scalars<<<1, kThreads, 0, st>>>(S, W.partC.p, W.npC, rtol, max_iter);
  note(W, st, "pcg_check", -1, 0.0);
  W.launches += 2;
  WN_CUDA(cudaGetLastError());
  WN_CHECK(apply_prec<TM>(s, W, precond, prec_input(B), B.z, S, st));
  const double bytes_before_iterations = W.bytes;
  chunk = std::max(2, chunk + (chunk & 1));  // even: the parity pattern repeats per chunk
  if (W.profile) use_graph = 0;  // every launch timed by its own event
  GraphCache& G = W.graphs[mode][precond];
  const int64_t key = chunk;
  for (int k = 0; k < chunk && k < max_iter; ++k) {
    W.cur_iter = k;
    WN_CHECK((pcg_iteration<TK, TM>(s, W, precond, k, S, st)));
  }
  int k0 = chunk;
  while (true) {
    WN_CUDA(cudaMemcpyAsync(hS, S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    WN_CUDA(cudaStreamSynchronize(st));
    if (hS->done || k0 >= max_iter) break;
    if (use_graph) {
      if (G.key != key || G.stream != st || !G.exec || G.fine_epoch != s->fine.epoch) {
        G.reset();
        cudaGraph_t graph;
        const int64_t before = W.launches;
        const double bytes_before = W.bytes;
        const double core = W.iter_core_bytes, prec = W.iter_prec_bytes;
        WN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = 0;
        // the iteration count and max_iter live on the device (k_check) and the chunk is
        // even, so one captured chunk serves every later chunk
        for (int k = 0; k < chunk && rc == 0; ++k) rc = pcg_iteration<TK, TM>(s, W, precond, chunk + k, S, st);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        WN_CHECK(rc);
        WN_CUDA(e);
        e = cudaGraphInstantiate(&G.exec, graph, 0);
        cudaGraphDestroy(graph);
        WN_CUDA(e);
        G.key = key;
        G.stream = st;
        G.fine_epoch = s->fine.epoch;
        G.kernels = W.launches - before;
        W.launches = before;
        W.bytes = bytes_before;  // captured, not run
        W.iter_core_bytes = core;
        W.iter_prec_bytes = prec;
      }
      WN_CUDA(cudaGraphLaunch(G.exec, st));
      W.launches += G.kernels;
    } else {
      for (int k = 0; k < chunk; ++k) {
        W.cur_iter = k0 + k;
        WN_CHECK((pcg_iteration<TK, TM>(s, W, precond, k0 + k, S, st)));
      }
    }
    k0 += chunk;
  }
  W.cur_iter = -1;
  // bytes of the iterations that ran: I products / updates / checks and I - 1 preconditioner
  // applies (the last check ends the loop before its apply); launches past the device-side
  // end of the loop return at once and count nothing
  const int I = hS->iters;
  W.bytes = bytes_before_iterations + I * W.iter_core_bytes + std::max(I - 1, 0) * W.iter_prec_bytes;
  for (size_t i = note0; i < W.notes.size(); ++i) {
    SolverWork::Note& nt = W.notes[i];
    if (nt.iter >= I || (nt.prec && nt.iter == I - 1)) nt.valid = false;
  }
  return 0;
}

// ---------------------------------------------------------------------------------------
// setup: host hierarchy -> device
// ---------------------------------------------------------------------------------------
int DevBsr::upload(const HostBsr& h) {
  br = h.br;
  bc = h.bc;
  n_rows = h.n_rows;
  n_cols = h.n_cols;
  nnzb = h.nnzb();
  WN_CHECK(rp.upload(h.rp));
  WN_CHECK(ci.upload(h.ci));
  WN_CHECK(v64.upload(h.v));
  std::vector<float> f(h.v.begin(), h.v.end());
  WN_CHECK(v32.upload(f));
  return 0;
}

static void cheb_coefficients(const wn_amg_params& prm, DevLevel& L) {
  const double lmax = prm.cheb_safety * L.rho;
  const double lmin = prm.cheb_lower * lmax;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  L.inv_theta = 1.0 / theta;
  L.c1.clear();
  L.c2.clear();
  for (int k = 1; k < prm.smoother_degree; ++k) {
    const double rho_new = 1.0 / (2.0 * sigma - rho_old);
    L.c1.push_back(rho_new * rho_old);
    L.c2.push_back(2.0 * rho_new / delta);
    rho_old = rho_new;
  }
}

static int ensure_work(Solid* s) {
  if (!s->work) s->work.reset(new SolverWork());
  SolverWork& W = *s->work;
  const int64_t n = s->n_nodes * s->bs;
  if (W.n != n) {
    W.n = n;
    WN_CHECK(W.p64.alloc(n));
    WN_CHECK(W.p32.alloc(n));
    WN_CHECK(W.u64.alloc(n));
    WN_CHECK(W.ulo.alloc(n));
    WN_CHECK(W.r64.alloc(n));
    WN_CHECK(W.r32.alloc(n));
    WN_CHECK(W.dinv64.alloc(n));
    WN_CHECK(W.dinv32.alloc(n));
    for (auto& a : W.graphs)
      for (auto& g : a) g.reset();
  }
  WN_CHECK(W.partA.alloc(SolverWork::kMaxParts));
  WN_CHECK(W.partB.alloc(SolverWork::kMaxParts));
  WN_CHECK(W.partC.alloc(SolverWork::kMaxParts));
  WN_CHECK(W.scal.alloc(2));
  if (!W.ev0) {
    WN_CUDA(cudaEventCreate(&W.ev0));
    WN_CUDA(cudaEventCreate(&W.ev1));
  }
  return 0;
}

int solver_setup(Solid* s, const wn_amg_params& prm) {
  WN_REQUIRE(s->assembled, WN_ESTATE, "AMG setup: matrix not assembled");
  WN_REQUIRE(prm.smoother_degree >= 1 && prm.smoother_degree <= 8, WN_EINVAL, "AMG setup: smoother_degree in [1, 8]");
  WN_REQUIRE(prm.max_levels >= 1 && prm.max_levels <= 16, WN_EINVAL, "AMG setup: max_levels in [1, 16]");
  const auto t0 = std::chrono::steady_clock::now();
  // WN_AMG_TRACE=1: the steps around the hierarchy build on stderr too
  const bool trace = std::getenv("WN_AMG_TRACE") != nullptr;
  auto tmark = t0;
  auto step = [&](const char* what) {
    if (!trace) return;
    cudaDeviceSynchronize();
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "solver_setup: %-24s %8.3f s\n", what, std::chrono::duration<double>(now - tmark).count());
    tmark = now;
  };
  std::unique_ptr<AmgHierarchy> H(new AmgHierarchy());
  // device setup first (1 = a row beyond its shared-memory capacities: the host builder then)
  int dev_rc = 1;
  if (prm.setup_on_device) {
    dev_rc = amg_build_device(s, prm, *H);
    WN_CHECK(dev_rc < 0 || dev_rc > 1 ? dev_rc : 0);
    if (dev_rc == 1) H.reset(new AmgHierarchy());
  }
  if (dev_rc != 0) {
    const int nb = s->bs * s->bs;
    std::vector<double> soa(s->nnzb * nb), vals(s->nnzb * nb);
    WN_CUDA(cudaMemcpy(soa.data(), s->k64.p, soa.size() * sizeof(double), cudaMemcpyDeviceToHost));
    if (s->bs == 3) {
      for (int64_t b = 0; b < s->nnzb; ++b)  // component-major on the device -> row-major blocks
        for (int k = 0; k < 9; ++k) vals[b * 9 + k] = soa[k * s->nnzb + b];
    } else {
      vals.swap(soa);  // 6x6 blocks are stored row-major already
    }
    std::vector<double>().swap(soa);
    const uint8_t* fixed = s->bcs_applied ? s->h_fixed.data() : nullptr;
    WN_CHECK(amg_build(prm, s->n_nodes, s->bs, s->h_row_ptr.data(), s->h_col_idx.data(), vals.data(),
                       s->h_nodes.data(), fixed, H->host));
    H->levels.resize(H->host.levels.size());
  }
  step("hierarchy build");
  H->degree = prm.smoother_degree;
  static uint64_t next_id = 0;
  H->id = ++next_id;
  for (size_t l = 0; l < H->host.levels.size(); ++l) {
    const HostLevel& h = H->host.levels[l];
    DevLevel& L = H->levels[l];
    L.bs = h.bs;
    L.n_nodes = h.n_nodes;
    if (l == 0) {
      L.a_rp = s->row_ptr.p;
      L.a_ci = s->col_idx.p;
    }
    if (!H->device_built) {
      if (l > 0) WN_CHECK(L.A.upload(h.A));
      WN_CHECK(L.dinv64.upload(h.dinv));
      std::vector<float> f(h.dinv.begin(), h.dinv.end());
      WN_CHECK(L.dinv32.upload(f));
      WN_CHECK(L.P.upload(h.P));
      WN_CHECK(L.R.upload(h.R));
      if (l > 0) L.h_A_rp = h.A.rp;
      L.h_P_rp = h.P.rp;
      L.h_R_rp = h.R.rp;
    }
  }
  // block-Jacobi smoothing of the 6-DOF levels: their basis is changed on the device before
  // the packs are made (it rewrites A, P, R, 1/diag and rho of those levels)
  if (prm.coarse_block_smoother) WN_CHECK(amg_coarse_block_basis(*H, prm));
  step("coarse block basis");
  for (size_t l = 0; l < H->host.levels.size(); ++l) {
    const HostLevel& h = H->host.levels[l];
    DevLevel& L = H->levels[l];
    L.rho = h.rho;
    cheb_coefficients(prm, L);
    // matrices of at least stream_min_mb MB (FP32) are streamed from tile-major packs (on the
    // 1M-DOF I-beam: level 1 and the transfers of levels 0-1, 24-142 MB; streaming level 2 and
    // the level-1 transfers too, at 4 MB rather than 32 MB, took 0.8 ms off a 47 ms solve)
    auto stream_if_large = [&](StreamMat& m, const std::vector<int32_t>& h_rp, const DevBsr& db) -> int {
      if (prm.stream_min_mb < 0.0 ||
          (double)(db.nnzb * db.br * db.bc * (int64_t)sizeof(float)) < prm.stream_min_mb * 1048576.0)
        return 0;
      WN_CHECK(m.make_plan(h_rp.data(), db.n_rows, db.br, db.bc));
      return m.pack(db.rp.p, db.ci.p, db.v32.p, db.v64.p, 0, 0);
    };
    if (l > 0) WN_CHECK(stream_if_large(L.As, L.h_A_rp, L.A));
    WN_CHECK(stream_if_large(L.Ps, L.h_P_rp, L.P));
    WN_CHECK(stream_if_large(L.Rs, L.h_R_rp, L.R));
    WN_CHECK(L.v64.alloc(h.n_nodes * h.bs));
    WN_CHECK(L.v32.alloc(h.n_nodes * h.bs));
  }
  step("level packs and vectors");
  H->n_coarse = H->host.n_coarse;
  WN_CHECK(H->coarse_inv.upload(H->host.coarse_inv));
  WN_CHECK(H->cb64.alloc(H->n_coarse));
  WN_CHECK(H->cx64.alloc(H->n_coarse));
  WN_CHECK(H->cb32.alloc(H->n_coarse));
  WN_CHECK(H->cx32.alloc(H->n_coarse));
  WN_CUDA(cudaDeviceSynchronize());
  step("coarse upload");
  H->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  s->amg = std::move(H);  // frees the previous hierarchy
  step("previous hierarchy freed");
  WN_CHECK(ensure_work(s));
  for (auto& a : s->work->graphs)
    for (auto& g : a) g.reset();
  step("graphs reset");
  return 0;
}

// ---------------------------------------------------------------------------------------
// solve
// ---------------------------------------------------------------------------------------
// r64 = F - K (u64 + ulo) with the compensated kernel; *rr = ||r64||^2
static int true_residual(Solid* s, SolverWork& W, const double* F, float* r32, cudaStream_t st, double* rr) {
  auto launch = [&](auto kern) {
    W.npC = resident_grid(kern, kThreads, (s->n_nodes * 32 + kThreads - 1) / kThreads);
    kern<<<W.npC, kThreads, 0, st>>>(s->n_nodes, s->row_ptr.p, s->col_idx.p, s->k64.p, s->nnzb, F, W.u64.p, W.ulo.p,
                                     W.r64.p, r32, W.partC.p);
  };
  if (s->bs == 3)
    launch(k_outer_residual_dd<3>);
  else
    launch(k_outer_residual_dd<6>);
  note(W, st, "outer_residual", -1,
       mat_bytes(s->nnzb, s->bs, s->bs, s->n_nodes, 8) + 4.0 * W.n * 8 + (r32 ? 4.0 * W.n : 0.0));
  k_reduce_rr<<<1, kThreads, 0, st>>>(W.scal.p + 1, W.partC.p, W.npC);
  note(W, st, "reduce", -1, 0.0);
  W.launches += 2;
  WN_CUDA(cudaGetLastError());
  PcgScalars h;
  WN_CUDA(cudaMemcpyAsync(&h, W.scal.p + 1, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  *rr = h.rr;
  return 0;
}

// out = s * in, elementwise
__global__ void k_scale_copy(int64_t n, const float* __restrict__ s, const float* __restrict__ in,
                             float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = s[i] * in[i];
}

// The FP16 V-cycle's inputs for the current matrix: the equilibration S = diag(K)^-1/2 (every
// solve) and the FP16 pack of S K S (rebuilt when the values changed since it was made).  It
// needs a C3D10 system with the streamed fine level and an AMG hierarchy.
static int prepare_half(Solid* s, SolverWork& W, cudaStream_t st) {
  WN_REQUIRE(s->bs == 3 && s->amg, WN_EINVAL, "FP16 V-cycle: needs a C3D10 (3x3) system with the AMG preconditioner");
  WN_REQUIRE(s->stream_fine && s->fine.n_tiles > 0 && s->fine.size16 > 0 && s->fine.packed, WN_ESTATE,
             "FP16 V-cycle: needs the streamed fine level (wn_solid_set_stream(h, 1))");
  WN_REQUIRE(!s->amg->levels.empty(), WN_ESTATE, "FP16 V-cycle: the hierarchy has no fine level to smooth");
  if (W.s32.n != W.n) {
    WN_CHECK(W.s64.alloc(W.n));
    WN_CHECK(W.s32.alloc(W.n));
    WN_CHECK(W.q32.alloc(W.n));
  }
  k_fill_scale<<<vec_grid(W.n), kThreads, 0, st>>>(s->n_nodes, s->nnzb, s->diag_block.p, s->k64.p, W.s64.p, W.s32.p,
                                                   W.q32.p);
  WN_CUDA(cudaGetLastError());
  note(W, st, "fill_scale", -1, 28.0 * W.n);
  W.launches++;
  if (s->fine.version16 != s->values_version) {
    WN_CHECK(s->fine.pack_half33(s->row_ptr.p, s->col_idx.p, s->block_row.p, s->k64.p, s->nnzb, W.s64.p,
                                 s->values_version, st));
    note(W, st, "pack_half", -1, mat_bytes(s->nnzb, 3, 3, s->n_nodes, 8) + mat_bytes(s->nnzb, 3, 3, s->n_nodes, 2));
    W.launches++;
  }
  return 0;
}

// Outer loop common to all modes: u = 0; r = F - K u; while ||r|| > rtol ||F||: solve K d = r
// approximately with the inner PCG, u += d, recompute the residual.  u is kept as a
// double-double pair and r is evaluated with compensated products and sums, so the test
// resolves residuals below the FP64 rounding level of K u (which for load cases with large
// displacements can lie near 1e-8 ||F||); the returned u is the pair rounded to FP64.
//   mode 0 (fp64):  inner PCG FP64 (matrix, vectors, V-cycle), target 0.25 rtol ||F|| / ||r||
//   mode 1 (mixed): inner PCG FP64 with an FP32 AMG V-cycle (FP32 values, vectors and
//                   accumulation; FP64 coarsest inverse), same target
//   mode 2 (fp32 IR): inner PCG entirely FP32 (FP32 K SpMV) to max(inner_rtol, target);
//                   the classic iterative refinement of solid_solver.py:271-300
//   mode 3 (mixed, FP16 V-cycle): mode 1 with the fine level of the V-cycle on the
//                   equilibrated matrix S K S in FP16 (FP32 arithmetic and vectors); the
//                   reference's tri-precision preconditioner (mixed_precision.py:96-103)
// FP64 dot products everywhere.  The FP64 loop makes the stopping test the true residual.
template <typename TK, typename TM>
static int outer_loop(Solid* s, SolverWork& W, int mode, const double* F, double fnorm, const wn_solve_params& prm,
                      int chunk, cudaStream_t st, int* total_iters, int* outer, int* status, double* rr) {
  const int64_t n = W.n;
  const int max_outer = prm.max_outer > 0 ? prm.max_outer : 10;
  PcgScalars hS{};
  WN_CUDA(cudaMemsetAsync(W.u64.p, 0, n * sizeof(double), st));
  WN_CUDA(cudaMemsetAsync(W.ulo.p, 0, n * sizeof(double), st));
  WN_CUDA(cudaMemcpyAsync(W.r64.p, F, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  *rr = fnorm * fnorm;
  bool first = true;
  while (true) {
    if (!first) WN_CHECK(true_residual(s, W, F, mode == 2 ? W.r32.p : nullptr, st, rr));
    const double rn = std::sqrt(*rr);
    if (!std::isfinite(*rr)) {
      *status = WN_EBREAKDOWN;
      break;
    }
    if (rn <= prm.rtol * fnorm) break;
    if (*outer >= max_outer || *total_iters >= prm.max_iter) {
      *status = WN_ENOCONV;
      break;
    }
    // inner target a quarter of the remaining factor: the inner PCG's recursive residual drifts
    // from the true one by FP64 rounding (about 5e-9 ||F|| on the 1M-DOF I-beam), so a target
    // of rtol / 4 lets the first pass meet rtol on the true residual without a second pass
    double target = std::min(0.5, 0.25 * prm.rtol * fnorm / rn);
    if (mode == 2) {
      const double inner = prm.inner_rtol > 0.0 ? prm.inner_rtol : 1e-4;
      target = std::max(target, inner);
      if (first) {  // r32 = (float) F
        WN_CHECK(true_residual(s, W, F, W.r32.p, st, rr));
      }
    }
    first = false;
    const TK* b;
    if constexpr (std::is_same<TK, float>::value)
      b = W.r32.p;
    else
      b = W.r64.p;
    WN_CHECK((pcg_solve<TK, TM>(s, W, mode, b, target, prm.max_iter - *total_iters, prm.precond, chunk,
                                prm.use_graph, W.scal.p, st, &hS)));
    *total_iters += hS.iters;
    ++*outer;
    if (hS.status == WN_EBREAKDOWN || hS.status == WN_ETIMEOUT) {
      *status = hS.status;
      break;
    }
    PcgBufs<TK, TM> B = pcg_bufs<TK, TM>(s, W);
    k_accumulate<TK><<<vec_grid(n), kThreads, 0, st>>>(n, W.u64.p, W.ulo.p, B.x);
    note(W, st, "accumulate", -1, 4.0 * n * 8 + (double)n * sizeof(TK));
    W.launches++;
    WN_CUDA(cudaGetLastError());
  }
  return 0;
}

int solver_solve(Solid* s, const double* F, double* u, const wn_solve_params& prm, wn_solve_stats* stats,
                 cudaStream_t st) {
  WN_REQUIRE(s->assembled, WN_ESTATE, "solve: matrix not assembled");
  WN_REQUIRE(prm.precond >= 0 && prm.precond <= 3, WN_EINVAL,
             "solve: precond must be 0 (none), 1 (jacobi), 2 (amg) or 3 (block jacobi)");
  WN_REQUIRE(prm.precision >= 0 && prm.precision <= 3, WN_EINVAL,
             "solve: precision must be 0 (fp64), 1 (mixed: fp32 AMG in fp64 PCG), 2 (fp32 PCG in fp64 refinement) "
             "or 3 (mixed with the fp16 fine-level V-cycle)");
  WN_REQUIRE(prm.precision != 3 || prm.precond == 2, WN_EINVAL,
             "solve: precision 3 (fp16 V-cycle) needs precond 2 (amg)");
  WN_REQUIRE(prm.max_iter > 0 && prm.rtol > 0.0, WN_EINVAL, "solve: max_iter > 0 and rtol > 0 required");
  if (prm.precond == 2 && !s->amg) WN_CHECK(solver_setup(s, amg_default_params()));
  WN_CHECK(ensure_work(s));
  SolverWork& W = *s->work;
  W.launches = 0;
  if (st == 0) {  // stream capture is not allowed on the legacy default stream
    if (!W.own) WN_CUDA(cudaStreamCreate(&W.own));  // blocking: ordered with stream 0
    st = W.own;
  }
  const int64_t n = W.n;
  const int chunk = prm.chunk > 0 ? prm.chunk : 8;
  PcgScalars hS{};
  W.bytes = 0.0;
  W.profile = prm.profile != 0;
  W.notes.clear();
  W.cur_iter = -1;
  W.cur_prec = false;
  if (W.profile && W.note_events.empty()) {
    cudaEvent_t e = nullptr;
    WN_CUDA(cudaEventCreate(&e));
    W.note_events.push_back(e);
  }
  if (W.profile) WN_CUDA(cudaEventRecord(W.note_events[0], st));
  k_fill_dinv<<<vec_grid(n), kThreads, 0, st>>>(s->n_nodes, s->bs, s->nnzb, s->diag_block.p, s->k64.p, W.dinv64.p,
                                                 W.dinv32.p);
  note(W, st, "fill_dinv", -1, 20.0 * n);
  W.launches++;
  if (prm.precond == 3) {  // block pseudo-inverses of the current values
    const int64_t nb = s->n_nodes * s->bs * s->bs;
    if (W.binv64.n != nb) {
      WN_CHECK(W.binv64.alloc(nb));
      WN_CHECK(W.binv32.alloc(nb));
    }
    if (s->bs == 3)
      k_fill_block_pinv<3><<<grid_for(s->n_nodes, 1, 128, 8), 128, 0, st>>>(s->n_nodes, s->nnzb, s->diag_block.p,
                                                                             s->k64.p, W.binv64.p, W.binv32.p);
    else
      k_fill_block_pinv<6><<<grid_for(s->n_nodes, 1, 128, 8), 128, 0, st>>>(s->n_nodes, s->nnzb, s->diag_block.p,
                                                                             s->k64.p, W.binv64.p, W.binv32.p);
    note(W, st, "fill_block_pinv", -1, 20.0 * nb);
    W.launches++;
    WN_CUDA(cudaGetLastError());
  }
  WN_CUDA(cudaEventRecord(W.ev0, st));
  W.npC = resident_grid(k_dot_self<double>, kThreads, (n + kThreads - 1) / kThreads);
  k_dot_self<double><<<W.npC, kThreads, 0, st>>>(n, F, W.partC.p);
  note(W, st, "dot", -1, 8.0 * n);
  k_reduce_rr<<<1, kThreads, 0, st>>>(W.scal.p + 1, W.partC.p, W.npC);
  note(W, st, "reduce", -1, 0.0);
  W.launches += 2;
  WN_CUDA(cudaMemcpyAsync(&hS, W.scal.p + 1, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  const double fnorm = std::sqrt(hS.rr);
  int total_iters = 0, outer = 0, status = 0;
  double rr = 0.0;
  if (fnorm == 0.0) {
    WN_CUDA(cudaMemsetAsync(u, 0, n * sizeof(double), st));
  } else if (!std::isfinite(fnorm)) {
    status = WN_EBREAKDOWN;
    rr = hS.rr;
    WN_CUDA(cudaMemsetAsync(u, 0, n * sizeof(double), st));
  } else {
    if (prm.precision == 0)
      WN_CHECK((outer_loop<double, double>(s, W, 0, F, fnorm, prm, chunk, st, &total_iters, &outer, &status, &rr)));
    else if (prm.precision == 1)
      WN_CHECK((outer_loop<double, float>(s, W, 1, F, fnorm, prm, chunk, st, &total_iters, &outer, &status, &rr)));
    else if (prm.precision == 3) {
      WN_CHECK(prepare_half(s, W, st));
      W.half = true;
      const int rc = outer_loop<double, float>(s, W, 3, F, fnorm, prm, chunk, st, &total_iters, &outer, &status, &rr);
      W.half = false;
      WN_CHECK(rc);
    } else
      WN_CHECK((outer_loop<float, float>(s, W, 2, F, fnorm, prm, chunk, st, &total_iters, &outer, &status, &rr)));
    WN_CUDA(cudaMemcpyAsync(u, W.u64.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  WN_CUDA(cudaEventRecord(W.ev1, st));
  WN_CUDA(cudaEventSynchronize(W.ev1));
  float ms = 0.f;
  WN_CUDA(cudaEventElapsedTime(&ms, W.ev0, W.ev1));
  if (W.profile) {  // per kernel class: launches that did their work, event-timed durations
    W.last_profile.clear();
    std::map<std::string, size_t> row_of;
    for (size_t i = 0; i < W.notes.size(); ++i) {
      const SolverWork::Note& nt = W.notes[i];
      if (!nt.valid) continue;
      float t = 0.f;
      WN_CUDA(cudaEventElapsedTime(&t, W.note_events[i], W.note_events[i + 1]));
      const std::string name = nt.level >= 0 ? "l" + std::to_string(nt.level) + "." + nt.kind : std::string(nt.kind);
      auto it = row_of.find(name);
      if (it == row_of.end()) {
        it = row_of.emplace(name, W.last_profile.size()).first;
        W.last_profile.push_back(SolverWork::ProfileRow{name, 0, 0.0, 0.0});
      }
      SolverWork::ProfileRow& r = W.last_profile[it->second];
      r.count++;
      r.ms += t;
      r.bytes += nt.bytes;
    }
    W.profile = false;
  }
  if (stats) {
    stats->iterations = total_iters;
    stats->outer_iterations = outer;
    stats->status = status;
    stats->rel_res = fnorm > 0.0 ? std::sqrt(rr) / fnorm : 0.0;
    stats->solve_seconds = ms * 1e-3;
    stats->kernel_launches = W.launches;
    stats->setup_seconds = s->amg ? s->amg->setup_seconds : 0.0;
    stats->n_levels = s->amg ? (int)s->amg->levels.size() + 1 : 0;
    stats->algorithmic_bytes = W.bytes;
  }
  return 0;
}

int solver_profile(Solid* s, int capacity, int* n_rows, char* names, int64_t* counts, double* ms, double* bytes) {
  WN_REQUIRE(s->work, WN_ESTATE, "solve profile: no solve has run on this handle");
  const auto& P = s->work->last_profile;
  *n_rows = (int)P.size();
  for (int i = 0; i < capacity && i < (int)P.size(); ++i) {
    if (names) {
      std::strncpy(names + (size_t)i * 48, P[i].name.c_str(), 47);
      names[(size_t)i * 48 + 47] = 0;
    }
    if (counts) counts[i] = P[i].count;
    if (ms) ms[i] = P[i].ms;
    if (bytes) bytes[i] = P[i].bytes;
  }
  return 0;
}

int amg_vcycle(Solid* s, int precision, const void* r, void* z, cudaStream_t st) {
  WN_REQUIRE(s->amg, WN_ESTATE, "vcycle: no AMG hierarchy (call wn_amg_setup)");
  WN_CHECK(ensure_work(s));
  SolverWork& W = *s->work;
  k_fill_dinv<<<vec_grid(W.n), kThreads, 0, st>>>(s->n_nodes, s->bs, s->nnzb, s->diag_block.p, s->k64.p, W.dinv64.p,
                                                  W.dinv32.p);
  WN_CUDA(cudaMemsetAsync(W.scal.p, 0, sizeof(PcgScalars), st));  // done = 0
  if (precision == 0)
    return vcycle<double>(s, *s->amg, W, 0, (const double*)r, (double*)z, nullptr, W.scal.p, st);
  if (precision == 3) {  // the FP16 V-cycle: input S r, output unscaled by its last step
    WN_CHECK(prepare_half(s, W, st));
    k_scale_copy<<<vec_grid(W.n), kThreads, 0, st>>>(W.n, W.s32.p, (const float*)r, W.r32.p);
    WN_CUDA(cudaGetLastError());
    W.half = true;
    const int rc = vcycle<float>(s, *s->amg, W, 0, W.r32.p, (float*)z, nullptr, W.scal.p, st);
    W.half = false;
    return rc;
  }
  return vcycle<float>(s, *s->amg, W, 0, (const float*)r, (float*)z, nullptr, W.scal.p, st);
}

}  // namespace wn
