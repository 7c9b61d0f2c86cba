// Multi-right-hand-side PCG: kBatch (32) load cases against one matrix and one AMG hierarchy.
//
// The reference solves load cases one at a time (each a solve_c3d10_pcg call,
// wnfea/solver/solid_solver.py:197-308); here the batch shares every matrix read.  Each
// load case keeps its own Krylov recurrence -- its own alpha, beta, convergence test and
// iteration count -- so every column reproduces the single-RHS PCG; only the products are
// batched:
//   * block rows are handled by groups of 8 lanes, lane g of a group owning load cases
//     4g..4g+3 (16-byte vector loads of the DOF-major n x 32 vectors), 4 rows per warp;
//   * per-case FP64 dot products are two-stage and deterministic (per-CTA partials of all
//     32 cases, reduced in a fixed order by a one-CTA scalar kernel);
//   * finished cases take alpha = beta = 0 and stop changing while the rest iterate;
//   * the batched V-cycle mirrors the single-RHS one (Chebyshev smoothing, restriction,
//     prolongation, dense coarsest inverse) in FP32 (mixed) or FP64;
//   * an FP64 refinement loop checks every case on its true residual F - K U and restarts
//     only the cases that are not yet at rtol.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <type_traits>

#include "amg.h"
#include "block.h"
#include "common.cuh"
#include "solid.h"
#include "spmv.cuh"
#include "solver.h"

namespace wn {
namespace {

constexpr int kThreads = 256;
constexpr int kRowsPerWarp = 4;  // 8 lanes per block row

// ---------------------------------------------------------------------------------------
// 4-case vectors
// ---------------------------------------------------------------------------------------
template <typename T>
struct C4 {
  T v[4];
};
__device__ __forceinline__ C4<float> ld4(const float* __restrict__ p) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  return {{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ C4<double> ld4(const double* __restrict__ p) {
  const double2 a = reinterpret_cast<const double2*>(p)[0];
  const double2 b = reinterpret_cast<const double2*>(p)[1];
  return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, const C4<float>& v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
__device__ __forceinline__ void st4(double* p, const C4<double>& v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v.v[0], v.v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v.v[2], v.v[3]);
}
template <typename TO, typename TI>
__device__ __forceinline__ C4<TO> cvt4(const C4<TI>& a) {
  return {{(TO)a.v[0], (TO)a.v[1], (TO)a.v[2], (TO)a.v[3]}};
}

// ---------------------------------------------------------------------------------------
// row loop and per-case reductions
// ---------------------------------------------------------------------------------------
// Defines c0 (first load case of this lane) and loops `row` over the block rows of this
// group.  Lanes leave the loop independently (no shuffles inside).
#define BATCH_ROW_LOOP(n_rows)                                                           \
  const int c0 = (threadIdx.x & 7) * 4;                                                  \
  const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;           \
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;                         \
  for (int64_t row = warp0 * kRowsPerWarp + ((threadIdx.x & 31) >> 3); row < (n_rows);   \
       row += nwarps * kRowsPerWarp)

// Element loop over an n x kBatch vector in 4-case quads: defines c0 and the quad index t
// (elements 4t..4t+3, DOF 4t / kBatch).  The grid stride is a multiple of 8 quads, so a
// thread always sees the same four cases.
#define BATCH_QUAD_LOOP(n)                                                                     \
  const int c0 = (threadIdx.x & 7) * 4;                                                        \
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (n) * (kBatch / 4);     \
       t += (int64_t)gridDim.x * blockDim.x)

// CTA partials of the four per-lane case sums d[0..3] (cases c0..c0+3 with c0 = (lane & 7) * 4)
// into part[blockIdx.x * kBatch + case], in a fixed order.  All threads of the CTA call it.
__device__ __forceinline__ void write_case_parts(double (&d)[4], double* __restrict__ part) {
  __shared__ double sh[kThreads / 32][kBatch];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d[k] += __shfl_xor_sync(0xffffffffu, d[k], 8);
    d[k] += __shfl_xor_sync(0xffffffffu, d[k], 16);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane < 8)
#pragma unroll
    for (int k = 0; k < 4; ++k) sh[w][lane * 4 + k] = d[k];
  __syncthreads();
  if (threadIdx.x < kBatch) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k][threadIdx.x];
    part[(int64_t)blockIdx.x * kBatch + threadIdx.x] = s;
  }
}

// one-CTA fixed-order sums of nparts x kBatch partials; thread j < kBatch receives case j
__device__ __forceinline__ double reduce_case_parts(const double* __restrict__ part, int nparts) {
  __shared__ double sh[kThreads];
  const int c = threadIdx.x & 31, sub = threadIdx.x >> 5, nsub = blockDim.x >> 5;
  double s = 0.0;
  for (int k = sub; k < nparts; k += nsub) s += part[(int64_t)k * kBatch + c];
  sh[threadIdx.x] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < kBatch)
    for (int k = 0; k < nsub; ++k) t += sh[k * 32 + threadIdx.x];
  __syncthreads();
  return t;
}

// ---------------------------------------------------------------------------------------
// batched block-row product: acc[r][k] = sum_q A(row, q)[r][c] * x(col_q, c)[case c0 + k]
// ---------------------------------------------------------------------------------------
template <typename T>
struct BLoad {
  const T* __restrict__ x;
  __device__ __forceinline__ C4<T> operator()(int64_t i, int c0) const { return ld4(x + i * kBatch + c0); }
};
template <typename T>
struct BD0 {  // first Chebyshev step from zero: dinv_i b_i / theta
  const T* __restrict__ b;
  const T* __restrict__ dinv;
  T inv_theta;
  __device__ __forceinline__ C4<T> operator()(int64_t i, int c0) const {
    C4<T> v = ld4(b + i * kBatch + c0);
    const T di = dinv[i];
#pragma unroll
    for (int k = 0; k < 4; ++k) v.v[k] = di * v.v[k] * inv_theta;
    return v;
  }
};
template <typename TK, typename TM>
struct BPNew {  // p_new = z + beta p_old, per case
  const TM* __restrict__ z;
  const TK* __restrict__ p;
  C4<TK> beta;
  __device__ __forceinline__ C4<TK> operator()(int64_t i, int c0) const {
    const C4<TK> zz = cvt4<TK>(ld4(z + i * kBatch + c0));
    const C4<TK> pp = ld4(p + i * kBatch + c0);
    C4<TK> o;
#pragma unroll
    for (int k = 0; k < 4; ++k) o.v[k] = zz.v[k] + beta.v[k] * pp.v[k];
    return o;
  }
};

template <int BR, int BC, Layout LY, typename T, typename XF>
__device__ __forceinline__ void batch_block_row(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                const T* __restrict__ av, int64_t stride, int64_t row, int c0,
                                                const XF& xf, T (&acc)[BR][4]) {
#pragma unroll
  for (int r = 0; r < BR; ++r)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[r][k] = T(0);
  const int32_t q0 = rp[row], q1 = rp[row + 1];
#pragma unroll 2
  for (int32_t q = q0; q < q1; ++q) {
    const int64_t col = ci[q];
    C4<T> xv[BC];
#pragma unroll
    for (int c = 0; c < BC; ++c) xv[c] = xf(col * BC + c, c0);
#pragma unroll
    for (int r = 0; r < BR; ++r)
#pragma unroll
      for (int c = 0; c < BC; ++c) {
        const T a = (LY == kSoA) ? av[(int64_t)(r * BC + c) * stride + q] : av[(int64_t)q * (BR * BC) + r * BC + c];
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[r][k] = fma(a, xv[c].v[k], acc[r][k]);
      }
  }
}

template <int BS>
struct BLayout {
  static constexpr Layout value = (BS == 3) ? kSoA : kAoS;
};

// ---------------------------------------------------------------------------------------
// batched V-cycle kernels (same arithmetic per case as the single-RHS smoother kernels)
// ---------------------------------------------------------------------------------------
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) kb_pre_first(int64_t n_rows, const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                         int64_t stride, const T* __restrict__ b,
                                                         const T* __restrict__ dinv, T inv_theta, int deg, T c1, T c2,
                                                         T* __restrict__ x, T* __restrict__ r, T* __restrict__ d,
                                                         T* __restrict__ res, const int* __restrict__ done) {
  if (*done) return;
  BATCH_ROW_LOOP(n_rows) {
    T acc[BS][4];
    batch_block_row<BS, BS, BLayout<BS>::value>(rp, ci, av, stride, row, c0, BD0<T>{b, dinv, inv_theta}, acc);
#pragma unroll
    for (int rr = 0; rr < BS; ++rr) {
      const int64_t i = row * BS + rr;
      const int64_t o = i * kBatch + c0;
      const T di = dinv[i];
      const C4<T> bi = ld4(b + o);
      C4<T> xo, ro, dd;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const T t = acc[rr][k];
        const T d0 = di * bi.v[k] * inv_theta;
        if (deg == 1) {
          xo.v[k] = d0;
          ro.v[k] = bi.v[k] - t;
        } else {
          const T r1 = di * bi.v[k] - di * t;
          const T d1 = c1 * d0 + c2 * r1;
          xo.v[k] = d0 + d1;
          ro.v[k] = r1;
          dd.v[k] = d1;
        }
      }
      st4(x + o, xo);
      if (deg == 1) {
        st4(res + o, ro);
      } else {
        st4(r + o, ro);
        st4(d + o, dd);
      }
    }
  }
}

// r -= D^-1 A d_in; d_out = c1 d_in + c2 r; x += d_out; part (if set): b . x per case
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) kb_cheb_step(int64_t n_rows, const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                         int64_t stride, const T* __restrict__ dinv,
                                                         const T* __restrict__ d_in, T* __restrict__ d_out,
                                                         T* __restrict__ r, T* __restrict__ x, T c1, T c2,
                                                         const T* __restrict__ b, double* __restrict__ part,
                                                         const int* __restrict__ done) {
  if (*done) return;
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_ROW_LOOP(n_rows) {
      T acc[BS][4];
      batch_block_row<BS, BS, BLayout<BS>::value>(rp, ci, av, stride, row, c0, BLoad<T>{d_in}, acc);
#pragma unroll
      for (int rr = 0; rr < BS; ++rr) {
        const int64_t i = row * BS + rr;
        const int64_t o = i * kBatch + c0;
        const T di = dinv[i];
        const C4<T> rv = ld4(r + o), dv = ld4(d_in + o), xv = ld4(x + o);
        C4<T> ro, dn, xn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          ro.v[k] = rv.v[k] - di * acc[rr][k];
          dn.v[k] = c1 * dv.v[k] + c2 * ro.v[k];
          xn.v[k] = xv.v[k] + dn.v[k];
        }
        st4(r + o, ro);
        st4(d_out + o, dn);
        st4(x + o, xn);
        if (part) {
          const C4<T> bv = ld4(b + o);
#pragma unroll
          for (int k = 0; k < 4; ++k) dot[k] += (double)bv.v[k] * (double)xn.v[k];
        }
      }
    }
  }
  if (part) write_case_parts(dot, part);
}

// res = b - A x
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) kb_residual(int64_t n_rows, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                        int64_t stride, const T* __restrict__ b,
                                                        const T* __restrict__ x, T* __restrict__ res,
                                                        const int* __restrict__ done) {
  if (*done) return;
  BATCH_ROW_LOOP(n_rows) {
    T acc[BS][4];
    batch_block_row<BS, BS, BLayout<BS>::value>(rp, ci, av, stride, row, c0, BLoad<T>{x}, acc);
#pragma unroll
    for (int rr = 0; rr < BS; ++rr) {
      const int64_t o = (row * BS + rr) * kBatch + c0;
      const C4<T> bv = ld4(b + o);
      C4<T> ro;
#pragma unroll
      for (int k = 0; k < 4; ++k) ro.v[k] = bv.v[k] - acc[rr][k];
      st4(res + o, ro);
    }
  }
}

// first post-smoothing step from x: r0 = D^-1 (b - A x), d0 = r0 / theta, x2 = x + d0
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) kb_post_first(int64_t n_rows, const int32_t* __restrict__ rp,
                                                          const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                          int64_t stride, const T* __restrict__ b,
                                                          const T* __restrict__ dinv, T inv_theta,
                                                          const T* __restrict__ x, T* __restrict__ x2,
                                                          T* __restrict__ r, T* __restrict__ d,
                                                          double* __restrict__ part, const int* __restrict__ done) {
  if (*done) return;
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_ROW_LOOP(n_rows) {
      T acc[BS][4];
      batch_block_row<BS, BS, BLayout<BS>::value>(rp, ci, av, stride, row, c0, BLoad<T>{x}, acc);
#pragma unroll
      for (int rr = 0; rr < BS; ++rr) {
        const int64_t i = row * BS + rr;
        const int64_t o = i * kBatch + c0;
        const T di = dinv[i];
        const C4<T> bv = ld4(b + o), xv = ld4(x + o);
        C4<T> ro, dd, xn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          ro.v[k] = di * (bv.v[k] - acc[rr][k]);
          dd.v[k] = ro.v[k] * inv_theta;
          xn.v[k] = xv.v[k] + dd.v[k];
          if (part) dot[k] += (double)bv.v[k] * (double)xn.v[k];
        }
        st4(r + o, ro);
        st4(d + o, dd);
        st4(x2 + o, xn);
      }
    }
  }
  if (part) write_case_parts(dot, part);
}

// y = A x or y += A x for the block-contiguous transfer operators (BR x BC blocks)
template <int BR, int BC, typename T>
__global__ void __launch_bounds__(kThreads) kb_level_spmv(int64_t n_rows, const int32_t* __restrict__ rp,
                                                          const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                          const T* __restrict__ x, T* __restrict__ y, int accumulate,
                                                          const int* __restrict__ done) {
  if (*done) return;
  BATCH_ROW_LOOP(n_rows) {
    T acc[BR][4];
    batch_block_row<BR, BC, kAoS>(rp, ci, av, 0, row, c0, BLoad<T>{x}, acc);
#pragma unroll
    for (int rr = 0; rr < BR; ++rr) {
      const int64_t o = (row * BR + rr) * kBatch + c0;
      C4<T> v;
#pragma unroll
      for (int k = 0; k < 4; ++k) v.v[k] = acc[rr][k];
      if (accumulate) {
        const C4<T> yv = ld4(y + o);
#pragma unroll
        for (int k = 0; k < 4; ++k) v.v[k] += yv.v[k];
      }
      st4(y + o, v);
    }
  }
}

// coarsest level: X = A_c^-1 B with the dense FP64 inverse; one warp per row, lane = case
template <typename T>
__global__ void __launch_bounds__(kThreads) kb_coarse(int64_t n, const double* __restrict__ inv,
                                                      const T* __restrict__ b, T* __restrict__ x,
                                                      const int* __restrict__ done) {
  if (*done) return;
  const int lane = threadIdx.x & 31;
  const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp0; row < n; row += nwarps) {
    const double* __restrict__ rowp = inv + row * n;
    double s = 0.0;
    for (int64_t j = 0; j < n; ++j) s += rowp[j] * (double)b[j * kBatch + lane];
    x[row * kBatch + lane] = (T)s;
  }
}

// ---------------------------------------------------------------------------------------
// batched PCG kernels
// ---------------------------------------------------------------------------------------

// r = b, x = 0, rm = (TM) b (if rm), partC = b . b per case
template <typename TM>
__global__ void __launch_bounds__(kThreads) kb_init_vecs(int64_t n, const double* __restrict__ b,
                                                         double* __restrict__ x, double* __restrict__ r,
                                                         TM* __restrict__ rm, double* __restrict__ partC) {
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_QUAD_LOOP(n) {
      const C4<double> v = ld4(b + 4 * t);
      st4(r + 4 * t, v);
      st4(x + 4 * t, C4<double>{{0.0, 0.0, 0.0, 0.0}});
      if (rm) st4(rm + 4 * t, cvt4<TM>(v));
#pragma unroll
      for (int k = 0; k < 4; ++k) dot[k] += v.v[k] * v.v[k];
    }
    (void)c0;
  }
  write_case_parts(dot, partC);
}

// per-case targets; cases with rtol_j >= 1 (already converged outside) or a zero right-hand
// side start finished
__global__ void kb_init_scalars(BlockScalars* S, const double* __restrict__ partC, int nparts,
                                const double* __restrict__ rtol, int max_iter) {
  const double bb = reduce_case_parts(partC, nparts);
  __shared__ int sdone[kBatch];
  if (threadIdx.x < kBatch) {
    const int j = threadIdx.x;
    const bool finite = isfinite(bb);
    S->bnorm2[j] = bb;
    S->tol2[j] = rtol[j] * rtol[j] * bb;
    S->rr[j] = bb;
    S->rz[j] = 0.0;
    S->alpha[j] = 0.0;
    S->beta[j] = 0.0;
    S->col_iters[j] = 0;
    S->col_status[j] = finite ? 0 : WN_EBREAKDOWN;
    const int d = (bb == 0.0 || !finite || rtol[j] >= 1.0) ? 1 : 0;
    S->col_done[j] = d;
    sdone[j] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int all = 1;
    for (int j = 0; j < kBatch; ++j) all &= sdone[j];
    S->done = all;
    S->iters = 0;
    S->status = 0;
    S->max_iter = max_iter;
  }
}

// z = D^-1 r (jacobi) or z = r; partA = r . z per case
template <typename T>
__global__ void __launch_bounds__(kThreads) kb_prec_vec(int64_t n, const T* __restrict__ r,
                                                        const T* __restrict__ dinv, int jacobi, T* __restrict__ z,
                                                        double* __restrict__ partA, const int* __restrict__ done) {
  if (*done) return;
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_QUAD_LOOP(n) {
      const C4<T> rv = ld4(r + 4 * t);
      const T di = jacobi ? dinv[(4 * t) / kBatch] : T(1);
      C4<T> zv;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        zv.v[k] = jacobi ? di * rv.v[k] : rv.v[k];
        dot[k] += (double)rv.v[k] * (double)zv.v[k];
      }
      st4(z + 4 * t, zv);
    }
    (void)c0;
  }
  write_case_parts(dot, partA);
}

// rz_new = r . z (partA); beta = rz_new / rz (0 at the first iteration and for finished cases)
__global__ void kb_beta(BlockScalars* S, const double* __restrict__ partA, int nparts, int first) {
  if (S->done) return;
  const double rz_new = reduce_case_parts(partA, nparts);
  __shared__ int sdone[kBatch];
  if (threadIdx.x < kBatch) {
    const int j = threadIdx.x;
    int d = S->col_done[j];
    double beta = 0.0;
    if (!d) {
      if (!isfinite(rz_new)) {
        S->col_status[j] = WN_EBREAKDOWN;
        d = 1;
      } else if (!first) {
        const double rz = S->rz[j];
        beta = rz != 0.0 ? rz_new / rz : 0.0;
      }
    }
    S->rz[j] = rz_new;
    S->beta[j] = d ? 0.0 : beta;
    S->col_done[j] = d;
    sdone[j] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int all = 1;
    for (int j = 0; j < kBatch; ++j) all &= sdone[j];
    S->done = all;
  }
}

// p_new = z + beta p_old; q = A p_new (fine matrix, component-major FP64); partB = p_new . q
template <typename TM>
__global__ void __launch_bounds__(kThreads) kb_spmv_dot(int64_t n_rows, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const double* __restrict__ av,
                                                        int64_t stride, const TM* __restrict__ z,
                                                        const double* __restrict__ p_old, double* __restrict__ p_new,
                                                        double* __restrict__ q, double* __restrict__ partB,
                                                        const BlockScalars* __restrict__ S) {
  if (S->done) return;
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_ROW_LOOP(n_rows) {
      const C4<double> beta = {{S->beta[c0], S->beta[c0 + 1], S->beta[c0 + 2], S->beta[c0 + 3]}};
      const BPNew<double, TM> pf{z, p_old, beta};
      double acc[3][4];
      batch_block_row<3, 3, kSoA>(rp, ci, av, stride, row, c0, pf, acc);
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        const int64_t i = row * 3 + rr;
        const int64_t o = i * kBatch + c0;
        const C4<double> pv = pf(i, c0);
        C4<double> qv;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          qv.v[k] = acc[rr][k];
          dot[k] += pv.v[k] * qv.v[k];
        }
        st4(p_new + o, pv);
        st4(q + o, qv);
      }
    }
  }
  write_case_parts(dot, partB);
}

// alpha = rz / (p . q) for the running cases; a non-positive curvature ends that case
__global__ void kb_alpha(BlockScalars* S, const double* __restrict__ partB, int nparts) {
  if (S->done) return;
  const double gamma = reduce_case_parts(partB, nparts);
  if (threadIdx.x < kBatch) {
    const int j = threadIdx.x;
    double alpha = 0.0;
    if (!S->col_done[j]) {
      alpha = S->rz[j] / gamma;
      if (!(gamma > 0.0) || !isfinite(alpha)) {
        S->col_status[j] = WN_EBREAKDOWN;
        S->col_done[j] = 1;
        alpha = 0.0;
      }
    }
    S->alpha[j] = alpha;
  }
}

// x += alpha p; r -= alpha q; rm = (TM) r (if rm); partC = r . r per case
template <typename TM>
__global__ void __launch_bounds__(kThreads) kb_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                      TM* __restrict__ rm, const double* __restrict__ p,
                                                      const double* __restrict__ q, double* __restrict__ partC,
                                                      const BlockScalars* __restrict__ S) {
  if (S->done) return;
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_QUAD_LOOP(n) {
      const double a0 = S->alpha[c0], a1 = S->alpha[c0 + 1], a2 = S->alpha[c0 + 2], a3 = S->alpha[c0 + 3];
      const double a[4] = {a0, a1, a2, a3};
      C4<double> xv = ld4(x + 4 * t), rv = ld4(r + 4 * t);
      const C4<double> pv = ld4(p + 4 * t), qv = ld4(q + 4 * t);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (a[k] != 0.0) {  // finished cases keep x and r exactly (their p may be anything)
          xv.v[k] += a[k] * pv.v[k];
          rv.v[k] -= a[k] * qv.v[k];
        }
        dot[k] += rv.v[k] * rv.v[k];
      }
      st4(x + 4 * t, xv);
      st4(r + 4 * t, rv);
      if (rm) st4(rm + 4 * t, cvt4<TM>(rv));
    }
  }
  write_case_parts(dot, partC);
}

// convergence test of every running case; the batch ends when all cases are finished or
// the iteration limit is reached (the unfinished cases then report WN_ENOCONV)
__global__ void kb_check(BlockScalars* S, const double* __restrict__ partC, int nparts) {
  if (S->done) return;
  const double rr = reduce_case_parts(partC, nparts);
  __shared__ int sdone[kBatch];
  const int it = S->iters + 1;
  if (threadIdx.x < kBatch) {
    const int j = threadIdx.x;
    int d = S->col_done[j];
    if (!d) {
      S->rr[j] = rr;
      S->col_iters[j] += 1;
      if (!isfinite(rr)) {
        S->col_status[j] = WN_EBREAKDOWN;
        d = 1;
      } else if (rr <= S->tol2[j]) {
        d = 1;
      } else if (it >= S->max_iter) {
        S->col_status[j] = WN_ENOCONV;
      }
    }
    S->col_done[j] = d;
    sdone[j] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int all = 1;
    for (int j = 0; j < kBatch; ++j) all &= sdone[j];
    S->iters = it;
    if (!all && it >= S->max_iter) {
      S->status = WN_ENOCONV;
      all = 1;
    }
    S->done = all;
  }
}

// R = F - K U (FP64, component-major fine matrix); partC = R . R per case
__global__ void __launch_bounds__(kThreads) kb_outer_residual(int64_t n_rows, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci,
                                                              const double* __restrict__ av, int64_t stride,
                                                              const double* __restrict__ F,
                                                              const double* __restrict__ U, double* __restrict__ R,
                                                              double* __restrict__ partC) {
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_ROW_LOOP(n_rows) {
      double acc[3][4];
      batch_block_row<3, 3, kSoA>(rp, ci, av, stride, row, c0, BLoad<double>{U}, acc);
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        const int64_t o = (row * 3 + rr) * kBatch + c0;
        const C4<double> fv = ld4(F + o);
        C4<double> rv;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          rv.v[k] = fv.v[k] - acc[rr][k];
          dot[k] += rv.v[k] * rv.v[k];
        }
        st4(R + o, rv);
      }
    }
  }
  write_case_parts(dot, partC);
}

// partC = x . x per case
__global__ void __launch_bounds__(kThreads) kb_dot_self(int64_t n, const double* __restrict__ x,
                                                        double* __restrict__ partC) {
  double dot[4] = {0.0, 0.0, 0.0, 0.0};
  {
    BATCH_QUAD_LOOP(n) {
      const C4<double> v = ld4(x + 4 * t);
#pragma unroll
      for (int k = 0; k < 4; ++k) dot[k] += v.v[k] * v.v[k];
    }
    (void)c0;
  }
  write_case_parts(dot, partC);
}

// S->rr[j] = sum of partC (one CTA)
__global__ void kb_reduce_rr(BlockScalars* S, const double* __restrict__ partC, int nparts) {
  const double rr = reduce_case_parts(partC, nparts);
  if (threadIdx.x < kBatch) S->rr[threadIdx.x] = rr;
}

// U += X
__global__ void kb_accumulate(int64_t n, double* __restrict__ U, const double* __restrict__ X) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * kBatch;
       i += (int64_t)gridDim.x * blockDim.x)
    U[i] += X[i];
}

// pack columns [j0, j0 + m) of a row-major n x ld matrix into the n x kBatch batch (zero
// padding), and back
__global__ void kb_pack(int64_t n, const double* __restrict__ src, int64_t ld, int64_t j0, int m,
                        double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * kBatch;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / kBatch;
    const int j = (int)(i - row * kBatch);
    dst[i] = j < m ? src[row * ld + j0 + j] : 0.0;
  }
}
__global__ void kb_unpack(int64_t n, const double* __restrict__ src, int64_t ld, int64_t j0, int m,
                          double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * kBatch;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / kBatch;
    const int j = (int)(i - row * kBatch);
    if (j < m) dst[row * ld + j0 + j] = src[i];
  }
}

// 1 / diag of the fine matrix (component-major values), the rule of solid_solver.py:230
__global__ void kb_fill_dinv(int64_t n_rows, int64_t nnzb, const int32_t* __restrict__ diag_block,
                             const double* __restrict__ k64, double* __restrict__ d64, float* __restrict__ d32) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_rows * 3;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = t / 3;
    const int c = (int)(t - row * 3);
    const double dv = k64[(int64_t)(c * 4) * nnzb + diag_block[row]];
    const double inv = (fabs(dv) > 1e-12) ? 1.0 / dv : 1.0;
    d64[t] = inv;
    d32[t] = (float)inv;
  }
}

// ---------------------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------------------
inline int rows_work(int64_t n_rows) { return (int)((n_rows * (32 / kRowsPerWarp) + kThreads - 1) / kThreads); }
inline int quads_work(int64_t n) { return (int)((n * (kBatch / 4) + kThreads - 1) / kThreads); }

template <typename T>
struct BPrec;
template <>
struct BPrec<float> {
  static const float* A0(Solid* s) { return s->k32.p; }
  static const float* Av(DevLevel& L) { return L.A.v32.p; }
  static const float* Pv(DevLevel& L) { return L.P.v32.p; }
  static const float* Rv(DevLevel& L) { return L.R.v32.p; }
  static const float* dinv(DevLevel& L) { return L.dinv32.p; }
  static BatchLevelVecs<float>& lv(BlockWork& W, int l) { return W.lv32[l]; }
  static float* cb(BlockWork& W) { return W.cb32.p; }
  static float* cx(BlockWork& W) { return W.cx32.p; }
  static const float* fine_dinv(BlockWork& W) { return W.dinv32.p; }
  static float* z(BlockWork& W) { return W.z32.p; }
  static float* rm(BlockWork& W) { return W.r32.p; }  // r in FP32 for the V-cycle
};
template <>
struct BPrec<double> {
  static const double* A0(Solid* s) { return s->k64.p; }
  static const double* Av(DevLevel& L) { return L.A.v64.p; }
  static const double* Pv(DevLevel& L) { return L.P.v64.p; }
  static const double* Rv(DevLevel& L) { return L.R.v64.p; }
  static const double* dinv(DevLevel& L) { return L.dinv64.p; }
  static BatchLevelVecs<double>& lv(BlockWork& W, int l) { return W.lv64[l]; }
  static double* cb(BlockWork& W) { return W.cb64.p; }
  static double* cx(BlockWork& W) { return W.cx64.p; }
  static const double* fine_dinv(BlockWork& W) { return W.dinv64.p; }
  static double* z(BlockWork& W) { return W.z64.p; }
  static double* rm(BlockWork&) { return nullptr; }  // the V-cycle reads the FP64 r directly
};

template <int BR, int BC, typename T>
void batch_level_spmv(const DevBsr& M, const T* vals, const T* x, T* y, int accumulate, const int* done,
                      cudaStream_t st) {
  auto k = kb_level_spmv<BR, BC, T>;
  k<<<resident_grid(k, kThreads, rows_work(M.n_rows)), kThreads, 0, st>>>(M.n_rows, M.rp.p, M.ci.p, vals, x, y,
                                                                          accumulate, done);
}

// one batched V-cycle at level lvl: out = V(b); part (if set) receives b . out per case
template <typename T>
int batch_vcycle(Solid* s, AmgHierarchy& H, BlockWork& W, int lvl, const T* b, T* out, double* part,
                 const int* done, cudaStream_t st) {
  const int nlev = (int)H.levels.size();
  if (lvl == nlev) {
    kb_coarse<T><<<resident_grid(kb_coarse<T>, kThreads, (H.n_coarse * 32 + kThreads - 1) / kThreads), kThreads, 0,
                   st>>>(H.n_coarse, H.coarse_inv.p, b, out, done);
    W.launches++;
    return 0;
  }
  DevLevel& L = H.levels[lvl];
  BatchLevelVecs<T>& V = BPrec<T>::lv(W, lvl);
  const int64_t nr = L.n_nodes;
  const T* dinv = (lvl == 0) ? BPrec<T>::fine_dinv(W) : BPrec<T>::dinv(L);
  const int deg = H.degree;
  const T it = (T)L.inv_theta;
  const int64_t sd = (lvl == 0) ? s->nnzb : 0;
  const int work = rows_work(nr);
  auto run = [&](auto bs_tag) -> int {
    constexpr int BS = decltype(bs_tag)::value;
    auto rg = [&](auto kern) { return resident_grid(kern, kThreads, work); };
    const int32_t* rp = lvl == 0 ? s->row_ptr.p : L.A.rp.p;
    const int32_t* ci = lvl == 0 ? s->col_idx.p : L.A.ci.p;
    const T* av = lvl == 0 ? BPrec<T>::A0(s) : BPrec<T>::Av(L);
    const T c1 = deg >= 2 ? (T)L.c1[0] : T(0), c2 = deg >= 2 ? (T)L.c2[0] : T(0);
    kb_pre_first<BS, T><<<rg(kb_pre_first<BS, T>), kThreads, 0, st>>>(nr, rp, ci, av, sd, b, dinv, it, deg, c1, c2,
                                                                      V.x.p, V.r.p, V.d.p, V.res.p, done);
    W.launches++;
    T* din = V.d.p;
    T* dout = V.d2.p;
    for (int k = 2; k < deg; ++k) {
      kb_cheb_step<BS, T><<<rg(kb_cheb_step<BS, T>), kThreads, 0, st>>>(nr, rp, ci, av, sd, dinv, din, dout, V.r.p,
                                                                        V.x.p, (T)L.c1[k - 1], (T)L.c2[k - 1], b,
                                                                        nullptr, done);
      W.launches++;
      std::swap(din, dout);
    }
    if (deg >= 2) {
      kb_residual<BS, T><<<rg(kb_residual<BS, T>), kThreads, 0, st>>>(nr, rp, ci, av, sd, b, V.x.p, V.res.p, done);
      W.launches++;
    }
    const bool last = lvl + 1 >= nlev;
    T* bc = last ? BPrec<T>::cb(W) : BPrec<T>::lv(W, lvl + 1).b.p;
    T* xc = last ? BPrec<T>::cx(W) : BPrec<T>::lv(W, lvl + 1).x2.p;
    batch_level_spmv<6, BS, T>(L.R, BPrec<T>::Rv(L), V.res.p, bc, 0, done, st);
    W.launches++;
    WN_CHECK(batch_vcycle<T>(s, H, W, lvl + 1, bc, xc, nullptr, done, st));
    batch_level_spmv<BS, 6, T>(L.P, BPrec<T>::Pv(L), xc, V.x.p, 1, done, st);
    W.launches++;
    double* part_last = (deg == 1) ? part : nullptr;
    const int gpf = rg(kb_post_first<BS, T>);
    if (part_last) W.npA = gpf;
    kb_post_first<BS, T><<<gpf, kThreads, 0, st>>>(nr, rp, ci, av, sd, b, dinv, it, V.x.p, out, V.r.p, V.d.p,
                                                   part_last, done);
    W.launches++;
    din = V.d.p;
    dout = V.d2.p;
    for (int k = 1; k < deg; ++k) {
      double* pk = (k == deg - 1) ? part : nullptr;
      const int gcs = rg(kb_cheb_step<BS, T>);
      if (pk) W.npA = gcs;
      kb_cheb_step<BS, T><<<gcs, kThreads, 0, st>>>(nr, rp, ci, av, sd, dinv, din, dout, V.r.p, out,
                                                    (T)L.c1[k - 1], (T)L.c2[k - 1], b, pk, done);
      W.launches++;
      std::swap(din, dout);
    }
    return 0;
  };
  WN_CHECK(L.bs == 3 ? run(std::integral_constant<int, 3>{}) : run(std::integral_constant<int, 6>{}));
  WN_CUDA(cudaGetLastError());
  return 0;
}

// z = M r for all cases, partA = r . z per case
template <typename TM>
int batch_prec(Solid* s, BlockWork& W, int precond, const TM* r, TM* z, const int* done, cudaStream_t st) {
  if (precond == 2) return batch_vcycle<TM>(s, *s->amg, W, 0, r, z, W.partA.p, done, st);
  const int g = resident_grid(kb_prec_vec<TM>, kThreads, quads_work(W.n));
  W.npA = g;
  kb_prec_vec<TM><<<g, kThreads, 0, st>>>(W.n, r, BPrec<TM>::fine_dinv(W), precond == 1 ? 1 : 0, z, W.partA.p,
                                          done);
  W.launches++;
  WN_CUDA(cudaGetLastError());
  return 0;
}

template <typename TM>
const TM* prec_input(BlockWork& W) {
  if constexpr (std::is_same<TM, double>::value)
    return W.r.p;
  else
    return W.r32.p;
}

// one batched PCG iteration (parity k & 1 selects the p buffers)
template <typename TM>
int batch_iteration(Solid* s, BlockWork& W, int precond, int k, BlockScalars* S, cudaStream_t st) {
  const int par = k & 1;
  double* p_new = par ? W.p1.p : W.p0.p;
  double* p_old = par ? W.p0.p : W.p1.p;
  const int gsd = resident_grid(kb_spmv_dot<TM>, kThreads, rows_work(s->n_nodes));
  kb_spmv_dot<TM><<<gsd, kThreads, 0, st>>>(s->n_nodes, s->row_ptr.p, s->col_idx.p, s->k64.p, s->nnzb,
                                            BPrec<TM>::z(W), p_old, p_new, W.q.p, W.partB.p, S);
  W.npB = gsd;
  kb_alpha<<<1, kThreads, 0, st>>>(S, W.partB.p, W.npB);
  const int gup = resident_grid(kb_update<TM>, kThreads, quads_work(W.n));
  kb_update<TM><<<gup, kThreads, 0, st>>>(W.n, W.x.p, W.r.p, BPrec<TM>::rm(W), p_new, W.q.p, W.partC.p, S);
  W.npC = gup;
  kb_check<<<1, kThreads, 0, st>>>(S, W.partC.p, W.npC);
  W.launches += 4;
  WN_CUDA(cudaGetLastError());
  WN_CHECK(batch_prec<TM>(s, W, precond, prec_input<TM>(W), BPrec<TM>::z(W), &S->done, st));
  kb_beta<<<1, kThreads, 0, st>>>(S, W.partA.p, W.npA, 0);
  W.launches++;
  WN_CUDA(cudaGetLastError());
  return 0;
}

// batched PCG on b (n x kBatch) from x = 0 with the per-case targets in W.rtol_cols
template <typename TM>
int batch_pcg(Solid* s, BlockWork& W, int vmode, const double* b, int max_iter, int precond, int chunk,
              int use_graph, BlockScalars* S, cudaStream_t st, BlockScalars* hS) {
  const size_t vb = (size_t)W.n * kBatch * sizeof(double);
  WN_CUDA(cudaMemsetAsync(W.p0.p, 0, vb, st));  // first iteration: p = z + 0 * p_old
  WN_CUDA(cudaMemsetAsync(W.p1.p, 0, vb, st));
  W.npC = resident_grid(kb_init_vecs<TM>, kThreads, quads_work(W.n));
  kb_init_vecs<TM><<<W.npC, kThreads, 0, st>>>(W.n, b, W.x.p, W.r.p, BPrec<TM>::rm(W), W.partC.p);
  kb_init_scalars<<<1, kThreads, 0, st>>>(S, W.partC.p, W.npC, W.rtol_cols.p, max_iter);
  W.launches += 2;
  WN_CUDA(cudaGetLastError());
  WN_CHECK(batch_prec<TM>(s, W, precond, prec_input<TM>(W), BPrec<TM>::z(W), &S->done, st));
  kb_beta<<<1, kThreads, 0, st>>>(S, W.partA.p, W.npA, 1);
  W.launches++;
  chunk = std::max(2, chunk + (chunk & 1));  // even: the parity pattern repeats per chunk
  GraphCache& G = W.graphs[vmode][precond];
  const int64_t key = chunk;
  int k0 = 0;
  while (true) {
    WN_CUDA(cudaMemcpyAsync(hS, S, sizeof(BlockScalars), cudaMemcpyDeviceToHost, st));
    WN_CUDA(cudaStreamSynchronize(st));
    if (hS->done || k0 >= max_iter) break;
    if (use_graph) {
      if (G.key != key || G.stream != st || !G.exec) {
        G.reset();
        cudaGraph_t graph;
        const int64_t before = W.launches;
        WN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = 0;
        for (int k = 0; k < chunk && rc == 0; ++k) rc = batch_iteration<TM>(s, W, precond, k, S, st);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        WN_CHECK(rc);
        WN_CUDA(e);
        e = cudaGraphInstantiate(&G.exec, graph, 0);
        cudaGraphDestroy(graph);
        WN_CUDA(e);
        G.key = key;
        G.stream = st;
        G.kernels = W.launches - before;
        W.launches = before;
      }
      WN_CUDA(cudaGraphLaunch(G.exec, st));
      W.launches += G.kernels;
    } else {
      for (int k = 0; k < chunk; ++k) WN_CHECK(batch_iteration<TM>(s, W, precond, k0 + k, S, st));
    }
    k0 += chunk;
  }
  return 0;
}

int ensure_block_work(Solid* s, int vmode, int precond) {
  if (!s->bwork) s->bwork.reset(new BlockWork());
  BlockWork& W = *s->bwork;
  const int64_t n = s->n_nodes * 3;
  const int64_t nb = n * kBatch;
  if (W.n != n) {
    W.n = n;
    WN_CHECK(W.F.alloc(nb));
    WN_CHECK(W.U.alloc(nb));
    WN_CHECK(W.R.alloc(nb));
    WN_CHECK(W.x.alloc(nb));
    WN_CHECK(W.r.alloc(nb));
    WN_CHECK(W.p0.alloc(nb));
    WN_CHECK(W.p1.alloc(nb));
    WN_CHECK(W.q.alloc(nb));
    WN_CHECK(W.dinv64.alloc(n));
    WN_CHECK(W.dinv32.alloc(n));
    for (auto& a : W.graphs)
      for (auto& g : a) g.reset();
  }
  if (vmode == 1) {
    WN_CHECK(W.z32.alloc(nb));
    WN_CHECK(W.r32.alloc(nb));
  } else {
    WN_CHECK(W.z64.alloc(nb));
  }
  WN_CHECK(W.partA.alloc((int64_t)BlockWork::kMaxParts * kBatch));
  WN_CHECK(W.partB.alloc((int64_t)BlockWork::kMaxParts * kBatch));
  WN_CHECK(W.partC.alloc((int64_t)BlockWork::kMaxParts * kBatch));
  WN_CHECK(W.scal.alloc(2));
  WN_CHECK(W.rtol_cols.alloc(kBatch));
  W.h_rtol.assign(kBatch, 1.0);
  if (precond == 2) {
    AmgHierarchy& H = *s->amg;
    if (W.hierarchy_id != H.id) {
      W.lv32.clear();
      W.lv64.clear();
      W.cb32.release();
      W.cx32.release();
      W.cb64.release();
      W.cx64.release();
      W.hierarchy_id = H.id;
      for (auto& a : W.graphs)
        for (auto& g : a) g.reset();
    }
    const size_t nl = H.levels.size();
    if (vmode == 1 && W.lv32.size() != nl) {
      W.lv32.resize(nl);
      for (size_t l = 0; l < nl; ++l) WN_CHECK(W.lv32[l].alloc(H.levels[l].n_nodes * H.levels[l].bs * kBatch));
      WN_CHECK(W.cb32.alloc(H.n_coarse * kBatch));
      WN_CHECK(W.cx32.alloc(H.n_coarse * kBatch));
    }
    if (vmode == 0 && W.lv64.size() != nl) {
      W.lv64.resize(nl);
      for (size_t l = 0; l < nl; ++l) WN_CHECK(W.lv64[l].alloc(H.levels[l].n_nodes * H.levels[l].bs * kBatch));
      WN_CHECK(W.cb64.alloc(H.n_coarse * kBatch));
      WN_CHECK(W.cx64.alloc(H.n_coarse * kBatch));
    }
  }
  if (!W.ev0) {
    WN_CUDA(cudaEventCreate(&W.ev0));
    WN_CUDA(cudaEventCreate(&W.ev1));
  }
  return 0;
}

// per-case norms of an n x kBatch FP64 vector into host rr[]
int case_norms2(BlockWork& W, const double* v, BlockScalars* S1, cudaStream_t st, BlockScalars* hS) {
  W.npC = resident_grid(kb_dot_self, kThreads, quads_work(W.n));
  kb_dot_self<<<W.npC, kThreads, 0, st>>>(W.n, v, W.partC.p);
  kb_reduce_rr<<<1, kThreads, 0, st>>>(S1, W.partC.p, W.npC);
  W.launches += 2;
  WN_CUDA(cudaGetLastError());
  WN_CUDA(cudaMemcpyAsync(hS, S1, sizeof(BlockScalars), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  return 0;
}

struct BatchResult {
  int iterations = 0, outer = 0, status = 0;
  int case_iters[kBatch] = {};
  int case_status[kBatch] = {};
  double case_rel[kBatch] = {};
};

// FP64 refinement over the batch in W.F (m live cases): U = 0, R = F; while some case has
// ||R_j|| > rtol ||F_j||: batched PCG on R with per-case inner targets, U += X, R = F - K U.
template <typename TM>
int batch_outer(Solid* s, BlockWork& W, int vmode, int m, const wn_solve_params& prm, int chunk, cudaStream_t st,
                BatchResult& res) {
  const int64_t n = W.n;
  const size_t vb = (size_t)n * kBatch * sizeof(double);
  BlockScalars* S = W.scal.p;
  BlockScalars* S1 = W.scal.p + 1;
  BlockScalars hS{};
  WN_CHECK(case_norms2(W, W.F.p, S1, st, &hS));
  double fnorm[kBatch], rr[kBatch];
  for (int j = 0; j < kBatch; ++j) {
    fnorm[j] = std::sqrt(hS.rr[j]);
    rr[j] = hS.rr[j];
  }
  WN_CUDA(cudaMemsetAsync(W.U.p, 0, vb, st));
  WN_CUDA(cudaMemcpyAsync(W.R.p, W.F.p, vb, cudaMemcpyDeviceToDevice, st));
  const int max_outer = prm.max_outer > 0 ? prm.max_outer : 10;
  bool first = true;
  while (true) {
    if (!first) {
      W.npC = resident_grid(kb_outer_residual, kThreads, rows_work(s->n_nodes));
      kb_outer_residual<<<W.npC, kThreads, 0, st>>>(s->n_nodes, s->row_ptr.p, s->col_idx.p, s->k64.p, s->nnzb,
                                                    W.F.p, W.U.p, W.R.p, W.partC.p);
      kb_reduce_rr<<<1, kThreads, 0, st>>>(S1, W.partC.p, W.npC);
      W.launches += 2;
      WN_CUDA(cudaGetLastError());
      WN_CUDA(cudaMemcpyAsync(&hS, S1, sizeof(BlockScalars), cudaMemcpyDeviceToHost, st));
      WN_CUDA(cudaStreamSynchronize(st));
      for (int j = 0; j < kBatch; ++j) rr[j] = hS.rr[j];
    }
    first = false;
    bool all = true;
    for (int j = 0; j < kBatch; ++j) {
      double t = 1.0;  // 1 = case finished (or padding)
      if (j < m) {
        const double rn = std::sqrt(rr[j]);
        if (!std::isfinite(fnorm[j]) || !std::isfinite(rr[j])) {
          res.case_status[j] = WN_EBREAKDOWN;  // corrupt load case or diverged: not iterated on
        } else if (fnorm[j] > 0.0 && res.case_status[j] != WN_EBREAKDOWN && rn > prm.rtol * fnorm[j]) {
          t = std::min(0.5, 0.5 * prm.rtol * fnorm[j] / rn);
          all = false;
        }
      }
      W.h_rtol[j] = t;
    }
    if (all) break;
    if (res.outer >= max_outer || res.iterations >= prm.max_iter) {
      res.status = WN_ENOCONV;
      break;
    }
    WN_CUDA(cudaMemcpyAsync(W.rtol_cols.p, W.h_rtol.data(), kBatch * sizeof(double), cudaMemcpyHostToDevice, st));
    WN_CHECK((batch_pcg<TM>(s, W, vmode, W.R.p, prm.max_iter - res.iterations, prm.precond, chunk, prm.use_graph, S,
                            st, &hS)));
    res.iterations += hS.iters;
    ++res.outer;
    for (int j = 0; j < m; ++j) {
      res.case_iters[j] += hS.col_iters[j];
      if (hS.col_status[j] == WN_EBREAKDOWN) res.case_status[j] = WN_EBREAKDOWN;
    }
    kb_accumulate<<<grid_for(n * kBatch, 1, kThreads, 8), kThreads, 0, st>>>(n, W.U.p, W.x.p);
    W.launches++;
    WN_CUDA(cudaGetLastError());
  }
  for (int j = 0; j < m; ++j) {
    res.case_rel[j] = fnorm[j] > 0.0 ? std::sqrt(rr[j]) / fnorm[j] : 0.0;
    const bool ok = res.case_rel[j] <= prm.rtol;
    if (res.case_status[j] == 0 && !ok) res.case_status[j] = WN_ENOCONV;
    if (res.case_status[j] == WN_EBREAKDOWN) res.status = WN_EBREAKDOWN;
    else if (res.case_status[j] == WN_ENOCONV && res.status == 0) res.status = WN_ENOCONV;
  }
  return 0;
}

}  // namespace

int solver_solve_multi(Solid* s, int n_rhs, const double* F, double* U, const wn_solve_params& prm,
                       wn_solve_stats* stats, int* case_iters, double* case_rel, cudaStream_t st) {
  WN_REQUIRE(s->assembled, WN_ESTATE, "multi-RHS solve: matrix not assembled");
  WN_REQUIRE(n_rhs >= 0, WN_EINVAL, "multi-RHS solve: n_rhs >= 0 required");
  WN_REQUIRE(prm.precond >= 0 && prm.precond <= 2, WN_EINVAL, "multi-RHS solve: precond in {0, 1, 2}");
  WN_REQUIRE(prm.precision == 0 || prm.precision == 1, WN_EINVAL,
             "multi-RHS solve: precision must be 0 (fp64) or 1 (fp32 V-cycle in fp64 PCG)");
  WN_REQUIRE(prm.max_iter > 0 && prm.rtol > 0.0, WN_EINVAL, "multi-RHS solve: max_iter > 0 and rtol > 0 required");
  if (prm.precond == 2 && !s->amg) WN_CHECK(solver_setup(s, amg_default_params()));
  const int vmode = prm.precision == 1 ? 1 : 0;
  WN_CHECK(ensure_block_work(s, vmode, prm.precond));
  BlockWork& W = *s->bwork;
  W.launches = 0;
  if (st == 0) {
    if (!W.own) WN_CUDA(cudaStreamCreate(&W.own));
    st = W.own;
  }
  const int64_t n = W.n;
  const int chunk = prm.chunk > 0 ? prm.chunk : 8;
  kb_fill_dinv<<<grid_for(n, 1, kThreads, 8), kThreads, 0, st>>>(s->n_nodes, s->nnzb, s->diag_block.p, s->k64.p,
                                                                 W.dinv64.p, W.dinv32.p);
  W.launches++;
  WN_CUDA(cudaEventRecord(W.ev0, st));
  int total_iters = 0, total_outer = 0, status = 0;
  double worst = 0.0;
  for (int j0 = 0; j0 < n_rhs; j0 += kBatch) {
    const int m = std::min(kBatch, n_rhs - j0);
    kb_pack<<<grid_for(n * kBatch, 1, kThreads, 8), kThreads, 0, st>>>(n, F, n_rhs, j0, m, W.F.p);
    W.launches++;
    WN_CUDA(cudaGetLastError());
    BatchResult res;
    if (vmode == 1)
      WN_CHECK(batch_outer<float>(s, W, vmode, m, prm, chunk, st, res));
    else
      WN_CHECK(batch_outer<double>(s, W, vmode, m, prm, chunk, st, res));
    kb_unpack<<<grid_for(n * kBatch, 1, kThreads, 8), kThreads, 0, st>>>(n, W.U.p, n_rhs, j0, m, U);
    W.launches++;
    WN_CUDA(cudaGetLastError());
    total_iters += res.iterations;
    total_outer += res.outer;
    if (res.status == WN_EBREAKDOWN || (res.status != 0 && status == 0)) status = res.status;
    for (int j = 0; j < m; ++j) {
      if (case_iters) case_iters[j0 + j] = res.case_iters[j];
      if (case_rel) case_rel[j0 + j] = res.case_rel[j];
      worst = std::max(worst, res.case_rel[j]);
    }
  }
  WN_CUDA(cudaEventRecord(W.ev1, st));
  WN_CUDA(cudaEventSynchronize(W.ev1));
  float ms = 0.f;
  WN_CUDA(cudaEventElapsedTime(&ms, W.ev0, W.ev1));
  if (stats) {
    stats->iterations = total_iters;
    stats->outer_iterations = total_outer;
    stats->status = status;
    stats->rel_res = worst;
    stats->solve_seconds = ms * 1e-3;
    stats->kernel_launches = W.launches;
    stats->setup_seconds = s->amg ? s->amg->setup_seconds : 0.0;
    stats->n_levels = s->amg ? (int)s->amg->levels.size() + 1 : 0;
  }
  return 0;
}

}  // namespace wn
