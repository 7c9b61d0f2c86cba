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
//   * mixed precision: FP32 matrix / V-cycle / vectors with FP32 accumulation inside an
//     FP64 refinement loop whose residual r = F - K u uses the FP64 matrix.
#include <chrono>
#include <cmath>
#include <cstring>

#include "amg.h"
#include "common.cuh"
#include "kernels.h"
#include "solid.h"
#include "spmv.cuh"
#include "solver.h"

namespace wn {

// ---------------------------------------------------------------------------------------
// reductions shared by the PCG kernels
// ---------------------------------------------------------------------------------------
constexpr int kThreads = 256;

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
struct XPNew {  // p_j = z_j + beta p_old_j
  const T* __restrict__ z;
  const T* __restrict__ p;
  T beta;
  __device__ __forceinline__ T operator()(int64_t j) const { return z[j] + beta * p[j]; }
};

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
__global__ void __launch_bounds__(kThreads) k_pre_first(int64_t n_rows, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                        const T* __restrict__ b, const T* __restrict__ dinv,
                                                        T inv_theta, int deg, T c1, T c2, T* __restrict__ x,
                                                        T* __restrict__ r, T* __restrict__ d, T* __restrict__ res,
                                                        const PcgScalars* __restrict__ S) {
  if (S->done) return;
  WARP_ROW_LOOP(n_rows) {
    T acc[BS];
    warp_block_row<BS, BS, T, T>(rp, ci, av, row, XD0<T>{b, dinv, inv_theta}, acc, lane);
    if (lane < BS) {
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
__global__ void __launch_bounds__(kThreads) k_cheb_step(int64_t n_rows, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                        const T* __restrict__ dinv, const T* __restrict__ d_in,
                                                        T* __restrict__ d_out, T* __restrict__ r, T* __restrict__ x,
                                                        T c1, T c2, const T* __restrict__ b, double* __restrict__ part,
                                                        const PcgScalars* __restrict__ S) {
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double dot = 0.0;
  WARP_ROW_LOOP(n_rows) {
    T acc[BS];
    warp_block_row<BS, BS, T, T>(rp, ci, av, row, XLoad<T, T>{d_in}, acc, lane);
    if (lane < BS) {
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
__global__ void __launch_bounds__(kThreads) k_residual(int64_t n_rows, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                       const T* __restrict__ b, const T* __restrict__ x,
                                                       T* __restrict__ res, const PcgScalars* __restrict__ S) {
  if (S->done) return;
  WARP_ROW_LOOP(n_rows) {
    T acc[BS];
    warp_block_row<BS, BS, T, T>(rp, ci, av, row, XLoad<T, T>{x}, acc, lane);
    if (lane < BS) {
      const int64_t i = row * BS + lane;
      res[i] = b[i] - pick<BS>(acc, lane);
    }
  }
}

// y = A x (accumulate = 0) or y += A x (accumulate = 1) for a BR x BC block matrix
template <int BR, int BC, typename T>
__global__ void __launch_bounds__(kThreads) k_level_spmv(int64_t n_rows, const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                         const T* __restrict__ x, T* __restrict__ y, int accumulate,
                                                         const PcgScalars* __restrict__ S) {
  if (S->done) return;
  WARP_ROW_LOOP(n_rows) {
    T acc[BR];
    warp_block_row<BR, BC, T, T>(rp, ci, av, row, XLoad<T, T>{x}, acc, lane);
    if (lane < BR) {
      const int64_t i = row * BR + lane;
      const T v = pick<BR>(acc, lane);
      y[i] = accumulate ? y[i] + v : v;
    }
  }
}

// First post-smoothing step from a nonzero x: r0 = D^-1 (b - A x), d0 = r0 / theta,
// x2 = x + d0 (x2 is a separate buffer: x is still read by neighbouring rows).
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) k_post_first(int64_t n_rows, const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                         const T* __restrict__ b, const T* __restrict__ dinv,
                                                         T inv_theta, const T* __restrict__ x, T* __restrict__ x2,
                                                         T* __restrict__ r, T* __restrict__ d, double* __restrict__ part,
                                                         const PcgScalars* __restrict__ S) {
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  double dot = 0.0;
  WARP_ROW_LOOP(n_rows) {
    T acc[BS];
    warp_block_row<BS, BS, T, T>(rp, ci, av, row, XLoad<T, T>{x}, acc, lane);
    if (lane < BS) {
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

// coarsest level: x = A_c^-1 b with the dense FP64 inverse (one warp per row)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_coarse(int64_t n, const double* __restrict__ inv,
                                                     const T* __restrict__ b, T* __restrict__ x,
                                                     const PcgScalars* __restrict__ S) {
  if (S->done) return;
  WARP_ROW_LOOP(n) {
    double s = 0.0;
    const double* rowp = inv + row * n;
    for (int64_t j = lane; j < n; j += 32) s += rowp[j] * (double)b[j];
    s = warp_sum(s);
    if (lane == 0) x[row] = (T)s;
  }
}

// ---------------------------------------------------------------------------------------
// PCG kernels
// ---------------------------------------------------------------------------------------

// r = b, x = 0, partC = b . b ; (+ zero-RHS handling in k_init_scalars)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_init_vecs(int64_t n, const T* __restrict__ b, T* __restrict__ x,
                                                        T* __restrict__ r, double* __restrict__ partC) {
  __shared__ double sh[kThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T v = b[i];
    r[i] = v;
    x[i] = T(0);
    s += (double)v * (double)v;
  }
  write_part(s, partC, sh);
}

__global__ void k_init_scalars(PcgScalars* S, const double* __restrict__ partC, int nparts, double rtol) {
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
    S->done = (bb == 0.0 || !isfinite(bb)) ? 1 : 0;
    if (!isfinite(bb)) S->status = WN_EBREAKDOWN;
  }
}

// z = D^-1 r (jacobi = 1) or z = r (jacobi = 0); partA = r . z
template <typename T>
__global__ void __launch_bounds__(kThreads) k_prec_vec(int64_t n, const T* __restrict__ r, const T* __restrict__ dinv,
                                                       int jacobi, T* __restrict__ z, double* __restrict__ partA,
                                                       const PcgScalars* __restrict__ S) {
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

// iteration k: rz = sum(partA); beta = rz / rz_prev (0 at k = 0); p_new = z + beta p_old;
// q = A p_new; partB = p_new . q.  Parity par = k & 1 selects the p buffers and rz slot.
template <int BS, typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_dot(int64_t n_rows, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci, const T* __restrict__ av,
                                                       const T* __restrict__ z, const T* __restrict__ p_old,
                                                       T* __restrict__ p_new, T* __restrict__ q,
                                                       const double* __restrict__ partA, double* __restrict__ partB,
                                                       int nparts, int first, int par, PcgScalars* __restrict__ S) {
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  const double rz = reduce_parts(partA, nparts, sh);
  const double rz_prev = S->rz[par ^ 1];
  const T beta = first ? T(0) : (T)(rz / rz_prev);
  double dot = 0.0;
  WARP_ROW_LOOP(n_rows) {
    T acc[BS];
    warp_block_row<BS, BS, T, T>(rp, ci, av, row, XPNew<T>{z, p_old, beta}, acc, lane);
    if (lane < BS) {
      const int64_t i = row * BS + lane;
      const T pi = z[i] + beta * p_old[i];
      const T qi = pick<BS>(acc, lane);
      p_new[i] = pi;
      q[i] = qi;
      dot += (double)pi * (double)qi;
    }
  }
  write_part(dot, partB, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0) S->rz[par] = rz;
}

// alpha = rz / (p . q); x += alpha p; r -= alpha q; partC = r . r
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                     const T* __restrict__ p, const T* __restrict__ q,
                                                     const double* __restrict__ partB, double* __restrict__ partC,
                                                     int nparts, int par, PcgScalars* __restrict__ S) {
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
  const T a = (T)alpha;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    const T ri = r[i] - a * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  write_part(s, partC, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0) S->alpha = alpha;
}

// convergence test after iteration k (one CTA)
__global__ void k_check(PcgScalars* S, const double* __restrict__ partC, int nparts, int k, int max_iter) {
  __shared__ double sh[kThreads / 32];
  if (S->done) return;
  const double rr = reduce_parts(partC, nparts, sh);
  if (threadIdx.x == 0) {
    S->rr = rr;
    S->iters = k + 1;
    if (!isfinite(rr)) {
      S->status = WN_EBREAKDOWN;
      S->done = 1;
    } else if (rr <= S->tol2) {
      S->done = 1;
    } else if (k + 1 >= max_iter) {
      S->status = WN_ENOCONV;
      S->done = 1;
    }
  }
}

// ---------------------------------------------------------------------------------------
// mixed-precision refinement kernels (FP64)
// ---------------------------------------------------------------------------------------

// r64 = F - K64 u64, r32 = (float) r64, partC = r64 . r64
__global__ void __launch_bounds__(kThreads) k_outer_residual(int64_t n_rows, const int32_t* __restrict__ rp,
                                                             const int32_t* __restrict__ ci,
                                                             const double* __restrict__ av, const double* __restrict__ F,
                                                             const double* __restrict__ u, double* __restrict__ r64,
                                                             float* __restrict__ r32, double* __restrict__ partC) {
  __shared__ double sh[kThreads / 32];
  double s = 0.0;
  WARP_ROW_LOOP(n_rows) {
    double acc[3];
    warp_block_row<3, 3, double, double>(rp, ci, av, row, XLoad<double, double>{u}, acc, lane);
    if (lane < 3) {
      const int64_t i = row * 3 + lane;
      const double ri = F[i] - pick<3>(acc, lane);
      r64[i] = ri;
      if (r32) r32[i] = (float)ri;
      s += ri * ri;
    }
  }
  write_part(s, partC, sh);
}

// u64 += (double) dx32
__global__ void k_accumulate(int64_t n, double* __restrict__ u, const float* __restrict__ dx) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    u[i] += (double)dx[i];
}

__global__ void k_fill_dinv(int64_t n_rows, const int32_t* __restrict__ diag_block, const double* __restrict__ k64,
                            double* __restrict__ d64, float* __restrict__ d32) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_rows * 3;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = t / 3;
    const int c = (int)(t - row * 3);
    const double dv = k64[(int64_t)diag_block[row] * 9 + c * 4];
    const double inv = (fabs(dv) > 1e-12) ? 1.0 / dv : 1.0;  // solid_solver.py:230
    d64[t] = inv;
    d32[t] = (float)inv;
  }
}

// ---------------------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------------------
static inline int rows_grid(int64_t n_rows) { return grid_for(n_rows, 32, kThreads, 8); }
static inline int vec_grid(int64_t n) { return grid_for(n, 1, kThreads, 8); }

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
                  const PcgScalars* S, cudaStream_t st) {
  const int nlev = (int)H.levels.size();
  if (lvl == nlev) {  // coarsest
    k_coarse<T><<<rows_grid(H.n_coarse), kThreads, 0, st>>>(H.n_coarse, H.coarse_inv.p, b, out, S);
    W.launches++;
    return 0;
  }
  DevLevel& L = H.levels[lvl];
  LevelVecs<T>& V = Prec<T>::vecs(L);
  const int64_t nr = L.n_nodes;
  const T* dinv = Prec<T>::dinv(L);
  const int deg = H.degree;
  const T it = (T)L.inv_theta;
  const int g = rows_grid(nr);
  auto run = [&](auto bs_tag) -> int {
    constexpr int BS = decltype(bs_tag)::value;
    const int32_t* rp;
    const int32_t* ci;
    const T* av;
    level_A<BS, T>(s, L, lvl, rp, ci, av);
    // pre-smoothing (+ residual)
    const T c1 = deg >= 2 ? (T)L.c1[0] : T(0), c2 = deg >= 2 ? (T)L.c2[0] : T(0);
    k_pre_first<BS, T><<<g, kThreads, 0, st>>>(nr, rp, ci, av, b, dinv, it, deg, c1, c2, V.x.p, V.r.p, V.d.p,
                                               V.res.p, S);
    W.launches++;
    T* din = V.d.p;
    T* dout = V.d2.p;
    for (int k = 2; k < deg; ++k) {
      k_cheb_step<BS, T><<<g, kThreads, 0, st>>>(nr, rp, ci, av, dinv, din, dout, V.r.p, V.x.p, (T)L.c1[k - 1],
                                                 (T)L.c2[k - 1], b, nullptr, S);
      W.launches++;
      std::swap(din, dout);
    }
    if (deg >= 2) {
      k_residual<BS, T><<<g, kThreads, 0, st>>>(nr, rp, ci, av, b, V.x.p, V.res.p, S);
      W.launches++;
    }
    // restriction b_c = R res
    DevLevel* Ln = lvl + 1 < nlev ? &H.levels[lvl + 1] : nullptr;
    T* bc = Ln ? Prec<T>::vecs(*Ln).b.p : Prec<T>::cb(H);
    T* xc = Ln ? Prec<T>::vecs(*Ln).x2.p : Prec<T>::cx(H);
    if (deg == 0) xc = Ln ? Prec<T>::vecs(*Ln).x.p : xc;
    k_level_spmv<6, BS, T><<<rows_grid(L.R.n_rows), kThreads, 0, st>>>(L.R.n_rows, L.R.rp.p, L.R.ci.p,
                                                                        Prec<T>::Rv(L), V.res.p, bc, 0, S);
    W.launches++;
    WN_CHECK(vcycle<T>(s, H, W, lvl + 1, bc, xc, nullptr, S, st));
    // prolongation x += P x_c
    k_level_spmv<BS, 6, T><<<g, kThreads, 0, st>>>(nr, L.P.rp.p, L.P.ci.p, Prec<T>::Pv(L), xc, V.x.p, 1, S);
    W.launches++;
    // post-smoothing: result in `out`
    double* part_last = (deg == 1) ? part : nullptr;
    k_post_first<BS, T><<<(part_last ? SolverWork::kParts : g), kThreads, 0, st>>>(nr, rp, ci, av, b, dinv, it, V.x.p,
                                                                                   out, V.r.p, V.d.p, part_last, S);
    W.launches++;
    din = V.d.p;
    dout = V.d2.p;
    for (int k = 1; k < deg; ++k) {
      double* pk = (k == deg - 1) ? part : nullptr;
      k_cheb_step<BS, T><<<(pk ? SolverWork::kParts : g), kThreads, 0, st>>>(
          nr, rp, ci, av, dinv, din, dout, V.r.p, out, (T)L.c1[k - 1], (T)L.c2[k - 1], b, pk, S);
      W.launches++;
      std::swap(din, dout);
    }
    return 0;
  };
  int rc;
  if (L.bs == 3)
    rc = run(std::integral_constant<int, 3>{});
  else
    rc = run(std::integral_constant<int, 6>{});
  WN_CHECK(rc);
  WN_CUDA(cudaGetLastError());
  return 0;
}

// z = M r with partials of r . z into partA
template <typename T>
static int apply_prec(Solid* s, SolverWork& W, int precond, const T* r, T* z, const PcgScalars* S, cudaStream_t st) {
  if (precond == 2) return vcycle<T>(s, *s->amg, W, 0, r, z, W.partA.p, S, st);
  k_prec_vec<T><<<SolverWork::kParts, kThreads, 0, st>>>(W.n, r, Prec<T>::fine_dinv(W), precond == 1 ? 1 : 0, z,
                                                         W.partA.p, S);
  W.launches++;
  WN_CUDA(cudaGetLastError());
  return 0;
}

// one PCG iteration k (parity k & 1)
template <typename T>
static int pcg_iteration(Solid* s, SolverWork& W, int precond, int k, int max_iter, PcgScalars* S, cudaStream_t st) {
  PcgVecs<T>& P = Prec<T>::pcg(W);
  const int par = k & 1;
  T* p_new = par ? P.p1.p : P.p0.p;
  T* p_old = par ? P.p0.p : P.p1.p;
  const int32_t* rp = s->row_ptr.p;
  const int32_t* ci = s->col_idx.p;
  const T* av = Prec<T>::A0(s);
  k_spmv_dot<3, T><<<SolverWork::kParts, kThreads, 0, st>>>(s->n_nodes, rp, ci, av, P.z.p, p_old, p_new, P.q.p,
                                                            W.partA.p, W.partB.p, SolverWork::kParts, k == 0, par, S);
  k_update<T><<<SolverWork::kParts, kThreads, 0, st>>>(W.n, P.x.p, P.r.p, p_new, P.q.p, W.partB.p, W.partC.p,
                                                       SolverWork::kParts, par, S);
  k_check<<<1, kThreads, 0, st>>>(S, W.partC.p, SolverWork::kParts, k, max_iter);
  W.launches += 3;
  WN_CUDA(cudaGetLastError());
  return apply_prec<T>(s, W, precond, P.r.p, P.z.p, S, st);
}

// PCG on the fine matrix in precision T: solves A x = b (b, x are the PcgVecs' r/x after
// init).  Iterations are replayed through a CUDA graph of `chunk` iterations.
template <typename T>
static int pcg_solve(Solid* s, SolverWork& W, int pi, const T* b, double rtol, int max_iter, int precond, int chunk,
                     int use_graph, PcgScalars* S, cudaStream_t st, PcgScalars* hS) {
  PcgVecs<T>& P = Prec<T>::pcg(W);
  k_init_vecs<T><<<SolverWork::kParts, kThreads, 0, st>>>(W.n, b, P.x.p, P.r.p, W.partC.p);
  k_init_scalars<<<1, kThreads, 0, st>>>(S, W.partC.p, SolverWork::kParts, rtol);
  W.launches += 2;
  WN_CUDA(cudaGetLastError());
  WN_CHECK(apply_prec<T>(s, W, precond, P.r.p, P.z.p, S, st));
  chunk = std::max(2, chunk + (chunk & 1));  // even: parity pattern repeats per chunk
  GraphCache& G = W.graphs[pi][1];
  const int64_t key = ((int64_t)precond << 40) ^ ((int64_t)chunk << 20) ^ (int64_t)max_iter;
  int k0 = 0;
  // the first chunk is issued directly (iteration 0 uses beta = 0)
  for (int k = 0; k < chunk && k < max_iter; ++k) WN_CHECK(pcg_iteration<T>(s, W, precond, k, max_iter, S, st));
  k0 = chunk;
  while (true) {
    WN_CUDA(cudaMemcpyAsync(hS, S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    WN_CUDA(cudaStreamSynchronize(st));
    if (hS->done || k0 >= max_iter) break;
    if (use_graph) {
      if (G.key != key || G.stream != st || !G.exec) {
        G.reset();
        cudaGraph_t graph;
        WN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = 0;
        // iteration indices inside the graph are relative: k_check uses k for the iteration
        // count, so the graph is captured for "k0 = chunk" and the host re-launches it with
        // the count advanced by the kernels themselves (S->iters); max_iter bounds it.
        for (int k = 0; k < chunk && rc == 0; ++k) rc = pcg_iteration<T>(s, W, precond, chunk + k, max_iter, S, st);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        WN_CHECK(rc);
        WN_CUDA(e);
        e = cudaGraphInstantiate(&G.exec, graph, 0);
        cudaGraphDestroy(graph);
        WN_CUDA(e);
        G.key = key;
        G.stream = st;
      }
      WN_CUDA(cudaGraphLaunch(G.exec, st));
    } else {
      for (int k = 0; k < chunk; ++k) WN_CHECK(pcg_iteration<T>(s, W, precond, k0 + k, max_iter, S, st));
    }
    k0 += chunk;
  }
  return 0;
}

}  // namespace wn
