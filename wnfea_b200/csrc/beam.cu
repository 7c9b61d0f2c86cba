// Co-rotational beam frames on sm_100a: internal force, consistent tangent assembled into a
// 6x6-block BSR matrix through an atomic-free element -> block gather, Dirichlet rows, and a
// block-Jacobi BiCGStab for the (in general nonsymmetric) tangent.
//
// The reference evaluates only the internal force (fast_kernels.py:451-537,
// kernels.cpp:19-204, hip_kernels.cpp:53-241) and obtains tangent actions by finite
// differences of the residual (jfnk_operator.py:98-134).  Here the tangent is the exact
// derivative of the same force code (forward-mode dual numbers, beam.cuh), one thread per
// (element, seed direction), so K_t v agrees with the JFNK directional derivative up to its
// truncation error and Newton converges quadratically.
#include <algorithm>
#include <cstring>
#include <vector>

#include "beam.cuh"
#include "common.cuh"
#include "device_array.h"
#include "kernels.h"
#include "wnfea_cuda.h"

namespace wn {

__device__ __forceinline__ void load_element(int64_t e, const double* __restrict__ nodes,
                                             const int32_t* __restrict__ el, const double* __restrict__ props,
                                             const double* __restrict__ eref, const double* __restrict__ L0,
                                             double x1[3], double x2[3], double ev[9], double p[6], double& l0,
                                             int64_t& n1, int64_t& n2) {
  n1 = el[e * 2];
  n2 = el[e * 2 + 1];
  for (int k = 0; k < 3; ++k) {
    x1[k] = nodes[n1 * 3 + k];
    x2[k] = nodes[n2 * 3 + k];
  }
  for (int k = 0; k < 9; ++k) ev[k] = eref[e * 9 + k];
  for (int k = 0; k < 6; ++k) p[k] = props[e * 6 + k];
  l0 = L0[e];
}

// f_e (n_el x 12), one thread per element (FP64)
__global__ void beam_force_kernel(int64_t n_el, const double* __restrict__ nodes, const int32_t* __restrict__ el,
                                  const double* __restrict__ props, const double* __restrict__ eref,
                                  const double* __restrict__ L0, const double* __restrict__ U,
                                  double* __restrict__ fe) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_el; e += (int64_t)gridDim.x * blockDim.x) {
    double x1[3], x2[3], ev[9], p[6], l0;
    int64_t n1, n2;
    load_element(e, nodes, el, props, eref, L0, x1, x2, ev, p, l0, n1, n2);
    double u1[3], t1[3], u2[3], t2[3], f[12];
    for (int k = 0; k < 3; ++k) {
      u1[k] = U[n1 * 6 + k];
      t1[k] = U[n1 * 6 + 3 + k];
      u2[k] = U[n2 * 6 + k];
      t2[k] = U[n2 * 6 + 3 + k];
    }
    beam_internal_force<double>(x1, x2, ev, l0, p, u1, t1, u2, t2, f);
    for (int k = 0; k < 12; ++k) fe[e * 12 + k] = f[k];
  }
}

// K_e column j = d f_e / d u_e[j]: one thread per (element, j), dual numbers seeded with
// e_j.  ke is n_el x 12 x 12 row-major (ke[e][i][j] = d f_i / d u_j).
__global__ void beam_tangent_kernel(int64_t n_el, const double* __restrict__ nodes, const int32_t* __restrict__ el,
                                    const double* __restrict__ props, const double* __restrict__ eref,
                                    const double* __restrict__ L0, const double* __restrict__ U,
                                    double* __restrict__ ke) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_el * 12;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / 12;
    const int j = (int)(t - e * 12);
    double x1[3], x2[3], ev[9], p[6], l0;
    int64_t n1, n2;
    load_element(e, nodes, el, props, eref, L0, x1, x2, ev, p, l0, n1, n2);
    Dual u1[3], t1[3], u2[3], t2[3], f[12];
    for (int k = 0; k < 3; ++k) {
      u1[k] = Dual(U[n1 * 6 + k], j == k ? 1.0 : 0.0);
      t1[k] = Dual(U[n1 * 6 + 3 + k], j == 3 + k ? 1.0 : 0.0);
      u2[k] = Dual(U[n2 * 6 + k], j == 6 + k ? 1.0 : 0.0);
      t2[k] = Dual(U[n2 * 6 + 3 + k], j == 9 + k ? 1.0 : 0.0);
    }
    beam_internal_force<Dual>(x1, x2, ev, l0, p, u1, t1, u2, t2, f);
    for (int i = 0; i < 12; ++i) ke[e * 144 + i * 12 + j] = f[i].d;
  }
}

// F (6 n) = sum over each node's incident (element, end) pairs, in element order
__global__ void beam_node_gather_kernel(int64_t n_nodes, const int64_t* __restrict__ inc_ptr,
                                        const int32_t* __restrict__ inc_ea, const double* __restrict__ fe,
                                        int accumulate, double* __restrict__ F) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_nodes * 6;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = t / 6;
    const int c = (int)(t - n * 6);
    double s = 0.0;
    for (int64_t q = inc_ptr[n]; q < inc_ptr[n + 1]; ++q) s += fe[(int64_t)inc_ea[q] * 6 + c];
    F[t] = accumulate ? F[t] + s : s;
  }
}

// BSR6 values: block b = sum of its element blocks (gather list src = e * 4 + 2 a + b,
// element order), Dirichlet rows/columns -> identity.  Block-contiguous (AoS) output.
__global__ void beam_gather_kernel(int64_t nnzb, const int32_t* __restrict__ gptr, const int32_t* __restrict__ gsrc,
                                   const double* __restrict__ ke, const int32_t* __restrict__ block_row,
                                   const int32_t* __restrict__ col_idx, const uint8_t* __restrict__ fixed,
                                   double* __restrict__ K) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnzb * 36;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / 36;
    const int k = (int)(t - b * 36);
    const int i = k / 6, j = k - (k / 6) * 6;
    double acc = 0.0;
    for (int32_t q = gptr[b]; q < gptr[b + 1]; ++q) {
      const int32_t src = gsrc[q];
      const int64_t e = src >> 2;
      const int a = (src >> 1) & 1, c = src & 1;
      acc += ke[e * 144 + (a * 6 + i) * 12 + c * 6 + j];
    }
    if (fixed) {
      const int64_t rd = (int64_t)block_row[b] * 6 + i, cd = (int64_t)col_idx[b] * 6 + j;
      if (fixed[rd] | fixed[cd]) acc = (rd == cd) ? 1.0 : 0.0;
    }
    K[t] = acc;
  }
}

// Inverse of each 6x6 diagonal block (Gauss-Jordan, partial pivoting); a singular block
// falls back to the inverse of its diagonal.
__global__ void beam_block_inverse_kernel(int64_t n_nodes, const int32_t* __restrict__ diag_block,
                                          const double* __restrict__ K, double* __restrict__ inv) {
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
    double a[6][12];
    const double* blk = K + (int64_t)diag_block[n] * 36;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 12; ++j) a[i][j] = j < 6 ? blk[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
    bool ok = true;
    for (int c = 0; c < 6 && ok; ++c) {
      int piv = c;
      for (int r = c + 1; r < 6; ++r)
        if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
      if (!(fabs(a[piv][c]) > 0.0)) {
        ok = false;
        break;
      }
      if (piv != c)
        for (int j = 0; j < 12; ++j) {
          const double tmp = a[c][j];
          a[c][j] = a[piv][j];
          a[piv][j] = tmp;
        }
      const double d = 1.0 / a[c][c];
      for (int j = 0; j < 12; ++j) a[c][j] *= d;
      for (int r = 0; r < 6; ++r)
        if (r != c) {
          const double f = a[r][c];
          for (int j = 0; j < 12; ++j) a[r][j] -= f * a[c][j];
        }
    }
    double* out = inv + n * 36;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        const double dg = blk[i * 6 + i];
        out[i * 6 + j] = ok ? a[i][j + 6] : (i == j ? (dg != 0.0 ? 1.0 / dg : 1.0) : 0.0);
      }
  }
}

// y_n = inv_n x_n (6x6 per node)
__global__ void beam_block_apply_kernel(int64_t n_nodes, const double* __restrict__ inv, const double* __restrict__ x,
                                        double* __restrict__ y) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_nodes * 6;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = t / 6;
    const int i = (int)(t - n * 6);
    double s = 0.0;
    for (int j = 0; j < 6; ++j) s += inv[n * 36 + i * 6 + j] * x[n * 6 + j];
    y[t] = s;
  }
}

// partial dots of (a, b) pairs into part[cta * 2 + k]; second stage sums in fixed order
__global__ void beam_dot2_kernel(int64_t n, const double* __restrict__ a0, const double* __restrict__ b0,
                                 const double* __restrict__ a1, const double* __restrict__ b1,
                                 double* __restrict__ part) {
  __shared__ double sh[8];
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    s0 += a0[i] * b0[i];
    if (a1) s1 += a1[i] * b1[i];
  }
  s0 = block_sum(s0, sh);
  s1 = block_sum(s1, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = s0;
    part[blockIdx.x * 2 + 1] = s1;
  }
}

// y = a x + b y + c z   (z may be null)
__global__ void beam_lincomb_kernel(int64_t n, double a, const double* __restrict__ x, double b, double* __restrict__ y,
                                    double c, const double* __restrict__ z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + (b != 0.0 ? b * y[i] : 0.0) + (z ? c * z[i] : 0.0);  // b == 0 ignores y
}


// Dense copy (row-major n x n, n = 6 n_nodes) of the BSR6 matrix; A must be zeroed first.
__global__ void beam_dense_kernel(int64_t n_nodes, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  const double* __restrict__ K, double* __restrict__ A) {
  const int64_t n = n_nodes * 6;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_nodes * 6;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = t / 6;
    const int i = (int)(t - row * 6);
    for (int32_t q = rp[row]; q < rp[row + 1]; ++q)
      for (int j = 0; j < 6; ++j) A[t * n + (int64_t)ci[q] * 6 + j] = K[(int64_t)q * 36 + i * 6 + j];
  }
}

// Blocked right-looking LU with partial pivoting and the solve of A x = b (x overwrites b),
// in panels of kLuPanel columns: per panel
//   beam_lu_panel_kernel   (one CTA)   pivots, row swaps, multipliers and rank-1 updates inside
//                                      the panel's columns, and the forward elimination of b;
//   beam_lu_swap_trsm_kernel (a thread per trailing column) the panel's row swaps and
//                                      U12 = L11^-1 A12 on the columns right of the panel;
//   beam_lu_update_kernel  (32 x 32 tiles) A22 -= L21 U12, each element subtracting the
//                                      panel's terms in column order;
// then beam_lu_backsub_kernel (one CTA).  Every element sees the unblocked algorithm's
// operations in its order (fused multiply-adds), so the factors and x do not depend on the
// panel width.  The multipliers of earlier panels are never read again (b is eliminated as
// the panels go), so row swaps touch the panel, the trailing columns and b only.
// status: 0 ok, 1 singular (a zero pivot column; the later kernels then see status != 0 and
// return).  Every loop is bounded by n.
constexpr int kLuPanel = 32;

__global__ void __launch_bounds__(1024) beam_lu_panel_kernel(int n, int k0, double* __restrict__ A,
                                                             double* __restrict__ b, int* __restrict__ piv,
                                                             int* __restrict__ status) {
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ int s_piv;
  __shared__ double s_pv;
  if (status[0] != 0) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int k1 = min(n, k0 + kLuPanel);
  for (int k = k0; k < k1; ++k) {
    // pivot: argmax |A[i][k]|, i >= k (ties -> smallest i)
    double best = -1.0;
    int bi = k;
    for (int i = k + tid; i < n; i += nt) {
      const double v = fabs(A[(int64_t)i * n + k]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      sv[warp] = best;
      si[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double bb = sv[0];
      int ii = si[0];
      for (int w = 1; w < nw; ++w)
        if (sv[w] > bb || (sv[w] == bb && si[w] < ii)) {
          bb = sv[w];
          ii = si[w];
        }
      s_piv = ii;
      s_pv = bb;
      piv[k - k0] = ii;
      if (!(bb > 0.0)) status[0] = 1;
    }
    __syncthreads();
    if (!(s_pv > 0.0)) return;
    const int p = s_piv;
    if (p != k) {  // the panel's columns and b
      for (int j = k0 + tid; j < k1; j += nt) {
        const double t = A[(int64_t)k * n + j];
        A[(int64_t)k * n + j] = A[(int64_t)p * n + j];
        A[(int64_t)p * n + j] = t;
      }
      if (tid == 0) {
        const double t = b[k];
        b[k] = b[p];
        b[p] = t;
      }
    }
    __syncthreads();
    const double pv = A[(int64_t)k * n + k];
    for (int i = k + 1 + tid; i < n; i += nt) {
      const double l = A[(int64_t)i * n + k] / pv;
      A[(int64_t)i * n + k] = l;
      b[i] = fma(-l, b[k], b[i]);
    }
    __syncthreads();
    // rank-1 update of the panel's remaining columns: a warp per row
    const double* __restrict__ pk = A + (int64_t)k * n;
    for (int i = k + 1 + warp; i < n; i += nw) {
      double* __restrict__ ai = A + (int64_t)i * n;
      const double l = ai[k];
      for (int j = k + 1 + lane; j < k1; j += 32) ai[j] = fma(-l, pk[j], ai[j]);
    }
    __syncthreads();
  }
}

// columns j >= k0 + kLuPanel: the panel's row swaps in order, then U12 = L11^-1 A12 (unit lower
// L11), one thread per column
__global__ void beam_lu_swap_trsm_kernel(int n, int k0, double* __restrict__ A, const int* __restrict__ piv,
                                         const int* __restrict__ status) {
  if (status[0] != 0) return;
  const int k1 = min(n, k0 + kLuPanel);
  for (int j = k1 + blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    for (int k = k0; k < k1; ++k) {
      const int p = piv[k - k0];
      if (p != k) {
        const double t = A[(int64_t)k * n + j];
        A[(int64_t)k * n + j] = A[(int64_t)p * n + j];
        A[(int64_t)p * n + j] = t;
      }
    }
    for (int k = k0; k < k1; ++k) {
      const double ukj = A[(int64_t)k * n + j];
      for (int i = k + 1; i < k1; ++i) A[(int64_t)i * n + j] = fma(-A[(int64_t)i * n + k], ukj, A[(int64_t)i * n + j]);
    }
  }
}

// A22 -= L21 U12 for rows and columns >= k0 + kLuPanel: a 32 x 32 tile per CTA (32 x 8 threads,
// four rows each), L21 and U12 tiles staged in shared memory
__global__ void __launch_bounds__(256) beam_lu_update_kernel(int n, int k0, double* __restrict__ A,
                                                             const int* __restrict__ status) {
  __shared__ double sl[32][kLuPanel + 1];
  __shared__ double su[kLuPanel][32 + 1];
  if (status[0] != 0) return;
  const int k1 = min(n, k0 + kLuPanel), w = k1 - k0;
  const int r0 = k1 + blockIdx.y * 32, c0 = k1 + blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < 32 * kLuPanel; e += 256) {
    const int r = e / kLuPanel, c = e % kLuPanel;
    sl[r][c] = (r0 + r < n && c < w) ? A[(int64_t)(r0 + r) * n + k0 + c] : 0.0;
    const int kr = e / 32, cc = e % 32;
    su[kr][cc] = (kr < w && c0 + cc < n) ? A[(int64_t)(k0 + kr) * n + c0 + cc] : 0.0;
  }
  __syncthreads();
  const int j = c0 + tx;
  if (j >= n) return;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = ty + 8 * q, i = r0 + r;
    if (i >= n) continue;
    double a = A[(int64_t)i * n + j];
    for (int k = 0; k < w; ++k) a = fma(-sl[r][k], su[k][tx], a);
    A[(int64_t)i * n + j] = a;
  }
}

// back substitution with the upper factor, column oriented
__global__ void __launch_bounds__(1024) beam_lu_backsub_kernel(int n, const double* __restrict__ A,
                                                               double* __restrict__ b, const int* __restrict__ status) {
  if (status[0] != 0) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int k = n - 1; k >= 0; --k) {
    if (tid == 0) b[k] /= A[(int64_t)k * n + k];
    __syncthreads();
    const double xk = b[k];
    for (int i = tid; i < k; i += nt) b[i] = fma(-A[(int64_t)i * n + k], xk, b[i]);
    __syncthreads();
  }
}

}  // namespace wn

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
namespace wn {

struct Beam {
  int device = 0;
  int64_t n_nodes = 0, n_el = 0, nnzb = 0;
  std::vector<int32_t> h_rp, h_ci;
  DArray<double> nodes, props, eref, L0;
  DArray<int32_t> el, rp, ci, block_row, diag_block, gptr, gsrc, inc_ea;
  DArray<int64_t> inc_ptr;
  DArray<uint8_t> fixed;
  DArray<double> fe, ke, K, dinv;
  // BiCGStab workspace
  DArray<double> r, rh, p, v, s, t, y, z, x, part;
  // dense LU workspace (small frames)
  DArray<double> dense;
  DArray<int> dstat;
  bool assembled = false;
};

static int build_beam_pattern(int64_t n_nodes, int64_t n_el, const int32_t* el, Beam& b, std::vector<int32_t>& rp,
                              std::vector<int32_t>& ci, std::vector<int32_t>& brow, std::vector<int32_t>& diag,
                              std::vector<int32_t>& gptr, std::vector<int32_t>& gsrc, std::vector<int64_t>& iptr,
                              std::vector<int32_t>& iea) {
  for (int64_t k = 0; k < n_el * 2; ++k)
    WN_REQUIRE(el[k] >= 0 && el[k] < n_nodes, WN_EMESH, "beam: element node index out of range");
  iptr.assign(n_nodes + 1, 0);
  for (int64_t k = 0; k < n_el * 2; ++k) iptr[el[k] + 1]++;
  for (int64_t i = 0; i < n_nodes; ++i) iptr[i + 1] += iptr[i];
  iea.resize(n_el * 2);
  {
    std::vector<int64_t> pos(iptr.begin(), iptr.end() - 1);
    for (int64_t e = 0; e < n_el; ++e)
      for (int a = 0; a < 2; ++a) iea[pos[el[e * 2 + a]]++] = (int32_t)(e * 2 + a);
  }
  rp.assign(n_nodes + 1, 0);
  std::vector<std::vector<int32_t>> rows(n_nodes);
  for (int64_t i = 0; i < n_nodes; ++i) {
    auto& r = rows[i];
    r.push_back((int32_t)i);  // every node keeps a diagonal block
    for (int64_t q = iptr[i]; q < iptr[i + 1]; ++q) {
      const int32_t e = iea[q] / 2;
      r.push_back(el[e * 2]);
      r.push_back(el[e * 2 + 1]);
    }
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    rp[i + 1] = rp[i] + (int32_t)r.size();
  }
  const int64_t nnzb = rp[n_nodes];
  ci.resize(nnzb);
  brow.resize(nnzb);
  diag.resize(n_nodes);
  for (int64_t i = 0; i < n_nodes; ++i)
    for (size_t k = 0; k < rows[i].size(); ++k) {
      ci[rp[i] + k] = rows[i][k];
      brow[rp[i] + k] = (int32_t)i;
      if (rows[i][k] == i) diag[i] = rp[i] + (int32_t)k;
    }
  // gather lists in (element, a, b) order
  auto find = [&](int32_t r, int32_t c) {
    return (int32_t)(std::lower_bound(ci.begin() + rp[r], ci.begin() + rp[r + 1], c) - ci.begin());
  };
  std::vector<int32_t> emap(n_el * 4);
  gptr.assign(nnzb + 1, 0);
  for (int64_t e = 0; e < n_el; ++e)
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 2; ++c) {
        const int32_t blk = find(el[e * 2 + a], el[e * 2 + c]);
        emap[e * 4 + a * 2 + c] = blk;
        gptr[blk + 1]++;
      }
  for (int64_t k = 0; k < nnzb; ++k) gptr[k + 1] += gptr[k];
  gsrc.resize(n_el * 4);
  std::vector<int32_t> pos(gptr.begin(), gptr.end() - 1);
  for (int64_t e = 0; e < n_el; ++e)
    for (int q = 0; q < 4; ++q) gsrc[pos[emap[e * 4 + q]]++] = (int32_t)(e * 4 + q);
  b.nnzb = nnzb;
  return 0;
}

static Beam* as_beam(void* h) { return reinterpret_cast<Beam*>(h); }

static int beam_dots(Beam* b, const double* a0, const double* b0, const double* a1, const double* b1, double* out2,
                     cudaStream_t st) {
  const int64_t n = b->n_nodes * 6;
  const int g = (int)std::min<int64_t>(256, (n + 255) / 256);
  beam_dot2_kernel<<<g, 256, 0, st>>>(n, a0, b0, a1, b1, b->part.p);
  WN_CUDA(cudaGetLastError());
  std::vector<double> h(2 * g);
  WN_CUDA(cudaMemcpyAsync(h.data(), b->part.p, sizeof(double) * 2 * g, cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  out2[0] = out2[1] = 0.0;
  for (int k = 0; k < g; ++k) {  // fixed order
    out2[0] += h[2 * k];
    out2[1] += h[2 * k + 1];
  }
  return 0;
}

}  // namespace wn

using namespace wn;

extern "C" {

int wn_beam_internal_forces(const double* nodes, const int32_t* elements, const double* props, const double* e_ref,
                            const double* L0_arr, const double* U, double* F_int, int n_elements, int n_nodes) {
  WN_REQUIRE(nodes && U && F_int && n_nodes > 0 && n_elements >= 0, WN_EINVAL, "wn_beam_internal_forces: bad argument");
  if (n_elements == 0) return 0;
  WN_REQUIRE(elements && props && e_ref && L0_arr, WN_EINVAL, "wn_beam_internal_forces: null argument");
  void* h = nullptr;
  WN_CHECK(wn_beam_create(n_nodes, n_elements, nodes, elements, props, e_ref, L0_arr, &h));
  Beam* b = as_beam(h);
  int rc = 0;
  DArray<double> dU, dF;
  rc = rc ? rc : dU.upload(U, (int64_t)n_nodes * 6);
  rc = rc ? rc : dF.upload(F_int, (int64_t)n_nodes * 6);
  if (rc == 0) {
    const int64_t ne = b->n_el;
    beam_force_kernel<<<grid_for(ne, 1, 128, 8), 128>>>(ne, b->nodes.p, b->el.p, b->props.p, b->eref.p, b->L0.p, dU.p,
                                                       b->fe.p);
    beam_node_gather_kernel<<<grid_for(n_nodes * 6, 1, 256, 8), 256>>>(n_nodes, b->inc_ptr.p, b->inc_ea.p, b->fe.p, 1,
                                                                       dF.p);
    cudaError_t e = cudaMemcpy(F_int, dF.p, dF.bytes(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      set_error("wn_beam_internal_forces: %s", cudaGetErrorString(e));
      rc = (int)e;
    }
  }
  wn_beam_destroy(h);
  return rc;
}

int wn_beam_create(int64_t n_nodes, int64_t n_el, const double* nodes, const int32_t* elements, const double* props,
                   const double* e_ref, const double* L0, void** out) {
  WN_REQUIRE(out && nodes && n_nodes > 0 && n_el >= 0 && (n_el == 0 || (elements && props && e_ref && L0)),
             WN_EINVAL, "wn_beam_create: bad argument");
  *out = nullptr;
  auto* b = new Beam();
  WN_CUDA(cudaGetDevice(&b->device));
  b->n_nodes = n_nodes;
  b->n_el = n_el;
  std::vector<int32_t> brow, diag, gptr, gsrc, iea;
  std::vector<int64_t> iptr;
  int rc = build_beam_pattern(n_nodes, n_el, elements, *b, b->h_rp, b->h_ci, brow, diag, gptr, gsrc, iptr, iea);
  const int64_t n = n_nodes * 6;
  rc = rc ? rc : b->nodes.upload(nodes, n_nodes * 3);
  rc = rc ? rc : b->el.upload(elements, n_el * 2);
  rc = rc ? rc : b->props.upload(props, n_el * 6);
  rc = rc ? rc : b->eref.upload(e_ref, n_el * 9);
  rc = rc ? rc : b->L0.upload(L0, n_el);
  rc = rc ? rc : b->rp.upload(b->h_rp);
  rc = rc ? rc : b->ci.upload(b->h_ci);
  rc = rc ? rc : b->block_row.upload(brow);
  rc = rc ? rc : b->diag_block.upload(diag);
  rc = rc ? rc : b->gptr.upload(gptr);
  rc = rc ? rc : b->gsrc.upload(gsrc);
  rc = rc ? rc : b->inc_ptr.upload(iptr);
  rc = rc ? rc : b->inc_ea.upload(iea);
  rc = rc ? rc : b->fixed.alloc(n);
  rc = rc ? rc : b->fixed.zero();
  rc = rc ? rc : b->fe.alloc(std::max<int64_t>(n_el, 1) * 12);
  rc = rc ? rc : b->ke.alloc(std::max<int64_t>(n_el, 1) * 144);
  rc = rc ? rc : b->K.alloc(b->nnzb * 36);
  rc = rc ? rc : b->dinv.alloc(n_nodes * 36);
  for (DArray<double>* v : {&b->r, &b->rh, &b->p, &b->v, &b->s, &b->t, &b->y, &b->z, &b->x})
    rc = rc ? rc : v->alloc(n);
  rc = rc ? rc : b->part.alloc(512);
  if (rc == 0) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_error("wn_beam_create: %s", cudaGetErrorString(e));
      rc = (int)e;
    }
  }
  if (rc != 0) {
    delete b;
    return rc;
  }
  *out = b;
  return 0;
}

int wn_beam_destroy(void* h) {
  if (h) {
    cudaSetDevice(as_beam(h)->device);
    delete as_beam(h);
  }
  return 0;
}

int wn_beam_info(void* h, int64_t* n_nodes, int64_t* n_el, int64_t* nnzb) {
  WN_REQUIRE(h, WN_EINVAL, "wn_beam_info: null handle");
  Beam* b = as_beam(h);
  if (n_nodes) *n_nodes = b->n_nodes;
  if (n_el) *n_el = b->n_el;
  if (nnzb) *nnzb = b->nnzb;
  return 0;
}

int wn_beam_get_pattern(void* h, int32_t* row_ptr, int32_t* col_idx) {
  WN_REQUIRE(h, WN_EINVAL, "wn_beam_get_pattern: null handle");
  Beam* b = as_beam(h);
  if (row_ptr) memcpy(row_ptr, b->h_rp.data(), sizeof(int32_t) * b->h_rp.size());
  if (col_idx) memcpy(col_idx, b->h_ci.data(), sizeof(int32_t) * b->h_ci.size());
  return 0;
}

int wn_beam_set_fixed(void* h, const uint8_t* fixed_mask) {
  WN_REQUIRE(h, WN_EINVAL, "wn_beam_set_fixed: null handle");
  Beam* b = as_beam(h);
  WN_CUDA(cudaSetDevice(b->device));
  if (fixed_mask)
    WN_CUDA(cudaMemcpy(b->fixed.p, fixed_mask, b->n_nodes * 6, cudaMemcpyHostToDevice));
  else
    WN_CHECK(b->fixed.zero());
  return 0;
}

int wn_beam_evaluate_device(void* h, const double* d_U, double* d_fint, int assemble_tangent, int apply_bcs,
                            uintptr_t stream) {
  WN_REQUIRE(h && d_U, WN_EINVAL, "wn_beam_evaluate_device: null argument");
  Beam* b = as_beam(h);
  WN_CUDA(cudaSetDevice(b->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t ne = b->n_el;
  if (d_fint) {
    if (ne) {
      beam_force_kernel<<<grid_for(ne, 1, 128, 8), 128, 0, st>>>(ne, b->nodes.p, b->el.p, b->props.p, b->eref.p,
                                                                b->L0.p, d_U, b->fe.p);
      WN_CUDA(cudaGetLastError());
    } else {
      WN_CHECK(b->fe.zero(st));
    }
    beam_node_gather_kernel<<<grid_for(b->n_nodes * 6, 1, 256, 8), 256, 0, st>>>(b->n_nodes, b->inc_ptr.p,
                                                                                 b->inc_ea.p, b->fe.p, 0, d_fint);
    WN_CUDA(cudaGetLastError());
  }
  if (assemble_tangent) {
    if (ne) {
      beam_tangent_kernel<<<grid_for(ne * 12, 1, 128, 8), 128, 0, st>>>(ne, b->nodes.p, b->el.p, b->props.p,
                                                                        b->eref.p, b->L0.p, d_U, b->ke.p);
      WN_CUDA(cudaGetLastError());
    }
    beam_gather_kernel<<<grid_for(b->nnzb * 36, 1, 256, 8), 256, 0, st>>>(
        b->nnzb, b->gptr.p, b->gsrc.p, b->ke.p, b->block_row.p, b->ci.p, apply_bcs ? b->fixed.p : nullptr, b->K.p);
    beam_block_inverse_kernel<<<grid_for(b->n_nodes, 1, 128, 8), 128, 0, st>>>(b->n_nodes, b->diag_block.p, b->K.p,
                                                                               b->dinv.p);
    WN_CUDA(cudaGetLastError());
    b->assembled = true;
  }
  return 0;
}

int wn_beam_evaluate(void* h, const double* U, double* fint, int assemble_tangent, int apply_bcs) {
  WN_REQUIRE(h && U, WN_EINVAL, "wn_beam_evaluate: null argument");
  Beam* b = as_beam(h);
  WN_CUDA(cudaSetDevice(b->device));
  const int64_t n = b->n_nodes * 6;
  DArray<double> dU, dF;
  WN_CHECK(dU.upload(U, n));
  if (fint) WN_CHECK(dF.alloc(n));
  WN_CHECK(wn_beam_evaluate_device(h, dU.p, fint ? dF.p : nullptr, assemble_tangent, apply_bcs, 0));
  if (fint) WN_CUDA(cudaMemcpy(fint, dF.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  WN_CUDA(cudaDeviceSynchronize());
  return 0;
}

int wn_beam_get_tangent(void* h, double* values) {
  WN_REQUIRE(h && values, WN_EINVAL, "wn_beam_get_tangent: null argument");
  Beam* b = as_beam(h);
  WN_REQUIRE(b->assembled, WN_ESTATE, "wn_beam_get_tangent: no tangent assembled");
  WN_CUDA(cudaMemcpy(values, b->K.p, b->K.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

int wn_beam_linear_system(void* h, void** out) {
  WN_REQUIRE(h && out, WN_EINVAL, "wn_beam_linear_system: null argument");
  Beam* b = as_beam(h);
  WN_REQUIRE(b->assembled, WN_ESTATE, "wn_beam_linear_system: assemble the tangent first");
  WN_CUDA(cudaSetDevice(b->device));
  std::vector<double> coords(b->n_nodes * 3);
  std::vector<uint8_t> fixed(b->n_nodes * 6);
  WN_CUDA(cudaMemcpy(coords.data(), b->nodes.p, coords.size() * sizeof(double), cudaMemcpyDeviceToHost));
  WN_CUDA(cudaMemcpy(fixed.data(), b->fixed.p, fixed.size(), cudaMemcpyDeviceToHost));
  bool any = false;
  for (uint8_t f : fixed) any = any || f;
  return make_bsr6_system(b->n_nodes, b->h_rp.data(), b->h_ci.data(), b->K.p, true, coords.data(),
                          any ? fixed.data() : nullptr, out);
}

int wn_beam_solve_device(void* h, const double* d_b, double* d_x, int method, double rtol, int max_iter, int* iters,
                         double* rel_res, uintptr_t stream) {
  WN_REQUIRE(h && d_b && d_x && rtol > 0 && max_iter > 0 && method >= 0 && method <= 2, WN_EINVAL,
             "wn_beam_solve_device: bad argument");
  Beam* b = as_beam(h);
  WN_REQUIRE(b->assembled, WN_ESTATE, "wn_beam_solve_device: assemble the tangent first");
  WN_CUDA(cudaSetDevice(b->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = b->n_nodes * 6;
  if (method == 1 || (method == 0 && n <= WN_BEAM_DENSE_MAX)) {
    WN_REQUIRE(n <= WN_BEAM_DENSE_MAX, WN_ETOOBIG, "wn_beam_solve_device: dense LU limited to %d DOFs",
               WN_BEAM_DENSE_MAX);
    WN_CHECK(b->dense.alloc(n * n));
    WN_CHECK(b->dstat.alloc(1 + kLuPanel));  // [0] status, [1..] the current panel's pivots
    WN_CUDA(cudaMemsetAsync(b->dense.p, 0, n * n * sizeof(double), st));
    WN_CUDA(cudaMemsetAsync(b->dstat.p, 0, sizeof(int), st));
    beam_dense_kernel<<<grid_for(n, 1, 256, 8), 256, 0, st>>>(b->n_nodes, b->rp.p, b->ci.p, b->K.p, b->dense.p);
    WN_CUDA(cudaMemcpyAsync(d_x, d_b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    const int ni = (int)n;
    int* piv = b->dstat.p + 1;
    for (int k0 = 0; k0 < ni; k0 += kLuPanel) {
      beam_lu_panel_kernel<<<1, 1024, 0, st>>>(ni, k0, b->dense.p, d_x, piv, b->dstat.p);
      const int rest = ni - std::min(ni, k0 + kLuPanel);
      if (rest > 0) {
        beam_lu_swap_trsm_kernel<<<(rest + 127) / 128, 128, 0, st>>>(ni, k0, b->dense.p, piv, b->dstat.p);
        const unsigned tiles = (unsigned)((rest + 31) / 32);
        beam_lu_update_kernel<<<dim3(tiles, tiles), 256, 0, st>>>(ni, k0, b->dense.p, b->dstat.p);
      }
    }
    beam_lu_backsub_kernel<<<1, 1024, 0, st>>>(ni, b->dense.p, d_x, b->dstat.p);
    WN_CUDA(cudaGetLastError());
    int stat = 0;
    WN_CUDA(cudaMemcpyAsync(&stat, b->dstat.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    WN_CUDA(cudaStreamSynchronize(st));
    if (iters) *iters = 1;
    // residual of the direct solve, on the (unfactored) BSR matrix
    WN_CHECK(launch_bsr_spmv_f64(6, 6, b->n_nodes, b->rp.p, b->ci.p, b->K.p, d_x, b->t.p, 1.0, 0.0, st));
    beam_lincomb_kernel<<<grid_for(n, 1, 256, 8), 256, 0, st>>>(n, 1.0, d_b, -1.0, b->t.p, 0.0, nullptr);
    WN_CUDA(cudaGetLastError());
    double d2[2];
    WN_CHECK(beam_dots(b, b->t.p, b->t.p, d_b, d_b, d2, st));
    if (rel_res) *rel_res = d2[1] > 0.0 ? std::sqrt(d2[0] / d2[1]) : 0.0;
    if (stat != 0) set_error("wn_beam_solve_device: singular tangent (zero pivot)");
    return stat == 0 ? 0 : WN_EBREAKDOWN;
  }
  const int gv = grid_for(n, 1, 256, 8);
  auto spmv = [&](const double* x, double* y) {
    return launch_bsr_spmv_f64(6, 6, b->n_nodes, b->rp.p, b->ci.p, b->K.p, x, y, 1.0, 0.0, st);
  };
  auto prec = [&](const double* x, double* y) {
    beam_block_apply_kernel<<<gv, 256, 0, st>>>(b->n_nodes, b->dinv.p, x, y);
    WN_CUDA(cudaGetLastError());
    return 0;
  };
  auto lin = [&](double a, const double* x, double bb, double* y, double c, const double* z) {
    beam_lincomb_kernel<<<gv, 256, 0, st>>>(n, a, x, bb, y, c, z);
    WN_CUDA(cudaGetLastError());
    return 0;
  };
  // preconditioned BiCGStab (van der Vorst 1992), x0 = 0
  double d2[2];
  WN_CUDA(cudaMemsetAsync(b->x.p, 0, n * sizeof(double), st));
  WN_CUDA(cudaMemcpyAsync(b->r.p, d_b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  WN_CUDA(cudaMemcpyAsync(b->rh.p, d_b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  WN_CUDA(cudaMemsetAsync(b->p.p, 0, n * sizeof(double), st));
  WN_CUDA(cudaMemsetAsync(b->v.p, 0, n * sizeof(double), st));
  WN_CHECK(beam_dots(b, d_b, d_b, nullptr, nullptr, d2, st));
  const double bnorm = std::sqrt(d2[0]);
  double rho = 1.0, alpha = 1.0, omega = 1.0, rn = bnorm;
  int it = 0, status = 0;
  if (bnorm == 0.0 || !std::isfinite(bnorm)) {
    status = std::isfinite(bnorm) ? 0 : WN_EBREAKDOWN;
  } else {
    for (it = 0; it < max_iter; ++it) {
      WN_CHECK(beam_dots(b, b->rh.p, b->r.p, nullptr, nullptr, d2, st));
      const double rho_new = d2[0];
      if (rho_new == 0.0 || !std::isfinite(rho_new)) {
        status = WN_EBREAKDOWN;
        break;
      }
      const double beta = (rho_new / rho) * (alpha / omega);
      rho = rho_new;
      WN_CHECK(lin(-omega * beta, b->v.p, beta, b->p.p, 1.0, b->r.p));  // p = r + beta (p - omega v)
      WN_CHECK(prec(b->p.p, b->y.p));
      WN_CHECK(spmv(b->y.p, b->v.p));
      WN_CHECK(beam_dots(b, b->rh.p, b->v.p, nullptr, nullptr, d2, st));
      alpha = rho / d2[0];
      WN_CHECK(lin(1.0, b->r.p, 0.0, b->s.p, -alpha, b->v.p));  // s = r - alpha v
      WN_CHECK(lin(alpha, b->y.p, 1.0, b->x.p, 0.0, nullptr));  // x += alpha y
      WN_CHECK(beam_dots(b, b->s.p, b->s.p, nullptr, nullptr, d2, st));
      if (std::sqrt(d2[0]) <= rtol * bnorm) {
        rn = std::sqrt(d2[0]);
        ++it;
        break;
      }
      WN_CHECK(prec(b->s.p, b->z.p));
      WN_CHECK(spmv(b->z.p, b->t.p));
      WN_CHECK(beam_dots(b, b->t.p, b->s.p, b->t.p, b->t.p, d2, st));
      omega = d2[1] > 0.0 ? d2[0] / d2[1] : 0.0;
      WN_CHECK(lin(omega, b->z.p, 1.0, b->x.p, 0.0, nullptr));         // x += omega z
      WN_CHECK(lin(1.0, b->s.p, 0.0, b->r.p, -omega, b->t.p));         // r = s - omega t
      WN_CHECK(beam_dots(b, b->r.p, b->r.p, nullptr, nullptr, d2, st));
      rn = std::sqrt(d2[0]);
      if (!std::isfinite(rn)) {
        status = WN_EBREAKDOWN;
        break;
      }
      if (rn <= rtol * bnorm) {
        ++it;
        break;
      }
      if (omega == 0.0) {
        status = WN_EBREAKDOWN;
        break;
      }
    }
    if (status == 0 && rn > rtol * bnorm) status = WN_ENOCONV;
  }
  WN_CUDA(cudaMemcpyAsync(d_x, b->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  WN_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = it;
  if (rel_res) *rel_res = bnorm > 0.0 ? rn / bnorm : 0.0;
  return status;
}

int wn_beam_solve(void* h, const double* rhs, double* x, int method, double rtol, int max_iter, int* iters,
                  double* rel_res) {
  WN_REQUIRE(h && rhs && x, WN_EINVAL, "wn_beam_solve: null argument");
  Beam* b = as_beam(h);
  WN_CUDA(cudaSetDevice(b->device));
  const int64_t n = b->n_nodes * 6;
  DArray<double> db, dx;
  WN_CHECK(db.upload(rhs, n));
  WN_CHECK(dx.alloc(n));
  const int rc = wn_beam_solve_device(h, db.p, dx.p, method, rtol, max_iter, iters, rel_res, 0);
  WN_CUDA(cudaMemcpy(x, dx.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  return rc;
}

}  // extern "C"
