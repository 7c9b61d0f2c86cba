// Smoothed-aggregation AMG setup on the device.
//
// The host builder (amg_setup.cpp, the template of amg_preconditioner.py:193-332) spends most of
// its time in the block products of the Galerkin operator (A P, then R (A P)), in the power
// iterations for rho(D^-1 A) and in the smoothed prolongator (I - w D^-1 A) P_tent -- all of
// them passes over matrices that already live in HBM.  Here each level runs:
//   device: 1/diag(A), rho(D^-1 A) by power iteration, the Frobenius norm of every block;
//   host:   the greedy aggregation from those norms and the per-aggregate QR of the near-null
//           space (sequential, and cheap: a few percent of the host builder's time);
//   device: P = (I - w D^-1 A) P_tent, R = P^T, A P, A_c = R (A P), symmetrised.
// Every device product is deterministic and follows the host builder's summation order (per
// output block: the left factor's row in order, then the block product r, s, t), and blocks that
// come out all zero are dropped as the host builder drops them.  Each sparse product is a
// symbolic pass (the sorted unique output columns of each row, found with a hash set in shared
// memory), a numeric pass (one thread per output block) and a compaction pass.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "amg.h"
#include "amg_device.h"
#include "common.cuh"
#include "pattern.h"
#include "solid.h"

namespace wn {
namespace {

constexpr int kT = 256;
constexpr int kSymThreads = 128;
constexpr int kHashCap = 4096;   // shared-memory hash set of one output row (ints)
constexpr int kUniqueCap = 1024;  // most distinct output columns of one row
constexpr int kWarpBuf = 1024;    // candidates per warp in the prolongator pattern

// a device block matrix as the setup kernels read it: row-major blocks (stride == 0) or
// component-major ones (entry (r, c) of block k at v[(r * bc + c) * stride + k]: the fine C3D10
// matrix)
struct DMat {
  int br, bc;
  int64_t n_rows, n_cols, nnzb;
  const int32_t* rp;
  const int32_t* ci;
  const double* v;
  int64_t stride;
  __device__ __forceinline__ double at(int64_t k, int r, int c) const {
    return stride ? v[(int64_t)(r * bc + c) * stride + k] : v[k * br * bc + r * bc + c];
  }
};

DMat dmat(const DevBsr& m) {
  return DMat{m.br, m.bc, m.n_rows, m.n_cols, m.nnzb, m.rp.p, m.ci.p, m.v64.p, 0};
}

// position of column c in the sorted row [lo, hi) of ci, -1 if absent
__device__ __forceinline__ int32_t find_col(const int32_t* __restrict__ ci, int32_t lo, int32_t hi, int32_t c) {
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    const int32_t v = ci[mid];
    if (v == c) return mid;
    if (v < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return -1;
}

// ---------------------------------------------------------------------------------------
// diagonal, power iteration, block norms
// ---------------------------------------------------------------------------------------
__global__ void ks_inv_diag(DMat A, double* __restrict__ dinv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_rows; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = find_col(A.ci, A.rp[i], A.rp[i + 1], (int32_t)i);
    for (int r = 0; r < A.br; ++r) {
      const double dv = k >= 0 ? A.at(k, r, r) : 0.0;
      dinv[i * A.br + r] = (dv != 0.0) ? 1.0 / dv : 1.0;
    }
  }
}

// y = A x with the host builder's order: per row DOF, per block the row's dot product, added in
// block order
__global__ void ks_spmv_rows(DMat A, const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < A.n_rows * A.br;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / A.br;
    const int r = (int)(t - i * A.br);
    double acc = 0.0;
    for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const double* xx = x + (int64_t)A.ci[k] * A.bc;
      double s = 0.0;
      for (int c = 0; c < A.bc; ++c) s += A.at(k, r, c) * xx[c];
      acc += s;
    }
    y[t] = acc;
  }
}

// per-CTA partial sums of v^2 (after v *= scale when scale != null); fixed order
__global__ void ks_sumsq(int64_t n, double* __restrict__ v, const double* __restrict__ scale,
                         double* __restrict__ part) {
  __shared__ double sh[kT / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double a = v[i];
    if (scale) {
      a *= scale[i];
      v[i] = a;
    }
    s += a * a;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void ks_divide(int64_t n, double* __restrict__ v, double d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] /= d;
}

// Frobenius norm of every block, bitwise the host builder's block_fro (the same explicit fused
// multiply-adds in the same order): the aggregation compares these norms, and on regular meshes
// many neighbours' blocks have equal norms, so a last-bit difference would break those ties
// differently and change the aggregates
__global__ void ks_block_norms(DMat A, double* __restrict__ nrm) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < A.nnzb; k += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < A.br; ++r)
      for (int c = 0; c < A.bc; ++c) {
        const double b = A.at(k, r, c);
        s = fma(b, b, s);
      }
    nrm[k] = sqrt(s);
  }
}

// ---------------------------------------------------------------------------------------
// smoothed prolongator P = P_tent - w D^-1 A P_tent (row i: bs x 6 blocks at the aggregates of
// i and of its neighbours)
// ---------------------------------------------------------------------------------------
// one warp per row: the sorted unique aggregates of the row (count, or columns when out_ci)
__global__ void ks_p_pattern(DMat A, const int32_t* __restrict__ agg, int smooth, int32_t* __restrict__ cnt,
                             const int32_t* __restrict__ rp_out, int32_t* __restrict__ ci_out, int* __restrict__ err) {
  __shared__ int32_t buf[kT / 32][kWarpBuf];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int32_t* b = buf[w];
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < A.n_rows; i += nw) {
    const int32_t k0 = A.rp[i], len = smooth ? A.rp[i + 1] - k0 : 0;
    const int m = len + 1;  // candidate 0: the row's own aggregate
    if (m > kWarpBuf) {
      if (lane == 0) *err = 1;
      continue;
    }
    for (int p = lane; p < m; p += 32) b[p] = p == 0 ? agg[i] : agg[A.ci[k0 + p - 1]];
    __syncwarp();
    // unique values: first occurrence of each value >= 0; rank = distinct values below it
    int local = 0;
    for (int p = lane; p < m; p += 32) {
      const int32_t v = b[p];
      bool first = v >= 0;
      for (int q = 0; q < p && first; ++q) first = b[q] != v;
      if (!first) continue;
      ++local;
      if (ci_out) {
        int rank = 0;
        for (int q = 0; q < m; ++q) {
          const int32_t u = b[q];
          if (u < 0 || u >= v) continue;
          bool fu = true;
          for (int z = 0; z < q && fu; ++z) fu = b[z] != u;
          rank += fu;
        }
        ci_out[rp_out[i] + rank] = v;
      }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if (lane == 0 && cnt) cnt[i] = local;
    __syncwarp();
  }
}

// values of the P pattern (thread per block); nzflag[k] = 1 if the block is not all zero
template <int BS>
__global__ void ks_p_values(DMat A, const int32_t* __restrict__ agg, const double* __restrict__ qnode,
                            const double* __restrict__ dinv, double w, const int32_t* __restrict__ prow,
                            const int32_t* __restrict__ pci, int64_t nnz, double* __restrict__ pv,
                            uint8_t* __restrict__ nzflag) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = prow[q];
    const int32_t a = pci[q];
    double s[BS * 6];
#pragma unroll
    for (int e = 0; e < BS * 6; ++e) s[e] = 0.0;
    if (agg[i] == a) {
#pragma unroll
      for (int e = 0; e < BS * 6; ++e) s[e] += qnode[i * BS * 6 + e];
    }
    if (w != 0.0) {
      for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int32_t j = A.ci[k];
        if (agg[j] != a) continue;
        const double* qj = qnode + (int64_t)j * BS * 6;
#pragma unroll
        for (int r = 0; r < BS; ++r) {
          const double f = -w * dinv[i * BS + r];
#pragma unroll
          for (int c = 0; c < BS; ++c) {
            const double av = A.at(k, r, c);
            if (av == 0.0) continue;
#pragma unroll
            for (int t = 0; t < 6; ++t) s[r * 6 + t] += f * av * qj[c * 6 + t];
          }
        }
      }
    }
    bool nz = false;
#pragma unroll
    for (int e = 0; e < BS * 6; ++e) {
      pv[q * BS * 6 + e] = s[e];
      nz = nz || s[e] != 0.0;
    }
    nzflag[q] = nz ? 1 : 0;
  }
}

// block-row index of every block
__global__ void ks_block_rows(int64_t n_rows, const int32_t* __restrict__ rp, int32_t* __restrict__ row) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x)
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) row[k] = (int32_t)i;
}

// nonzero blocks per row
__global__ void ks_count_nz(int64_t n_rows, const int32_t* __restrict__ rp, const uint8_t* __restrict__ nzflag,
                            int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = 0;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) c += nzflag[k];
    cnt[i] = c;
  }
}

// copy the nonzero blocks of each row, in order (thread per row)
__global__ void ks_compact(int64_t n_rows, int bsz, const int32_t* __restrict__ rp_in, const int32_t* __restrict__ ci_in,
                           const double* __restrict__ v_in, const uint8_t* __restrict__ nzflag,
                           const int32_t* __restrict__ rp_out, int32_t* __restrict__ ci_out, double* __restrict__ v_out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t o = rp_out[i];
    for (int32_t k = rp_in[i]; k < rp_in[i + 1]; ++k) {
      if (!nzflag[k]) continue;
      ci_out[o] = ci_in[k];
      for (int e = 0; e < bsz; ++e) v_out[(int64_t)o * bsz + e] = v_in[(int64_t)k * bsz + e];
      ++o;
    }
  }
}

// ---------------------------------------------------------------------------------------
// transpose (R = P^T): counts per column, scatter, then each column's entries ordered by row
// ---------------------------------------------------------------------------------------
__global__ void ks_col_count(int64_t nnz, const int32_t* __restrict__ ci, int32_t* __restrict__ cnt) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[ci[k]], 1);  // integer counts: order-independent
}

__global__ void ks_col_scatter(int64_t nnz, const int32_t* __restrict__ ci, const int32_t* __restrict__ row,
                               const int32_t* __restrict__ tp, int32_t* __restrict__ cursor,
                               int32_t* __restrict__ trow, int32_t* __restrict__ tsrc) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = ci[k];
    const int32_t p = tp[c] + atomicAdd(&cursor[c], 1);  // any slot of the column: ordered next
    trow[p] = row[k];
    tsrc[p] = (int32_t)k;
  }
}

// warp per column: entry rank = number of the column's entries with a smaller row; writes the
// transposed blocks (BR x BC source blocks -> BC x BR)
__global__ void ks_col_order(int64_t n_cols, int br, int bc, const int32_t* __restrict__ tp,
                             const int32_t* __restrict__ trow, const int32_t* __restrict__ tsrc,
                             const double* __restrict__ v, int32_t* __restrict__ tci, double* __restrict__ tv) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int bsz = br * bc;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n_cols; c += nw) {
    const int32_t a = tp[c], e = tp[c + 1];
    for (int32_t p = a + lane; p < e; p += 32) {
      const int32_t r = trow[p];
      int32_t rank = 0;
      for (int32_t q = a; q < e; ++q) rank += trow[q] < r;
      const int32_t o = a + rank;
      tci[o] = r;
      const double* s = v + (int64_t)tsrc[p] * bsz;
      double* d = tv + (int64_t)o * bsz;
      for (int rr = 0; rr < br; ++rr)
        for (int cc = 0; cc < bc; ++cc) d[cc * br + rr] = s[rr * bc + cc];
    }
  }
}

// ---------------------------------------------------------------------------------------
// sparse block product C = A B
// ---------------------------------------------------------------------------------------
// CTA per row of C: the sorted unique columns of A(i,:) B.  count pass (ci_out == null) or
// column pass.  err: bit 0 = hash table too full, bit 1 = too many distinct columns.
__global__ void __launch_bounds__(kSymThreads) ks_gemm_pattern(DMat A, const int32_t* __restrict__ brp,
                                                               const int32_t* __restrict__ bci,
                                                               int32_t* __restrict__ cnt,
                                                               const int32_t* __restrict__ rp_out,
                                                               int32_t* __restrict__ ci_out, int* __restrict__ err) {
  __shared__ int32_t table[kHashCap];
  __shared__ int32_t keys[kUniqueCap];
  __shared__ int n_keys, full;
  for (int64_t i = blockIdx.x; i < A.n_rows; i += gridDim.x) {
    for (int h = threadIdx.x; h < kHashCap; h += blockDim.x) table[h] = -1;
    if (threadIdx.x == 0) {
      n_keys = 0;
      full = 0;
    }
    __syncthreads();
    const int32_t k0 = A.rp[i], k1 = A.rp[i + 1];
    // candidate columns, one per (A block, B block) pair: warp w takes A's blocks w, w + 4, ...
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int32_t k = k0 + warp; k < k1; k += kSymThreads / 32) {
      const int32_t j = A.ci[k];
      for (int32_t q = brp[j] + lane; q < brp[j + 1]; q += 32) {
        const int32_t c = bci[q];
        uint32_t h = ((uint32_t)c * 2654435761u) & (kHashCap - 1);
        for (int probe = 0; probe < kHashCap; ++probe) {
          const int32_t prev = atomicCAS(&table[h], -1, c);
          if (prev == -1) {
            const int slot = atomicAdd(&n_keys, 1);
            if (slot < kUniqueCap)
              keys[slot] = c;
            else
              full = 1;
            break;
          }
          if (prev == c) break;
          h = (h + 1) & (kHashCap - 1);
        }
      }
    }
    __syncthreads();
    const int nk = n_keys;
    if (nk > kUniqueCap || nk * 4 > kHashCap * 3 || full) {
      if (threadIdx.x == 0) atomicOr(err, 2);
    } else if (ci_out) {
      for (int p = threadIdx.x; p < nk; p += blockDim.x) {
        const int32_t v = keys[p];
        int rank = 0;
        for (int q = 0; q < nk; ++q) rank += keys[q] < v;
        ci_out[rp_out[i] + rank] = v;
      }
    } else if (threadIdx.x == 0) {
      cnt[i] = nk;
    }
    __syncthreads();
  }
}

// thread per block of C: C(i, J) = sum over A(i,:) in order of A(i,k) B(k, J) (B's block found by
// binary search in its sorted row); nzflag = the block is not all zero
template <int AR, int AK, int BC>
__global__ void ks_gemm_values(DMat A, const int32_t* __restrict__ brp, const int32_t* __restrict__ bci,
                               const double* __restrict__ bv, const int32_t* __restrict__ crow,
                               const int32_t* __restrict__ cci, int64_t nnz, double* __restrict__ cv,
                               uint8_t* __restrict__ nzflag) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = crow[q];
    const int32_t J = cci[q];
    double acc[AR * BC];
#pragma unroll
    for (int e = 0; e < AR * BC; ++e) acc[e] = 0.0;
    for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int32_t j = A.ci[k];
      const int32_t p = find_col(bci, brp[j], brp[j + 1], J);
      if (p < 0) continue;
      const double* b = bv + (int64_t)p * AK * BC;
#pragma unroll
      for (int r = 0; r < AR; ++r)
#pragma unroll
        for (int s = 0; s < AK; ++s) {
          const double av = A.at(k, r, s);
#pragma unroll
          for (int t = 0; t < BC; ++t) acc[r * BC + t] += av * b[s * BC + t];
        }
    }
    bool nz = false;
#pragma unroll
    for (int e = 0; e < AR * BC; ++e) {
      cv[q * AR * BC + e] = acc[e];
      nz = nz || acc[e] != 0.0;
    }
    nzflag[q] = nz ? 1 : 0;
  }
}

// A <- (A + A^T) / 2 for a structurally symmetric block matrix (b x b blocks, thread per row)
__global__ void ks_symmetrize(int64_t n_rows, int b, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                              const double* __restrict__ v, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x)
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
      const int32_t j = ci[k];
      const int32_t f = find_col(ci, rp[j], rp[j + 1], (int32_t)i);
      const double* x = v + (int64_t)k * b * b;
      double* o = out + (int64_t)k * b * b;
      if (f < 0) {
        for (int e = 0; e < b * b; ++e) o[e] = x[e];
        continue;
      }
      const double* y = v + (int64_t)f * b * b;
      for (int r = 0; r < b; ++r)
        for (int c = 0; c < b; ++c) o[r * b + c] = 0.5 * (x[r * b + c] + y[c * b + r]);
    }
}

__global__ void ks_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// ---------------------------------------------------------------------------------------
// block-Jacobi smoothing of the coarse levels as a change of basis
// ---------------------------------------------------------------------------------------
// Per node i of a 6-DOF level: the Cholesky factor L_i of its diagonal block (D_i = L_i L_i^T)
// and L_i^-1, both lower triangular, row-major 6 x 6.  A pivot at or below 1e-13 of the block's
// largest diagonal entry (a direction the aggregate's prolongator columns do not span, e.g. a
// zero column next to a support) is replaced by 1 with its row and column of L zeroed: that DOF
// keeps the old basis, and L stays invertible.
__global__ void ks_block_chol(DMat A, double* __restrict__ lf, double* __restrict__ li) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_rows; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = find_col(A.ci, A.rp[i], A.rp[i + 1], (int32_t)i);
    double a[36], l[36], m[36];
    double scale = 0.0;
    for (int e = 0; e < 36; ++e) {
      a[e] = k >= 0 ? A.at(k, e / 6, e % 6) : ((e % 7) == 0 ? 1.0 : 0.0);
      l[e] = 0.0;
      m[e] = 0.0;
    }
    for (int r = 0; r < 6; ++r) scale = fmax(scale, fabs(a[r * 7]));
    for (int c = 0; c < 6; ++c) {
      double d = a[c * 7];
      for (int j = 0; j < c; ++j) d -= l[c * 6 + j] * l[c * 6 + j];
      if (!(d > 1e-13 * scale)) {
        for (int j = 0; j < c; ++j) l[c * 6 + j] = 0.0;
        l[c * 7] = 1.0;
        continue;  // l[r][c] = 0 below
      }
      const double dc = sqrt(d);
      l[c * 7] = dc;
      for (int r = c + 1; r < 6; ++r) {
        double s = a[r * 6 + c];
        for (int j = 0; j < c; ++j) s -= l[r * 6 + j] * l[c * 6 + j];
        l[r * 6 + c] = s / dc;
      }
    }
    // L^-1 by forward substitution, column by column
    for (int c = 0; c < 6; ++c) {
      m[c * 7] = 1.0 / l[c * 7];
      for (int r = c + 1; r < 6; ++r) {
        double s = 0.0;
        for (int j = c; j < r; ++j) s += l[r * 6 + j] * m[j * 6 + c];
        m[r * 6 + c] = -s / l[r * 7];
      }
    }
    for (int e = 0; e < 36; ++e) {
      lf[i * 36 + e] = l[e];
      li[i * 36 + e] = m[e];
    }
  }
}

// Y = (U X) V for one BR x 6 block, row by row with fixed-order fused multiply-adds; U, X, V
// and the store are accessors, so a block and its transpose go through the same operations
template <int BR, typename UF, typename XF, typename VF, typename YF>
__device__ __forceinline__ void basis_block(const UF& U, const XF& X, const VF& V, const YF& Y) {
  for (int r = 0; r < BR; ++r) {
    double t[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < BR; ++m) s = fma(U(r, m), X(m, c), s);
      t[c] = s;
    }
#pragma unroll
    for (int c2 = 0; c2 < 6; ++c2) {
      double s = 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) s = fma(t[c], V(c, c2), s);
      Y(r, c2, s);
    }
  }
}

// A^_ab = L_a^-1 A_ab L_b^-T on a 6-DOF level.  A block below the diagonal (a > b) is computed as
// the transpose of the canonical product of its mirror (L_b^-1 A_ba L_a^-T with A_ba = A_ab^T,
// bitwise, since the level matrices are symmetrised), and a diagonal block keeps the upper
// triangle of its product, mirrored, so A^ is exactly symmetric.
__global__ void ks_basis_level(int64_t nnzb, const int32_t* __restrict__ row, const int32_t* __restrict__ ci,
                               const double* __restrict__ v, const double* __restrict__ li, double* __restrict__ out) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnzb; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = row[k], b = ci[k];
    const bool up = a <= b;
    const int64_t lo = up ? a : b, hi = up ? b : a;
    const double* X = v + k * 36;
    double* Y = out + k * 36;
    basis_block<6>([&](int r, int m) { return li[lo * 36 + r * 6 + m]; },
                   [&](int m, int c) { return up ? X[m * 6 + c] : X[c * 6 + m]; },
                   [&](int c, int c2) { return li[hi * 36 + c2 * 6 + c]; },
                   [&](int r, int c2, double s) {
                     if (a == b) {  // a diagonal block: its upper triangle, mirrored
                       if (c2 >= r) Y[r * 6 + c2] = Y[c2 * 6 + r] = s;
                     } else if (up) {
                       Y[r * 6 + c2] = s;
                     } else {
                       Y[c2 * 6 + r] = s;
                     }
                   });
  }
}

// The transfer operator between a level f (BR DOFs per node) and the next level c:
// P^_ia = L_i^T P_ia L_a^-T (lf: the factors of level f, null = identity, the fine level;
// lic: the inverse factors of level c, null = identity, the dense coarsest level).  With
// transposed = 1 the blocks are those of R = P^T (row a, column i) and each is the transpose of
// the same product, so R^ = P^^T bitwise.
template <int BR>
__global__ void ks_basis_transfer(int64_t nnzb, const int32_t* __restrict__ row, const int32_t* __restrict__ ci,
                                  const double* __restrict__ v, const double* __restrict__ lf,
                                  const double* __restrict__ lic, int transposed, double* __restrict__ out) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnzb; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = transposed ? ci[k] : row[k], a = transposed ? row[k] : ci[k];
    const double* X = v + k * BR * 6;
    double* Y = out + k * BR * 6;
    basis_block<BR>([&](int r, int m) { return lf ? lf[i * 36 + m * 6 + r] : (r == m ? 1.0 : 0.0); },
                    [&](int m, int c) { return transposed ? X[c * BR + m] : X[m * 6 + c]; },
                    [&](int c, int c2) { return lic ? lic[a * 36 + c2 * 6 + c] : (c == c2 ? 1.0 : 0.0); },
                    [&](int r, int c2, double s) {
                      if (transposed)
                        Y[c2 * BR + r] = s;
                      else
                        Y[r * 6 + c2] = s;
                    });
  }
}

// ---------------------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------------------
int grid_n(int64_t n) { return grid_for(n, 1, kT, 16); }

template <typename T>
int download(const DArray<T>& d, int64_t n, std::vector<T>& h) {
  h.resize(n);
  if (n) WN_CUDA(cudaMemcpy(h.data(), d.p, sizeof(T) * n, cudaMemcpyDeviceToHost));
  return 0;
}

// exclusive scan of per-row counts (device) into a row pointer (device and host); total nnz
int scan_counts(const DArray<int32_t>& cnt, int64_t n, DArray<int32_t>& rp, std::vector<int32_t>& h_rp,
                int64_t* total) {
  std::vector<int32_t> c;
  WN_CHECK(download(cnt, n, c));
  h_rp.assign(n + 1, 0);
  int64_t acc = 0;
  for (int64_t i = 0; i < n; ++i) {
    acc += c[i];
    WN_REQUIRE(acc < (int64_t)INT32_MAX, WN_ETOOBIG, "device AMG setup: matrix too large for 32-bit indices");
    h_rp[i + 1] = (int32_t)acc;
  }
  *total = acc;
  WN_CHECK(rp.upload(h_rp));
  return 0;
}

// drop all-zero blocks: (rp_t, ci_t, v_t, flags) -> M (rp, ci, v64 set; host row pointer too)
int compact_into(int64_t n_rows, int br, int bc, int64_t n_cols, const DArray<int32_t>& rp_t,
                 const DArray<int32_t>& ci_t, const DArray<double>& v_t, const DArray<uint8_t>& flags, DevBsr& M,
                 std::vector<int32_t>& h_rp) {
  DArray<int32_t> cnt;
  WN_CHECK(cnt.alloc(std::max<int64_t>(n_rows, 1)));
  ks_count_nz<<<grid_n(n_rows), kT>>>(n_rows, rp_t.p, flags.p, cnt.p);
  WN_CUDA(cudaGetLastError());
  int64_t nnz = 0;
  WN_CHECK(scan_counts(cnt, n_rows, M.rp, h_rp, &nnz));
  WN_CHECK(M.ci.alloc(std::max<int64_t>(nnz, 1)));
  WN_CHECK(M.v64.alloc(std::max<int64_t>(nnz, 1) * br * bc));
  ks_compact<<<grid_n(n_rows), kT>>>(n_rows, br * bc, rp_t.p, ci_t.p, v_t.p, flags.p, M.rp.p, M.ci.p, M.v64.p);
  WN_CUDA(cudaGetLastError());
  M.br = br;
  M.bc = bc;
  M.n_rows = n_rows;
  M.n_cols = n_cols;
  M.nnzb = nnz;
  return 0;
}

// rho(D^-1 A) by power iteration from the host builder's start vector
int power_rho_device(const DMat& A, const DArray<double>& dinv, int iters, double* rho) {
  const int64_t n = A.n_rows * A.br;
  std::vector<double> x0(n);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int64_t i = 0; i < n; ++i) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    x0[i] = 0.5 + (double)(s % 1000003) / 1000003.0;
  }
  DArray<double> x, y, part;
  WN_CHECK(x.upload(x0));
  WN_CHECK(y.alloc(n));
  const int g = grid_n(n);
  WN_CHECK(part.alloc(g));
  std::vector<double> hp(g);
  auto norm = [&](double* v, const double* scale, double* out) -> int {
    ks_sumsq<<<g, kT>>>(n, v, scale, part.p);
    WN_CUDA(cudaGetLastError());
    WN_CUDA(cudaMemcpy(hp.data(), part.p, sizeof(double) * g, cudaMemcpyDeviceToHost));
    double t = 0.0;
    for (int k = 0; k < g; ++k) t += hp[k];
    *out = std::sqrt(t);
    return 0;
  };
  double lam = 0.0;
  double* xp = x.p;
  double* yp = y.p;
  for (int it = 0; it < std::max(iters, 1); ++it) {
    double nx = 0.0;
    WN_CHECK(norm(xp, nullptr, &nx));
    if (nx == 0.0) {
      *rho = 1.0;
      return 0;
    }
    ks_divide<<<g, kT>>>(n, xp, nx);
    ks_spmv_rows<<<grid_n(n), kT>>>(A, xp, yp);
    WN_CUDA(cudaGetLastError());
    WN_CHECK(norm(yp, dinv.p, &lam));
    std::swap(xp, yp);
  }
  *rho = lam;
  return 0;
}

// C = A B (B row-major blocks); the product's blocks AR x BC
template <int AR, int AK, int BC>
int gemm(const DMat& A, const DevBsr& B, DevBsr& C, std::vector<int32_t>& h_rp) {
  const int64_t n = A.n_rows;
  DArray<int32_t> cnt, rp_t, ci_t, row_t;
  DArray<int> err;
  WN_CHECK(cnt.alloc(std::max<int64_t>(n, 1)));
  WN_CHECK(err.alloc(1));
  WN_CHECK(err.zero());
  const int gs = (int)std::min<int64_t>(std::max<int64_t>(n, 1), (int64_t)kNumSMs * 16);
  ks_gemm_pattern<<<gs, kSymThreads>>>(A, B.rp.p, B.ci.p, cnt.p, nullptr, nullptr, err.p);
  WN_CUDA(cudaGetLastError());
  int e = 0;
  WN_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return 1;  // a row beyond the shared-memory capacities: the caller falls back
  int64_t nnz = 0;
  std::vector<int32_t> h_rp_t;
  WN_CHECK(scan_counts(cnt, n, rp_t, h_rp_t, &nnz));
  WN_CHECK(ci_t.alloc(std::max<int64_t>(nnz, 1)));
  WN_CHECK(row_t.alloc(std::max<int64_t>(nnz, 1)));
  ks_gemm_pattern<<<gs, kSymThreads>>>(A, B.rp.p, B.ci.p, nullptr, rp_t.p, ci_t.p, err.p);
  ks_block_rows<<<grid_n(n), kT>>>(n, rp_t.p, row_t.p);
  DArray<double> v_t;
  DArray<uint8_t> flags;
  WN_CHECK(v_t.alloc(std::max<int64_t>(nnz, 1) * AR * BC));
  WN_CHECK(flags.alloc(std::max<int64_t>(nnz, 1)));
  ks_gemm_values<AR, AK, BC><<<grid_n(nnz), kT>>>(A, B.rp.p, B.ci.p, B.v64.p, row_t.p, ci_t.p, nnz, v_t.p, flags.p);
  WN_CUDA(cudaGetLastError());
  return compact_into(n, AR, BC, B.n_cols, rp_t, ci_t, v_t, flags, C, h_rp);
}

int gemm_any(const DMat& A, const DevBsr& B, DevBsr& C, std::vector<int32_t>& h_rp) {
  if (A.br == 3 && A.bc == 3 && B.bc == 6) return gemm<3, 3, 6>(A, B, C, h_rp);
  if (A.br == 6 && A.bc == 3 && B.bc == 6) return gemm<6, 3, 6>(A, B, C, h_rp);
  if (A.br == 6 && A.bc == 6 && B.bc == 6) return gemm<6, 6, 6>(A, B, C, h_rp);
  set_error("device AMG setup: unexpected block product %dx%d . %dx%d", A.br, A.bc, B.br, B.bc);
  return WN_EINVAL;
}

// T = M^T (blocks transposed)
int transpose(const DevBsr& M, DevBsr& T, std::vector<int32_t>& h_rp) {
  const int64_t nnz = M.nnzb;
  DArray<int32_t> cnt, cursor, row, trow, tsrc;
  WN_CHECK(cnt.alloc(std::max<int64_t>(M.n_cols, 1)));
  WN_CHECK(cnt.zero());
  WN_CHECK(cursor.alloc(std::max<int64_t>(M.n_cols, 1)));
  WN_CHECK(cursor.zero());
  WN_CHECK(row.alloc(std::max<int64_t>(nnz, 1)));
  WN_CHECK(trow.alloc(std::max<int64_t>(nnz, 1)));
  WN_CHECK(tsrc.alloc(std::max<int64_t>(nnz, 1)));
  ks_col_count<<<grid_n(nnz), kT>>>(nnz, M.ci.p, cnt.p);
  ks_block_rows<<<grid_n(M.n_rows), kT>>>(M.n_rows, M.rp.p, row.p);
  WN_CUDA(cudaGetLastError());
  int64_t total = 0;
  WN_CHECK(scan_counts(cnt, M.n_cols, T.rp, h_rp, &total));
  ks_col_scatter<<<grid_n(nnz), kT>>>(nnz, M.ci.p, row.p, T.rp.p, cursor.p, trow.p, tsrc.p);
  WN_CHECK(T.ci.alloc(std::max<int64_t>(nnz, 1)));
  WN_CHECK(T.v64.alloc(std::max<int64_t>(nnz, 1) * M.br * M.bc));
  ks_col_order<<<grid_for(M.n_cols, 32, kT, 16), kT>>>(M.n_cols, M.br, M.bc, T.rp.p, trow.p, tsrc.p, M.v64.p, T.ci.p,
                                                      T.v64.p);
  WN_CUDA(cudaGetLastError());
  T.br = M.bc;
  T.bc = M.br;
  T.n_rows = M.n_cols;
  T.n_cols = M.n_rows;
  T.nnzb = nnz;
  return 0;
}

int fill_float(DevBsr& M) {
  const int64_t nv = std::max<int64_t>(M.nnzb, 1) * M.br * M.bc;
  WN_CHECK(M.v32.alloc(nv));
  ks_to_float<<<grid_n(nv), kT>>>(nv, M.v64.p, M.v32.p);
  WN_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace

int amg_build_device(Solid* s, const wn_amg_params& prm, AmgHierarchy& H) {
  const auto t0 = std::chrono::steady_clock::now();
  PhaseClock tr("amg_build_device");
  HostHierarchy& host = H.host;
  host = HostHierarchy();
  host.params = prm;
  std::vector<double> B;
  near_null_space(s->n_nodes, s->bs, s->h_nodes.data(), s->bcs_applied ? s->h_fixed.data() : nullptr, B);
  // level 0: the assembled matrix in place (component-major 3x3, or row-major 6x6)
  DMat A{s->bs, s->bs, s->n_nodes, s->n_nodes, s->nnzb, s->row_ptr.p, s->col_idx.p, s->k64.p,
         s->bs == 3 ? s->nnzb : 0};
  std::vector<int32_t> h_rp = s->h_row_ptr, h_ci = s->h_col_idx;
  DevBsr A_own;  // the current level's matrix for levels >= 1
  int bs = s->bs;
  int64_t n = s->n_nodes;
  H.levels.clear();
  for (int lvl = 0;; ++lvl) {
    const int64_t ndof = n * bs;
    if (ndof <= prm.coarse_size || lvl >= prm.max_levels - 1) break;
    HostLevel L;
    L.bs = bs;
    L.n_nodes = n;
    DevLevel D;
    D.bs = bs;
    D.n_nodes = n;
    WN_CHECK(D.dinv64.alloc(ndof));
    ks_inv_diag<<<grid_n(n), kT>>>(A, D.dinv64.p);
    WN_CUDA(cudaGetLastError());
    WN_CHECK(download(D.dinv64, ndof, L.dinv));
    WN_CHECK(power_rho_device(A, D.dinv64, prm.power_iters, &L.rho));
    tr.mark("rho", lvl);
    // aggregation on the host from the block norms
    DArray<double> nrm;
    WN_CHECK(nrm.alloc(std::max<int64_t>(A.nnzb, 1)));
    ks_block_norms<<<grid_n(A.nnzb), kT>>>(A, nrm.p);
    WN_CUDA(cudaGetLastError());
    std::vector<double> h_nrm;
    WN_CHECK(download(nrm, A.nnzb, h_nrm));
    nrm.release();
    L.n_agg = aggregate_norms(n, h_rp.data(), h_ci.data(), h_nrm.data(), prm.strength_theta, L.agg);
    if (L.n_agg == 0 || L.n_agg * 6 >= (int64_t)(0.8 * ndof)) break;  // coarsening stalled
    std::vector<double> Qnode, Bc;
    tentative_prolongator(n, bs, L.n_agg, L.agg, B, Qnode, Bc);
    tr.mark("aggregate+qr", lvl);
    // smoothed prolongator on the device
    DArray<int32_t> d_agg, cnt, rp_t, ci_t, row_t;
    DArray<double> d_q, v_t;
    DArray<uint8_t> flags;
    DArray<int> err;
    WN_CHECK(d_agg.upload(L.agg));
    WN_CHECK(d_q.upload(Qnode));
    WN_CHECK(cnt.alloc(n));
    WN_CHECK(err.alloc(1));
    WN_CHECK(err.zero());
    const int smooth = prm.smooth_prolongator ? 1 : 0;
    const double w = smooth ? prm.prolong_omega / L.rho : 0.0;
    const int gw = grid_for(n, 32, kT, 16);
    ks_p_pattern<<<gw, kT>>>(A, d_agg.p, smooth, cnt.p, nullptr, nullptr, err.p);
    WN_CUDA(cudaGetLastError());
    int e = 0;
    WN_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return 1;
    int64_t nnz_t = 0;
    std::vector<int32_t> h_rp_t;
    WN_CHECK(scan_counts(cnt, n, rp_t, h_rp_t, &nnz_t));
    WN_CHECK(ci_t.alloc(std::max<int64_t>(nnz_t, 1)));
    WN_CHECK(row_t.alloc(std::max<int64_t>(nnz_t, 1)));
    WN_CHECK(v_t.alloc(std::max<int64_t>(nnz_t, 1) * bs * 6));
    WN_CHECK(flags.alloc(std::max<int64_t>(nnz_t, 1)));
    ks_p_pattern<<<gw, kT>>>(A, d_agg.p, smooth, nullptr, rp_t.p, ci_t.p, err.p);
    ks_block_rows<<<grid_n(n), kT>>>(n, rp_t.p, row_t.p);
    if (bs == 3)
      ks_p_values<3><<<grid_n(nnz_t), kT>>>(A, d_agg.p, d_q.p, D.dinv64.p, w, row_t.p, ci_t.p, nnz_t, v_t.p, flags.p);
    else
      ks_p_values<6><<<grid_n(nnz_t), kT>>>(A, d_agg.p, d_q.p, D.dinv64.p, w, row_t.p, ci_t.p, nnz_t, v_t.p, flags.p);
    WN_CUDA(cudaGetLastError());
    std::vector<int32_t> h_rp_p, h_rp_r, h_rp_ap, h_rp_c;
    WN_CHECK(compact_into(n, bs, 6, L.n_agg, rp_t, ci_t, v_t, flags, D.P, h_rp_p));
    rp_t.release();
    ci_t.release();
    row_t.release();
    v_t.release();
    flags.release();
    WN_CHECK(transpose(D.P, D.R, h_rp_r));
    tr.mark("prolongator", lvl);
    // Galerkin product A_c = R (A P), symmetrised
    DevBsr AP, Ac;
    int rc = gemm_any(A, D.P, AP, h_rp_ap);
    if (rc == 1) return 1;
    WN_CHECK(rc);
    tr.mark("A*P", lvl);
    rc = gemm_any(dmat(D.R), AP, Ac, h_rp_c);
    if (rc == 1) return 1;
    WN_CHECK(rc);
    AP = DevBsr();
    DArray<double> sym;
    WN_CHECK(sym.alloc(std::max<int64_t>(Ac.nnzb, 1) * 36));
    ks_symmetrize<<<grid_n(Ac.n_rows), kT>>>(Ac.n_rows, 6, Ac.rp.p, Ac.ci.p, Ac.v64.p, sym.p);
    WN_CUDA(cudaGetLastError());
    std::swap(Ac.v64, sym);
    tr.mark("R*(AP)", lvl);
    // host row pointers for the streamed-kernel plans
    D.h_P_rp = std::move(h_rp_p);
    D.h_R_rp = std::move(h_rp_r);
    if (lvl > 0) {
      D.A = std::move(A_own);
      D.h_A_rp = h_rp;
    }
    host.levels.push_back(std::move(L));
    H.levels.push_back(std::move(D));
    A_own = std::move(Ac);
    A = dmat(A_own);
    h_rp = std::move(h_rp_c);
    WN_CHECK(download(A_own.ci, A_own.nnzb, h_ci));
    B.swap(Bc);
    bs = 6;
    n = host.levels.back().n_agg;
  }
  // coarsest level on the host (dense Cholesky and inverse)
  {
    std::vector<double> v;
    if (H.levels.empty()) {  // no level was built: the assembled matrix itself
      std::vector<double> raw;
      WN_CHECK(download(s->k64, A.nnzb * bs * bs, raw));
      if (A.stride) {  // component-major -> row-major blocks
        v.resize(raw.size());
        for (int64_t k = 0; k < A.nnzb; ++k)
          for (int e = 0; e < bs * bs; ++e) v[k * bs * bs + e] = raw[e * A.nnzb + k];
      } else {
        v.swap(raw);
      }
      h_rp = s->h_row_ptr;
      h_ci = s->h_col_idx;
    } else {
      WN_CHECK(download(A_own.v64, A.nnzb * bs * bs, v));
    }
    WN_CHECK(dense_coarse(n, bs, h_rp.data(), h_ci.data(), v.data(), host));
    tr.mark("coarse", -1);
  }
  // FP32 copies
  for (size_t l = 0; l < H.levels.size(); ++l) {
    DevLevel& D = H.levels[l];
    if (l > 0) WN_CHECK(fill_float(D.A));
    WN_CHECK(fill_float(D.P));
    WN_CHECK(fill_float(D.R));
    const int64_t nd = D.n_nodes * D.bs;
    WN_CHECK(D.dinv32.alloc(nd));
    ks_to_float<<<grid_n(nd), kT>>>(nd, D.dinv64.p, D.dinv32.p);
    WN_CUDA(cudaGetLastError());
  }
  WN_CUDA(cudaDeviceSynchronize());
  H.device_built = true;
  H.setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

int amg_coarse_block_basis(AmgHierarchy& H, const wn_amg_params& prm) {
  const int nlev = (int)H.levels.size();
  if (nlev < 2) return 0;  // no 6-DOF level with a smoother
  PhaseClock tr("amg_coarse_block_basis");
  // factors of the diagonal blocks of every 6-DOF level (index l >= 1), from the levels as built
  std::vector<DArray<double>> lf(nlev), li(nlev);
  for (int l = 1; l < nlev; ++l) {
    DevLevel& D = H.levels[l];
    WN_REQUIRE(D.bs == 6 && D.A.br == 6, WN_ESTATE, "coarse block basis: level %d is not a 6-DOF level", l);
    WN_CHECK(lf[l].alloc(D.n_nodes * 36));
    WN_CHECK(li[l].alloc(D.n_nodes * 36));
    ks_block_chol<<<grid_n(D.n_nodes), kT>>>(dmat(D.A), lf[l].p, li[l].p);
    WN_CUDA(cudaGetLastError());
  }
  auto rows_of = [&](const DevBsr& M, DArray<int32_t>& row) -> int {
    WN_CHECK(row.alloc(std::max<int64_t>(M.nnzb, 1)));
    ks_block_rows<<<grid_n(M.n_rows), kT>>>(M.n_rows, M.rp.p, row.p);
    WN_CUDA(cudaGetLastError());
    return 0;
  };
  auto refresh_float = [&](DevBsr& M) -> int {
    const int64_t nv = M.nnzb * M.br * M.bc;
    if (nv == 0) return 0;
    ks_to_float<<<grid_n(nv), kT>>>(nv, M.v64.p, M.v32.p);
    WN_CUDA(cudaGetLastError());
    return 0;
  };
  for (int l = 0; l < nlev; ++l) {
    DevLevel& D = H.levels[l];
    const double* lfl = l >= 1 ? lf[l].p : nullptr;
    const double* lic = l + 1 < nlev ? li[l + 1].p : nullptr;
    // the transfer operators P_l (level l+1 -> l) and R_l = P_l^T
    for (int t = 0; t < 2; ++t) {
      DevBsr& M = t == 0 ? D.P : D.R;
      if (M.nnzb == 0) continue;
      DArray<int32_t> row;
      DArray<double> out;
      WN_CHECK(rows_of(M, row));
      WN_CHECK(out.alloc(M.nnzb * M.br * M.bc));
      if (D.bs == 3)
        ks_basis_transfer<3><<<grid_n(M.nnzb), kT>>>(M.nnzb, row.p, M.ci.p, M.v64.p, lfl, lic, t, out.p);
      else
        ks_basis_transfer<6><<<grid_n(M.nnzb), kT>>>(M.nnzb, row.p, M.ci.p, M.v64.p, lfl, lic, t, out.p);
      WN_CUDA(cudaGetLastError());
      std::swap(M.v64, out);
      WN_CHECK(refresh_float(M));
    }
    if (l == 0) continue;
    // the level matrix, its diagonal (1 up to rounding) and rho(D^-1 A^) = rho(D_block^-1 A)
    {
      DArray<int32_t> row;
      DArray<double> out;
      WN_CHECK(rows_of(D.A, row));
      WN_CHECK(out.alloc(std::max<int64_t>(D.A.nnzb, 1) * 36));
      ks_basis_level<<<grid_n(D.A.nnzb), kT>>>(D.A.nnzb, row.p, D.A.ci.p, D.A.v64.p, li[l].p, out.p);
      WN_CUDA(cudaGetLastError());
      std::swap(D.A.v64, out);
      WN_CHECK(refresh_float(D.A));
    }
    const int64_t nd = D.n_nodes * 6;
    const DMat A = dmat(D.A);
    ks_inv_diag<<<grid_n(D.n_nodes), kT>>>(A, D.dinv64.p);
    WN_CUDA(cudaGetLastError());
    ks_to_float<<<grid_n(nd), kT>>>(nd, D.dinv64.p, D.dinv32.p);
    WN_CUDA(cudaGetLastError());
    HostLevel& h = H.host.levels[l];
    WN_CHECK(download(D.dinv64, nd, h.dinv));
    WN_CHECK(power_rho_device(A, D.dinv64, prm.power_iters, &h.rho));
    tr.mark("basis", l);
  }
  WN_CUDA(cudaDeviceSynchronize());
  H.basis_changed = true;
  H.host_synced = false;
  return 0;
}

// Host copies of the device level matrices (for the hierarchy exports)
int amg_sync_host(AmgHierarchy& H) {
  if (!(H.device_built || H.basis_changed) || H.host_synced) return 0;
  for (size_t l = 0; l < H.levels.size() && l < H.host.levels.size(); ++l) {
    DevLevel& D = H.levels[l];
    HostLevel& L = H.host.levels[l];
    auto get = [&](const DevBsr& M, HostBsr& h) -> int {
      h.br = M.br;
      h.bc = M.bc;
      h.n_rows = M.n_rows;
      h.n_cols = M.n_cols;
      WN_CHECK(download(M.rp, M.n_rows + 1, h.rp));
      WN_CHECK(download(M.ci, M.nnzb, h.ci));
      WN_CHECK(download(M.v64, M.nnzb * M.br * M.bc, h.v));
      return 0;
    };
    if (l > 0) WN_CHECK(get(D.A, L.A));
    WN_CHECK(get(D.P, L.P));
    WN_CHECK(get(D.R, L.R));
  }
  H.host_synced = true;
  return 0;
}

}  // namespace wn
