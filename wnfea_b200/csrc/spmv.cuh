// Block-row SpMV building block for block-sparse (BSR) matrices on sm_100a.
//
// A group of G lanes (G = 32: one warp; 16 or 8 for matrices with short rows) owns a block
// row; lane l of the group takes blocks s + l, s + l + G, ... .  A lane reads a whole
// BR x BC block with independent loads, its column index and the BC entries of x it
// multiplies, built by a caller-supplied functor (so fused kernels can form x on the fly),
// and accumulates BR row sums with fully unrolled FMAs -- no per-value index arithmetic.  A
// butterfly shuffle inside the group leaves the BR sums in every lane of the group.
//
// Two value layouts:
//   * kAoS -- blocks contiguous (row-major BR x BC, blocks in row order); 16-byte vector
//             loads when every block stays 16-byte aligned (6x6, 3x6/6x3 in FP64, 6x6 FP32);
//   * kSoA -- component-major: component k of block b at vals[k * stride + b].  Consecutive
//             lanes then read consecutive addresses for every component, so each load
//             instruction of the warp is one fully coalesced 128 / 256-byte request.  The
//             assembled fine-level matrix (3x3 blocks, 36 / 72 bytes) is stored this way.
// Accumulation is in TACC (FP64 for FP64 values, FP32 for the FP32 preconditioner).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wn {

enum Layout { kAoS = 0, kSoA = 1 };

template <typename TV, int N>
struct BlockLoad {
  __device__ __forceinline__ static void load(const TV* __restrict__ p, TV (&v)[N]) {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = __ldg(p + k);
  }
};
template <int N>
struct BlockLoadVec {
  __device__ __forceinline__ static void load_d(const double* __restrict__ p, double (&v)[N]) {
    static_assert(N % 2 == 0, "even");
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const double2 t = __ldg(q + k);
      v[2 * k] = t.x;
      v[2 * k + 1] = t.y;
    }
  }
  __device__ __forceinline__ static void load_f(const float* __restrict__ p, float (&v)[N]) {
    static_assert(N % 4 == 0, "multiple of 4");
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int k = 0; k < N / 4; ++k) {
      const float4 t = __ldg(q + k);
      v[4 * k] = t.x;
      v[4 * k + 1] = t.y;
      v[4 * k + 2] = t.z;
      v[4 * k + 3] = t.w;
    }
  }
};
// blocks of 18 / 36 values are 16-byte aligned (144 / 288 bytes FP64, 144 bytes FP32 6x6)
template <>
struct BlockLoad<double, 36> {
  __device__ __forceinline__ static void load(const double* __restrict__ p, double (&v)[36]) {
    BlockLoadVec<36>::load_d(p, v);
  }
};
template <>
struct BlockLoad<double, 18> {
  __device__ __forceinline__ static void load(const double* __restrict__ p, double (&v)[18]) {
    BlockLoadVec<18>::load_d(p, v);
  }
};
// 3x6 / 6x3 FP32 blocks (prolongation / restriction of the fine level): 72 bytes, 8-byte aligned
template <>
struct BlockLoad<float, 18> {
  __device__ __forceinline__ static void load(const float* __restrict__ p, float (&v)[18]) {
    const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float2 t = __ldg(q + k);
      v[2 * k] = t.x;
      v[2 * k + 1] = t.y;
    }
  }
};
template <>
struct BlockLoad<float, 36> {
  __device__ __forceinline__ static void load(const float* __restrict__ p, float (&v)[36]) {
    BlockLoadVec<36>::load_f(p, v);
  }
};

// Row sums acc[r] = sum_blocks sum_c A[blk][r][c] * x[col(blk) * BC + c] of block row `row`
// (when `active`), computed by the calling group of G lanes; every lane of the group must
// call (the shuffles use the full warp mask).  gl = lane index inside the group.
template <int BR, int BC, int G, Layout L, typename TV, typename TACC, typename XF>
__device__ __forceinline__ void group_block_row(const int32_t* __restrict__ row_ptr,
                                                const int32_t* __restrict__ col_idx, const TV* __restrict__ vals,
                                                int64_t stride, int64_t row, bool active, XF xf, TACC (&acc)[BR],
                                                int gl) {
  constexpr int BS = BR * BC;
#pragma unroll
  for (int r = 0; r < BR; ++r) acc[r] = TACC(0);
  int32_t s = 0, e = 0;
  if (active) {
    s = __ldg(row_ptr + row);
    e = __ldg(row_ptr + row + 1);
  }
  for (int32_t b = s + gl; b < e; b += G) {
    const int64_t col = __ldg(col_idx + b);
    TV v[BS];
    if constexpr (L == kSoA) {
#pragma unroll
      for (int k = 0; k < BS; ++k) v[k] = __ldg(vals + (int64_t)k * stride + b);
    } else {
      BlockLoad<TV, BS>::load(vals + (int64_t)b * BS, v);
    }
    TACC xv[BC];
#pragma unroll
    for (int c = 0; c < BC; ++c) xv[c] = xf(col * BC + c);
#pragma unroll
    for (int r = 0; r < BR; ++r)
#pragma unroll
      for (int c = 0; c < BC; ++c) acc[r] = fma((TACC)v[r * BC + c], xv[c], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < BR; ++r) {
    TACC t = acc[r];
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    acc[r] = t;
  }
}

// One warp per block row (G = 32).
template <int BR, int BC, Layout L, typename TV, typename TACC, typename XF>
__device__ __forceinline__ void warp_block_row(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col_idx,
                                               const TV* __restrict__ vals, int64_t stride, int64_t row, XF xf,
                                               TACC (&acc)[BR], int lane) {
  group_block_row<BR, BC, 32, L, TV, TACC>(row_ptr, col_idx, vals, stride, row, true, xf, acc, lane);
}

// Plain gather functor: x[j] converted to the accumulation type.
template <typename TX, typename TACC>
struct XLoad {
  const TX* __restrict__ x;
  __device__ __forceinline__ TACC operator()(int64_t j) const { return (TACC)x[j]; }
};

}  // namespace wn
