// Warp-per-block-row SpMV building block for block-sparse (BSR) matrices on sm_100a.
//
// One warp owns a block row; lane l takes blocks s + l, s + l + 32, ... of the row.  A lane
// reads a whole BR x BC block (contiguous, row-major) with independent loads -- 16-byte
// vector loads when the block size keeps every block 16-byte aligned (6x6, 3x6, 6x3 in
// FP64/FP32), 8/4-byte loads for the 72/36-byte 3x3 blocks -- plus its column index and
// the BC entries of x it multiplies, built by a caller-supplied functor (so fused kernels
// can form x on the fly).  There is no per-value index arithmetic: the BR x BC FMAs are
// fully unrolled into BR per-lane accumulators, and a butterfly shuffle leaves the BR row
// sums in every lane.  Consecutive lanes read consecutive blocks, so a warp streams the
// row's values as one contiguous range.  Accumulation is in TACC (FP64 for FP64 values,
// FP32 for the FP32 preconditioner).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wn {

template <typename TV, int N>
struct BlockLoad {
  // generic: N scalar loads through the read-only path
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
// blocks of 18 / 36 values are 16-byte aligned in both precisions (144 / 288 / 72 / 144 bytes)
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
template <>
struct BlockLoad<float, 36> {
  __device__ __forceinline__ static void load(const float* __restrict__ p, float (&v)[36]) {
    BlockLoadVec<36>::load_f(p, v);
  }
};

// Row sums acc[r] = sum_blocks sum_c A[blk][r][c] * x[col(blk) * BC + c] of block row `row`,
// computed by the calling warp; on return every lane holds all BR sums.
template <int BR, int BC, typename TV, typename TACC, typename XF>
__device__ __forceinline__ void warp_block_row(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col_idx,
                                               const TV* __restrict__ vals, int64_t row, XF xf, TACC (&acc)[BR],
                                               int lane) {
  constexpr int BS = BR * BC;
#pragma unroll
  for (int r = 0; r < BR; ++r) acc[r] = TACC(0);
  const int32_t s = __ldg(row_ptr + row);
  const int32_t e = __ldg(row_ptr + row + 1);
  for (int32_t b = s + lane; b < e; b += 32) {
    const int64_t col = __ldg(col_idx + b);
    TV v[BS];
    BlockLoad<TV, BS>::load(vals + (int64_t)b * BS, v);
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
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    acc[r] = t;
  }
}

// Plain gather functor: x[j] converted to the accumulation type.
template <typename TX, typename TACC>
struct XLoad {
  const TX* __restrict__ x;
  __device__ __forceinline__ TACC operator()(int64_t j) const { return (TACC)x[j]; }
};

}  // namespace wn
