// Warp-per-block-row SpMV building block for block-sparse (BSR) matrices on sm_100a.
//
// The values of one block row are contiguous (row-major BR x BC blocks, blocks in column
// order), so a warp streams the whole row as a flat array with 128-bit loads (double2 /
// float4), peeling the unaligned head and tail.  Each element knows its block (for the
// column index), its row r inside the block and its column c, gathers x[col * BC + c]
// through a caller-supplied functor (so fused kernels can build x on the fly) and adds into
// one of BR per-lane accumulators.  A butterfly shuffle leaves the BR row sums in every lane.
// Accumulation is in TACC (FP64 for FP64 values; FP32 for the FP32 inner solver).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wn {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
  __device__ __forceinline__ static void unpack(const double2& v, double* o) {
    o[0] = v.x;
    o[1] = v.y;
  }
};
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
  __device__ __forceinline__ static void unpack(const float4& v, float* o) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  }
};

template <int BR, int BC, typename TACC, typename XF>
__device__ __forceinline__ void accum_elem(int64_t k, TACC a, const int32_t* __restrict__ cols, XF& xf,
                                           TACC (&acc)[BR]) {
  constexpr int BS = BR * BC;
  const int64_t blk = k / BS;
  const int w = (int)(k - blk * BS);
  const int r = w / BC;
  const int c = w - r * BC;
  const TACC xv = xf((int64_t)cols[blk] * BC + c);
#pragma unroll
  for (int rr = 0; rr < BR; ++rr)
    if (rr == r) acc[rr] = fma(a, xv, acc[rr]);
}

// Row sums acc[r] = sum_blocks sum_c A[blk][r][c] * x[col(blk) * BC + c] of block row `row`,
// computed by the calling warp; on return every lane holds all BR sums.
template <int BR, int BC, typename TV, typename TACC, typename XF>
__device__ __forceinline__ void warp_block_row(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col_idx,
                                               const TV* __restrict__ vals, int64_t row, XF xf, TACC (&acc)[BR],
                                               int lane) {
  constexpr int BS = BR * BC;
  constexpr int VW = Vec16<TV>::n;
  using VT = typename Vec16<TV>::type;
#pragma unroll
  for (int r = 0; r < BR; ++r) acc[r] = TACC(0);
  const int64_t s = row_ptr[row];
  const int64_t e = row_ptr[row + 1];
  const int32_t* cols = col_idx + s;
  const int64_t base = s * BS;             // absolute element offset of the row
  const int64_t n = (e - s) * BS;          // elements in the row
  const int64_t abeg = (base + VW - 1) / VW * VW;
  int64_t head = abeg - base;
  if (head > n) head = n;
  const int64_t aend = (base + n) / VW * VW;
  // head (unaligned prefix, < VW elements)
  if (lane < head) accum_elem<BR, BC, TACC>(lane, (TACC)vals[base + lane], cols, xf, acc);
  // aligned body: 16-byte vectors
  if (aend > abeg) {
    const VT* vv = reinterpret_cast<const VT*>(vals + abeg);
    const int64_t nv = (aend - abeg) / VW;
#pragma unroll 4
    for (int64_t q = lane; q < nv; q += 32) {
      const VT pk = __ldg(vv + q);
      TV tmp[VW];
      Vec16<TV>::unpack(pk, tmp);
      const int64_t k0 = abeg - base + q * VW;
#pragma unroll
      for (int u = 0; u < VW; ++u) accum_elem<BR, BC, TACC>(k0 + u, (TACC)tmp[u], cols, xf, acc);
    }
    // tail
    const int64_t tail0 = aend - base;
    if (tail0 + lane < n && tail0 >= head) accum_elem<BR, BC, TACC>(tail0 + lane, (TACC)vals[base + tail0 + lane], cols, xf, acc);
  } else if (n > head) {
    // row shorter than one aligned vector after the head: scalar remainder
    for (int64_t k = head + lane; k < n; k += 32) accum_elem<BR, BC, TACC>(k, (TACC)vals[base + k], cols, xf, acc);
  }
#pragma unroll
  for (int r = 0; r < BR; ++r) {
    TACC v = acc[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[r] = v;
  }
}

// Plain gather functor: x[j] converted to the accumulation type.
template <typename TX, typename TACC>
struct XLoad {
  const TX* __restrict__ x;
  __device__ __forceinline__ TACC operator()(int64_t j) const { return (TACC)x[j]; }
};

}  // namespace wn
