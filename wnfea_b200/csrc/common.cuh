// Shared helpers for the sm_100a kernels of libwnfea_cuda: status codes, error capture,
// warp reductions and launch sizing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "wnfea_cuda.h"

namespace wn {

// Status codes (WN_OK, WN_EINVAL, ...) are the macros of the public header.


void set_error(const char* fmt, ...);
const char* last_error();

}  // namespace wn

#define WN_CUDA(call)                                                                \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess) {                                                         \
      wn::set_error("%s:%d: %s (%s)", __FILE__, __LINE__, cudaGetErrorString(_e), #call); \
      return (int)_e;                                                                \
    }                                                                                \
  } while (0)

#define WN_CHECK(status)          \
  do {                            \
    int _s = (status);            \
    if (_s != 0) return _s;       \
  } while (0)

#define WN_REQUIRE(cond, code, ...)  \
  do {                               \
    if (!(cond)) {                   \
      wn::set_error(__VA_ARGS__);    \
      return (code);                 \
    }                                \
  } while (0)

namespace wn {

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;  // B200; grids are sized in multiples of this

#if defined(__CUDACC__)
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of one double per thread; result valid in thread 0.  `sh` needs
// blockDim.x / 32 doubles.  Fixed reduction order -> deterministic.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    r = lane < nw ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

// Grid of at most one full wave: blocks resident on all SMs at once for `kernel` with
// `threads` threads per CTA (occupancy queried once per kernel), capped by the work.
int occupancy_per_sm(const void* kernel, int threads);  // cached per (kernel, threads), capi.cu
int stream_ctas_per_sm(const void* kernel, int threads, size_t smem);  // capi.cu

template <typename K>
inline int resident_grid(K kernel, int threads, int64_t work_ctas) {
  const int per_sm = occupancy_per_sm(reinterpret_cast<const void*>(kernel), threads);
  int64_t g = (int64_t)kNumSMs * per_sm;
  if (work_ctas < g) g = work_ctas;
  return g < 1 ? 1 : (int)g;
}

#endif  // __CUDACC__

inline int grid_for(int64_t work_items, int threads_per_item_group, int block, int max_waves = 16) {
  int64_t blocks = (work_items * threads_per_item_group + block - 1) / block;
  int64_t cap = (int64_t)kNumSMs * max_waves;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

}  // namespace wn
