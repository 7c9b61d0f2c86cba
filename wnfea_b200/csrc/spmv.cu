// Stand-alone BSR SpMV kernels y = alpha * A x + beta * y for the block shapes of the solve
// path (3x3 solid, 6x6 beam / coarse levels, 3x6 prolongation, 6x3 restriction), FP64
// values with FP64 accumulation and FP32 values with FP32 accumulation.  One warp per
// block row (16 lanes for the FP32 fine matrix), one resident wave of CTAs (grid-stride).
#include "common.cuh"
#include "kernels.h"
#include "spmv.cuh"
#include "stream.cuh"

namespace wn {

template <int BR, int BC, int G, Layout L, typename T>
__global__ void __launch_bounds__(256) bsr_spmv_kernel(int64_t n_rows, const int32_t* __restrict__ row_ptr,
                                                       const int32_t* __restrict__ col_idx, const T* __restrict__ vals,
                                                       int64_t stride, const T* __restrict__ x, T* __restrict__ y,
                                                       T alpha, T beta) {
  constexpr int RPW = 32 / G;  // block rows per warp
  const int gl = (threadIdx.x & 31) % G, grp = (threadIdx.x & 31) / G;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t rb = warp; rb * RPW < n_rows; rb += nwarps) {
    const int64_t row = rb * RPW + grp;
    const bool active = row < n_rows;
    T acc[BR];
    group_block_row<BR, BC, G, L, T, T>(row_ptr, col_idx, vals, stride, row, active, XLoad<T, T>{x}, acc, gl);
    if (active && gl < BR) {
      T v = acc[0];
#pragma unroll
      for (int r = 1; r < BR; ++r)
        if (gl == r) v = acc[r];
      const int64_t o = row * BR + gl;
      y[o] = (beta == T(0)) ? alpha * v : alpha * v + beta * y[o];
    }
  }
}

// Fine 3x3 matrix (rows of ~25 blocks): 16 lanes per row in FP32, a full warp in FP64
// (measured on the 1M-DOF I-beam: FP32 89 us with 16 lanes vs 92 with 32 and 95 with 8; FP64
// 129 us with 32 lanes vs 145 with 16); a full warp for the other shapes.
template <int BR, int BC, typename T, Layout L = kAoS, int G = 32>
static int launch(int64_t n_rows, const int32_t* rp, const int32_t* ci, const T* v, const T* x, T* y, T a, T b,
                  cudaStream_t st, int64_t stride = 0) {
  if (n_rows == 0) return 0;
  const int grid = resident_grid(bsr_spmv_kernel<BR, BC, G, L, T>, 256, (n_rows * G + 255) / 256);
  bsr_spmv_kernel<BR, BC, G, L, T><<<grid, 256, 0, st>>>(n_rows, rp, ci, v, stride, x, y, a, b);
  WN_CUDA(cudaGetLastError());
  return 0;
}

// y = A x on the fine 3x3 matrix streamed through shared memory (stream.cuh)
template <typename T>
struct EpiY {
  T* __restrict__ y;
  struct Pre {};
  __device__ __forceinline__ Pre load(int64_t) const { return {}; }
  __device__ __forceinline__ double store(int64_t i, const Pre&, T t) const {
    y[i] = t;
    return 0.0;
  }
};

template <typename T>
__global__ void __launch_bounds__(kStreamThreads, (StreamDefault<T, 3, 3>::kCtasPerSm)) k_stream_spmv(const PackTile* __restrict__ tiles, int n_tiles,
                                                                   const unsigned char* __restrict__ pack,
                                                                   const T* __restrict__ x, T* __restrict__ y,
                                                                   int* __restrict__ status, StreamCtl ctl) {
  extern __shared__ __align__(128) unsigned char smem[];
  stream_rows<T, 3, 3, typename StreamDefault<T, 3, 3>::type>(tiles, n_tiles, pack, XLoad<T, T>{x}, EpiY<T>{y},
                                                               smem, status, nullptr, ctl);
}

template <typename T>
static int launch_stream(const PackTile* tiles, int n_tiles, const unsigned char* pack, const T* x, T* y, int* status,
                         StreamCtl ctl, cudaStream_t st) {
  if (!tiles || !pack || n_tiles == 0) return 0;
  auto kern = k_stream_spmv<T>;
  const int per_sm =
      stream_ctas_per_sm(reinterpret_cast<const void*>(kern), kStreamThreads, stream_smem_bytes<T, 3, 3>());
  if (per_sm < 1) return 0;
  const int grid = std::max(1, std::min(n_tiles, kNumSMs * per_sm));
  kern<<<grid, kStreamThreads, stream_smem_bytes<T, 3, 3>(), st>>>(tiles, n_tiles, pack, x, y, status, ctl);
  WN_CUDA(cudaGetLastError());
  return 1;
}

int launch_solid_spmv_stream(int precision, const PackTile* tiles, int n_tiles, const unsigned char* pack,
                             const void* x, void* y, int* status, unsigned long long wait_ns, int withhold,
                             cudaStream_t st) {
  StreamCtl ctl;
  ctl.wait_ns = wait_ns;
  ctl.withhold = withhold;
  if (precision == 0)
    return launch_stream<double>(tiles, n_tiles, pack, (const double*)x, (double*)y, status, ctl, st);
  return launch_stream<float>(tiles, n_tiles, pack, (const float*)x, (float*)y, status, ctl, st);
}

int launch_solid_spmv_f64(int64_t n_rows, const int32_t* rp, const int32_t* ci, const double* v, int64_t nnzb,
                          const double* x, double* y, cudaStream_t st) {
  return launch<3, 3, double, kSoA, 32>(n_rows, rp, ci, v, x, y, 1.0, 0.0, st, nnzb);
}

int launch_solid_spmv_f32(int64_t n_rows, const int32_t* rp, const int32_t* ci, const float* v, int64_t nnzb,
                          const float* x, float* y, cudaStream_t st) {
  return launch<3, 3, float, kSoA, 16>(n_rows, rp, ci, v, x, y, 1.0f, 0.0f, st, nnzb);
}

int launch_bsr_spmv_f64(int br, int bc, int64_t n_rows, const int32_t* rp, const int32_t* ci, const double* v,
                        const double* x, double* y, double alpha, double beta, cudaStream_t st) {
  if (br == 3 && bc == 3) return launch<3, 3, double>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  if (br == 6 && bc == 6) return launch<6, 6, double>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  if (br == 3 && bc == 6) return launch<3, 6, double>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  if (br == 6 && bc == 3) return launch<6, 3, double>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  set_error("unsupported block shape %dx%d", br, bc);
  return WN_EINVAL;
}

int launch_bsr_spmv_f32(int br, int bc, int64_t n_rows, const int32_t* rp, const int32_t* ci, const float* v,
                        const float* x, float* y, float alpha, float beta, cudaStream_t st) {
  if (br == 3 && bc == 3) return launch<3, 3, float>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  if (br == 6 && bc == 6) return launch<6, 6, float>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  if (br == 3 && bc == 6) return launch<3, 6, float>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  if (br == 6 && bc == 3) return launch<6, 3, float>(n_rows, rp, ci, v, x, y, alpha, beta, st);
  set_error("unsupported block shape %dx%d", br, bc);
  return WN_EINVAL;
}

}  // namespace wn
