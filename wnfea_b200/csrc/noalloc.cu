// Element stiffness for callers that must not allocate device memory.
//
// wn_c3d10_element_stiffness allocates its device buffers (inputs, the per-element
// upper-triangle scratch, the output) on every call.  Some callers cannot do that: code
// whose device memory is owned by another allocator (a framework's caching allocator or a
// pool sized once at start-up, where an extra cudaMalloc can fail or fragment the pool), and
// latency-bound loops that cannot absorb the device-wide synchronisation of cudaFree.  This
// variant takes device inputs and a device output from the caller and keeps its only scratch
// -- the 55 upper-triangle 3x3 blocks of each element's Ke plus one status word -- in a
// fixed, file-scope device array, so the call itself allocates nothing.
#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "pattern.h"
#include "wnfea_cuda.h"

namespace wn {
namespace {

constexpr int64_t kNoAllocMaxElements = WN_NOALLOC_MAX_ELEMENTS;
constexpr int64_t kHeaderDoubles = 32;  // 256 bytes: status word, keeps the block region aligned
constexpr int64_t kScratchDoubles = kHeaderDoubles + kNoAllocMaxElements * 55 * 9;

// Shared by every call on a device and kept until the process exits (about 8.1 MB).
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch per device ordinal, looked up once per device (the first
// call on each device, with that device current).  The element kernel's constant tables are
// statically initialised, so this lookup is the only set-up.
static std::mutex g_mutex;
static void* g_scratch_addr[64] = {nullptr};

int scratch_address(double** out) {
  int dev = 0;
  WN_CUDA(cudaGetDevice(&dev));
  WN_REQUIRE(dev >= 0 && dev < 64, WN_EINVAL, "wn_c3d10_element_stiffness_noalloc: device ordinal %d >= 64", dev);
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_error("wn_c3d10_element_stiffness_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return (int)e;
    }
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<double*>(g_scratch_addr[dev]);
  return 0;
}

// Full symmetric Ke (n_el x 30 x 30) from the stored upper-triangle blocks.
__global__ void expand_upper_kernel(int64_t n_el, const double* __restrict__ upper, double* __restrict__ Ke) {
  const int64_t total = n_el * 900;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / 900;
    const int rc = (int)(t - e * 900);
    const int row = rc / 30, col = rc - (rc / 30) * 30;
    int a = row / 3, i = row - (row / 3) * 3;
    int b = col / 3, j = col - (col / 3) * 3;
    if (a > b) {  // lower triangle: transposed upper block
      int s = a;
      a = b;
      b = s;
      s = i;
      i = j;
      j = s;
    }
    Ke[t] = upper[(e * 55 + tri_index(a, b)) * 9 + i * 3 + j];
  }
}

}  // namespace
}  // namespace wn

using namespace wn;

extern "C" int wn_c3d10_element_stiffness_noalloc(int64_t n_el, int64_t n_nodes, const double* d_nodes,
                                                   const int32_t* d_conn, const double* d_props, double* d_Ke,
                                                   uintptr_t stream) {
  WN_REQUIRE(n_el >= 0 && n_nodes >= 0, WN_EINVAL, "wn_c3d10_element_stiffness_noalloc: negative size");
  WN_REQUIRE(n_el <= kNoAllocMaxElements, WN_ETOOBIG,
             "wn_c3d10_element_stiffness_noalloc: %lld elements exceed the fixed scratch capacity of %lld; "
             "split the batch or use wn_c3d10_element_stiffness",
             (long long)n_el, (long long)kNoAllocMaxElements);
  if (n_el == 0) return 0;
  WN_REQUIRE(d_nodes && d_conn && d_props && d_Ke, WN_EINVAL, "wn_c3d10_element_stiffness_noalloc: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  double* scratch = nullptr;
  WN_CHECK(scratch_address(&scratch));
  int* status = reinterpret_cast<int*>(scratch);  // header: error bits, cleared per call
  double* upper = scratch + kHeaderDoubles;
  WN_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
  // the element kernel checks every node index against n_nodes before it reads coordinates
  WN_CHECK(launch_ke_upper(n_el, n_nodes, d_nodes, d_conn, d_props, upper, status, st));
  expand_upper_kernel<<<grid_for(n_el * 900, 1, 256, 8), 256, 0, st>>>(n_el, upper, d_Ke);
  WN_CUDA(cudaGetLastError());
  int flag = 0;
  WN_CUDA(cudaMemcpyAsync(&flag, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  WN_REQUIRE(!(flag & 2), WN_EINVAL,
             "wn_c3d10_element_stiffness_noalloc: a connectivity entry lies outside [0, n_nodes = %lld)",
             (long long)n_nodes);
  WN_REQUIRE(flag == 0, WN_EMESH, "wn_c3d10_element_stiffness_noalloc: non-positive Jacobian determinant");
  return 0;
}
