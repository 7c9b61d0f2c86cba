// Owning device allocation with size bookkeeping.  Every allocation carries kTailSlack bytes
// beyond its n elements, so a 16-byte-granular bulk copy of a range that ends at the last
// element (rounded up to 16 bytes) stays inside the allocation.
//
// Allocations come from the device's default stream-ordered memory pool, which keeps up to
// kPoolKeepBytes of freed memory mapped for reuse: plain cudaMalloc / cudaFree of the large
// hierarchy and pack buffers map and unmap memory each time, and single calls of the AMG setup
// took 0.1-0.9 s that way.  release() waits for the device before it frees, as cudaFree does,
// so no stream can still be using a buffer when it returns to the pool.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <utility>
#include <vector>

#include "common.cuh"

namespace wn {

constexpr size_t kTailSlack = 16;
constexpr uint64_t kPoolKeepBytes = 4ull << 30;

// once per device: the default pool keeps kPoolKeepBytes of freed memory instead of unmapping it
inline void pool_keep_memory() {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || (done.load() >> dev) & 1ull) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = kPoolKeepBytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done.fetch_or(1ull << dev);
}

template <typename T>
struct DArray {
  T* p = nullptr;
  int64_t n = 0;
  DArray() = default;
  DArray(const DArray&) = delete;
  DArray& operator=(const DArray&) = delete;
  DArray(DArray&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DArray& operator=(DArray&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DArray() { release(); }
  void release() {
    if (p) {
      cudaDeviceSynchronize();
      cudaFreeAsync(p, 0);
    }
    p = nullptr;
    n = 0;
  }
  int alloc(int64_t count) {
    if (count == n && p) return 0;
    release();
    if (count <= 0) return 0;
    pool_keep_memory();
    WN_CUDA(cudaMallocAsync((void**)&p, sizeof(T) * (size_t)count + kTailSlack, 0));
    n = count;
    return 0;
  }
  int zero(cudaStream_t st = 0) {
    if (n) WN_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, st));
    return 0;
  }
  int upload(const T* h, int64_t count, cudaStream_t st = 0) {
    WN_CHECK(alloc(count));
    if (count) WN_CUDA(cudaMemcpyAsync(p, h, sizeof(T) * (size_t)count, cudaMemcpyHostToDevice, st));
    return 0;
  }
  int upload(const std::vector<T>& h, cudaStream_t st = 0) { return upload(h.data(), (int64_t)h.size(), st); }
  size_t bytes() const { return sizeof(T) * (size_t)n; }
};

// Page-locked host buffer (cudaMallocHost), grown on demand, for full-speed staging copies.
template <typename T>
struct PinnedArray {
  T* p = nullptr;
  int64_t n = 0;
  PinnedArray() = default;
  PinnedArray(const PinnedArray&) = delete;
  PinnedArray& operator=(const PinnedArray&) = delete;
  ~PinnedArray() {
    if (p) cudaFreeHost(p);
  }
  int at_least(int64_t count) {
    if (p && n >= count) return 0;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    WN_CUDA(cudaMallocHost((void**)&p, sizeof(T) * (size_t)count));
    n = count;
    return 0;
  }
};

}  // namespace wn
