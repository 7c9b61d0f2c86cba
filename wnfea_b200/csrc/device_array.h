// Owning device allocation (cudaMalloc / cudaFree) with size bookkeeping.  Every allocation
// carries kTailSlack bytes beyond its n elements, so a 16-byte-granular bulk copy of a range
// that ends at the last element (rounded up to 16 bytes) stays inside the allocation.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "common.cuh"

namespace wn {

constexpr size_t kTailSlack = 16;

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
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  int alloc(int64_t count) {
    if (count == n && p) return 0;
    release();
    if (count <= 0) return 0;
    WN_CUDA(cudaMalloc((void**)&p, sizeof(T) * (size_t)count + kTailSlack));
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
