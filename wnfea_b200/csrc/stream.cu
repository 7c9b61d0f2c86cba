// StreamMat: tile plans and tile-major packs of block-sparse matrices for the streamed kernels.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "stream_mat.h"

namespace wn {

template <int BR, int BC>
static int plan_shape(StreamMat& m, const int32_t* h_rp, int64_t n_rows) {
  using C32 = typename StreamDefault<float, BR, BC>::type;
  using C64 = typename StreamDefault<double, BR, BC>::type;
  static_assert(C32::kCap == C64::kCap && C32::kRowCap == C64::kRowCap, "one plan serves both precisions");
  std::vector<StreamTile> plan;
  std::vector<PackTile> d32, d64;
  if (!build_stream_tiles(h_rp, n_rows, plan, C32::kCap, C32::kRowCap) || plan.empty() ||
      plan.size() >= (size_t)INT32_MAX)
    return 0;
  const int64_t b32 = build_pack_tiles<float, BR * BC>(plan, d32);
  const int64_t b64 = build_pack_tiles<double, BR * BC>(plan, d64);
  if (b32 <= 0 || b64 <= 0) return 0;
  if constexpr (BR == 3 && BC == 3) {
    std::vector<PackTile> d16;
    const int64_t b16 = build_pack_tiles<__half, 9>(plan, d16);
    if (b16 > 0) {
      WN_CHECK(m.d16.upload(d16));
      m.size16 = b16;
    }
  }
  WN_CHECK(m.plan.upload(plan));
  WN_CHECK(m.d32.upload(d32));
  WN_CHECK(m.d64.upload(d64));
  m.size32 = b32;
  m.size64 = b64;
  m.n_tiles = (int)plan.size();
  return 0;
}

void StreamMat::clear() {
  ++epoch;
  n_tiles = 0;
  packed = false;
  structure = false;
  plan.release();
  d32.release();
  d64.release();
  p32.release();
  p64.release();
  d16.release();
  p16.release();
  size32 = size64 = size16 = 0;
  version16 = ~0ull;
}

int StreamMat::pack_half33(const int32_t* rp, const int32_t* ci, const int32_t* block_row, const double* v64,
                           int64_t stride, const double* scale, uint64_t version, cudaStream_t st) {
  WN_REQUIRE(br == 3 && bc == 3 && n_tiles > 0 && size16 > 0, WN_ESTATE, "FP16 pack: no 3x3 tile plan");
  const unsigned char* old = p16.p;
  WN_CHECK(p16.alloc(size16));
  if (p16.p != old) ++epoch;
  const int grid = std::min(n_tiles, kNumSMs * 8);
  k_pack_half33<<<grid, 256, 0, st>>>(n_tiles, plan.p, d16.p, rp, ci, block_row, v64, stride, scale, p16.p);
  WN_CUDA(cudaGetLastError());
  version16 = version;
  return 0;
}

int StreamMat::make_plan(const int32_t* h_rp, int64_t n_rows, int br_, int bc_) {
  clear();
  br = br_;
  bc = bc_;
  if (br == 3 && bc == 3) return plan_shape<3, 3>(*this, h_rp, n_rows);
  if (br == 6 && bc == 6) return plan_shape<6, 6>(*this, h_rp, n_rows);
  if (br == 3 && bc == 6) return plan_shape<3, 6>(*this, h_rp, n_rows);
  if (br == 6 && bc == 3) return plan_shape<6, 3>(*this, h_rp, n_rows);
  return 0;
}

template <int NV>
static int pack_shape(StreamMat& m, const int32_t* rp, const int32_t* ci, const float* v32, const double* v64,
                      int64_t stride, cudaStream_t st) {
  const int grid = std::min(m.n_tiles, kNumSMs * 8);
  k_pack_tiles<float, NV><<<grid, 256, 0, st>>>(m.n_tiles, m.plan.p, m.d32.p, rp, ci, v32, stride, m.p32.p);
  k_pack_tiles<double, NV><<<grid, 256, 0, st>>>(m.n_tiles, m.plan.p, m.d64.p, rp, ci, v64, stride, m.p64.p);
  WN_CUDA(cudaGetLastError());
  return 0;
}

int StreamMat::pack(const int32_t* rp, const int32_t* ci, const float* v32, const double* v64, int64_t stride,
                    cudaStream_t st) {
  packed = false;
  if (n_tiles == 0) return 0;
  const unsigned char *old32 = p32.p, *old64 = p64.p;
  WN_CHECK(p32.alloc(size32));
  WN_CHECK(p64.alloc(size64));
  if (p32.p != old32 || p64.p != old64) ++epoch;
  const int nv = br * bc;
  if (nv == 9) WN_CHECK(pack_shape<9>(*this, rp, ci, v32, v64, stride, st));
  else if (nv == 36) WN_CHECK(pack_shape<36>(*this, rp, ci, v32, v64, stride, st));
  else if (nv == 18) WN_CHECK(pack_shape<18>(*this, rp, ci, v32, v64, stride, st));
  else return 0;
  packed = true;
  structure = true;
  return 0;
}

}  // namespace wn
