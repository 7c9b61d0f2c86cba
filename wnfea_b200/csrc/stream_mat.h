// A block-sparse matrix prepared for the streamed kernels (stream.cuh): its tile plan, the
// segment descriptors of its FP32 and FP64 tile-major packs (and, for 3x3 blocks, of an FP16
// pack of the equilibrated matrix), and the packs themselves.  The
// plan depends on the pattern only (made once); the packs are refreshed whenever the values
// change.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_array.h"
#include "stream.cuh"

namespace wn {

struct StreamMat {
  int br = 0, bc = 0;
  int n_tiles = 0;  // 0: not streamed (a row exceeds the tile capacity, or no plan made)
  DArray<StreamTile> plan;
  DArray<PackTile> d32, d64;
  DArray<unsigned char> p32, p64;
  int64_t size32 = 0, size64 = 0;
  bool packed = false;  // the packs hold the current values
  bool structure = false;  // the packs hold the column indices and row starts (set by pack())
  StreamCtl ctl;         // wait limit of the streamed kernels on this matrix (and the test hook)
  // changes whenever the plan or pack buffers are released or reallocated: a captured graph
  // holds their addresses and is replayed only while the epoch it was captured at is current
  uint64_t epoch = 0;
  // Tile plan and descriptors of a br x bc matrix from its host row pointer (shapes 3x3, 6x6,
  // 3x6, 6x3; others are left unstreamed).  Packs are allocated by pack().
  int make_plan(const int32_t* h_rp, int64_t n_rows, int br, int bc);
  // Pack the device values (component-major with the given stride, or block-contiguous when
  // stride == 0) into both packs; a no-op without a plan.
  int pack(const int32_t* rp, const int32_t* ci, const float* v32, const double* v64, int64_t stride,
           cudaStream_t st);
  // 3x3 matrices: the FP16 pack of the equilibrated matrix S A S (k_pack_half33) for the FP16
  // V-cycle, built on demand and tagged with the values version it was built from
  DArray<PackTile> d16;
  DArray<unsigned char> p16;
  int64_t size16 = 0;
  uint64_t version16 = ~0ull;
  int pack_half33(const int32_t* rp, const int32_t* ci, const int32_t* block_row, const double* v64, int64_t stride,
                  const double* scale, uint64_t version, cudaStream_t st);
  // drop the plan and packs (the matrix is then run by the register kernels)
  void clear();
};

}  // namespace wn
