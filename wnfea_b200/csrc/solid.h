// The device-resident C3D10 system behind an opaque C-ABI handle: mesh, BSR3 pattern,
// element -> block map and gather lists, assembled FP64 / FP32 values, Dirichlet mask, the
// AMG hierarchy and the solver workspace.
#pragma once

#include <memory>
#include <mutex>
#include <vector>

#include "device_array.h"
#include "pattern.h"
#include "stream_mat.h"

namespace wn {

struct AmgHierarchy;  // amg.h
struct SolverWork;    // solver.cu
struct BlockWork;     // block.h

constexpr int kStreamStatusWord = 8;

struct Solid {
  int device = 0;
  int64_t n_nodes = 0, n_el = 0, nnzb = 0;
  // DOFs per node: 3 for the C3D10 system (component-major 3x3 values), 6 for a linear
  // beam-frame system made by wn_bsr6_system_create / wn_beam_linear_system (block-contiguous
  // 6x6 values); only the AMG and the single-RHS solve accept bs = 6
  int bs = 3;
  // host copies kept for the CSR/BSR export and the AMG setup
  std::vector<int32_t> h_row_ptr, h_col_idx, h_diag_block;
  std::vector<double> h_nodes;
  std::vector<uint8_t> h_fixed;
  // device mesh
  DArray<double> nodes;     // n_nodes x 3
  DArray<int32_t> conn;     // n_el x 10
  DArray<double> props;     // n_el x 2  [E, nu]
  // pattern + maps
  DArray<int32_t> row_ptr, col_idx, block_row, diag_block;
  DArray<int32_t> emap, gptr, gsrc;  // gsrc: only for the element-scratch assembly (no plan)
  // tile-owner assembly plan (pattern.h AssemblyPlan); asm_tiles == 0: element-scratch assembly
  int asm_tiles = 0, asm_ne_max = 0, asm_max_codes = 0;
  DArray<int32_t> asm_tile, asm_hdr, asm_el;
  DArray<uint16_t> asm_perm, asm_contrib;
  DArray<uint32_t> asm_chunks;
  DArray<int64_t> inc_ptr;
  DArray<int32_t> inc_ea;
  // values
  DArray<uint8_t> fixed;    // 3 n_nodes (0/1)
  DArray<double> k64;       // nnzb x 9
  DArray<float> k32;        // nnzb x 9
  DArray<double> ke;        // scratch: n_el x 55 x 9 element blocks
  DArray<double> fe;        // scratch: n_el x 30 element forces
  DArray<int> flags;        // device status words ([kStreamStatusWord]: streamed SpMV)
  // the fine matrix prepared for the streamed kernels (stream.cuh): tile plan made with the
  // pattern, FP32 / FP64 tile-major packs refreshed by every assembly
  StreamMat fine;
  bool stream_fine = true;  // wn_solid_set_stream: plan and packs kept (else the register kernels)
  bool stream_batched = false;  // wn_solid_set_stream(2): the batched solves stream the fine level too
  bool batch_stage_x = false;   // wn_solid_set_batch_staging: batched fine level with x staged per tile
  bool assembled = false;
  bool bcs_applied = false;
  uint64_t values_version = 0;  // bumped whenever the matrix values change (the FP16 pack's tag)
  std::unique_ptr<AmgHierarchy> amg;
  std::unique_ptr<SolverWork> work;
  std::unique_ptr<BlockWork> bwork;
  // host-buffer solve: device copies of F / u and a page-locked staging buffer (2 n), kept
  // between calls so that a call neither allocates nor copies from pageable memory; one event
  // per staged chunk of the result (its copy out of the staging buffer waits for that chunk only)
  DArray<double> io_f, io_u;
  PinnedArray<double> io_pin;
  std::vector<cudaEvent_t> io_ev;
  ~Solid();
};

}  // namespace wn
