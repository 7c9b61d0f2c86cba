// Host-side BSR3 pattern / element-map construction (see pattern.cpp).
#pragma once

#include <stdint.h>

#include <functional>
#include <vector>

namespace wn {

// Upper-triangle index of the element block pair (a, b), 0 <= a <= b < 10: row-major over
// the upper triangle, 55 entries.
inline constexpr int tri_index(int a, int b) { return a * 10 - (a * (a - 1)) / 2 + (b - a); }

struct Bsr3Pattern {
  int64_t n_nodes = 0;
  int64_t nnzb = 0;
  std::vector<int32_t> row_ptr;     // n_nodes + 1
  std::vector<int32_t> col_idx;     // nnzb, sorted within each row
  std::vector<int32_t> block_row;   // nnzb: row of each block
  std::vector<int32_t> diag_block;  // n_nodes: index of block (i, i)
  std::vector<int32_t> emap;        // n_el * 100: block of (conn[e][a], conn[e][b])
  std::vector<int32_t> gather_ptr;  // nnzb + 1
  std::vector<int32_t> gather_src;  // n_el * 100: (e * 55 + tri) * 2 + transposed
  std::vector<int64_t> inc_ptr;     // n_nodes + 1
  std::vector<int32_t> inc_ea;      // n_el * 10: incident (element * 10 + local node), e ascending
};

int build_bsr3_pattern(int64_t n_nodes, int64_t n_el, const int32_t* conn, Bsr3Pattern& out);
int host_threads();
void parallel_for(int64_t n, int nthreads, const std::function<void(int64_t, int64_t)>& fn);

// Plan of the tile-owner assembly (c3d10.cu assemble_tiles_kernel): the block rows are cut into
// the row tiles of the streamed fine matrix; the CTA of a tile computes the Cartesian shape
// derivatives of every element incident to its rows once (shared memory) and then sums each of
// its blocks' contributions, in element order, in registers -- no per-element scratch in
// global memory.
struct AssemblyTile {
  int32_t r0, r1, b0, b1;  // block rows [r0, r1) holding blocks [b0, b1)
};
struct AssemblyPlan {
  int n_tiles = 0;
  int ne_max = 0;                 // most distinct elements incident to one tile
  std::vector<AssemblyTile> tiles;
  std::vector<int32_t> el_ptr;    // n_tiles + 1
  std::vector<int32_t> el;        // the tile's incident elements, ascending
  // per block, its contributions in the gather order (gather_ptr): slot << 8 | a << 4 | b with
  // slot the element's index in its tile's list and (a, b) the element-local node pair
  std::vector<uint16_t> contrib;  // n_el * 100
  // per tile, its local block indices by descending contribution count (lanes of a warp then
  // carry blocks of similar cost): perm[b0 + k] = local index of the k-th block
  std::vector<uint16_t> perm;     // nnzb
  // Blocks with more than chunk_len contributions ("split" blocks; they lead perm) are summed
  // in chunks of at most chunk_len consecutive contributions by different threads and the
  // chunk sums added in chunk order.  Whether a block is split and where its chunks start
  // depend on its contribution count alone, so blocks (i, j) and (j, i) are cut alike.
  int chunk_len = 0;
  int max_chunks = 0;             // most chunks in one tile (<= kAsmChunkSlots)
  int max_codes = 0;              // most contributions in one tile
  std::vector<int32_t> chunk_ptr; // n_tiles + 1
  // per tile, the chunks of its split blocks in perm order: local block | first contribution
  // (offset in the block's list) << 9 | length << 19 | first chunk of its block << 25
  std::vector<uint32_t> chunks;
  std::vector<int32_t> n_split;   // per tile: its split blocks (perm[b0 .. b0 + n_split))
};
// chunk-sum slots of the assembly kernel's shared memory (one per chunk of a tile)
constexpr int kAsmChunkSlots = 32;
// 0: plan made; 1: the row tiles cannot be made (a row over the tile capacity) or a tile has
// more than ne_cap incident elements (the caller keeps the element-scratch assembly).
int build_assembly_plan(const Bsr3Pattern& pat, int64_t n_el, int tile_blocks, int tile_rows, int ne_cap,
                        AssemblyPlan& out);

}  // namespace wn
