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

}  // namespace wn
