// Host-side construction of the 3x3-block (BSR3) sparsity pattern of a C3D10 mesh, the
// element -> block map and its inverse (the per-block gather lists used by the atomic-free
// assembly kernel).
//
// The reference assembles scalar COO triplets from a 30-DOF node-major template and lets
// scipy sum duplicates (wnfea/solver/solid_solver.py:50-84).  Here the node graph is built
// once: block (i, j) exists iff nodes i and j share an element, columns sorted within each
// row.  Its 3x3 expansion is exactly the reference CSR pattern before BCs.  The map
// emap[e][10a+b] gives the block index of (conn[e][a], conn[e][b]); the gather list of a
// block holds its contributions ordered by (element, a, b), which fixes the summation
// order of every matrix entry and makes assembly bit-reproducible.
#include "pattern.h"

#include <algorithm>
#include <cstdlib>
#include <thread>
#include <vector>

namespace wn {

void parallel_for(int64_t n, int nthreads, const std::function<void(int64_t, int64_t)>& fn) {
  if (nthreads <= 1 || n < 4096) {
    fn(0, n);
    return;
  }
  std::vector<std::thread> th;
  int64_t chunk = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    int64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back(fn, a, b);
  }
  for (auto& x : th) x.join();
}

// host threads for the setup loops: WN_HOST_THREADS when set (read once per process), else the
// hardware concurrency, at most 32.  Every result is the same for any thread count.
int host_threads() {
  static const int forced = [] {
    const char* e = std::getenv("WN_HOST_THREADS");
    return e ? std::atoi(e) : 0;
  }();
  if (forced > 0) return forced < 64 ? forced : 64;
  unsigned h = std::thread::hardware_concurrency();
  if (h == 0) h = 1;
  if (h > 32) h = 32;
  return (int)h;
}

int build_bsr3_pattern(int64_t n_nodes, int64_t n_el, const int32_t* conn, Bsr3Pattern& out) {
  if (n_nodes <= 0 || n_el < 0) return -1;
  for (int64_t k = 0; k < n_el * 10; ++k)
    if (conn[k] < 0 || conn[k] >= n_nodes) return -3;
  if (n_el * 110 >= (int64_t)INT32_MAX) return -8;
  const int nth = host_threads();

  // node -> incident (element, local node) pairs e * 10 + a, elements ascending
  std::vector<int64_t>& inc_ptr = out.inc_ptr;
  inc_ptr.assign(n_nodes + 1, 0);
  for (int64_t k = 0; k < n_el * 10; ++k) inc_ptr[conn[k] + 1]++;
  for (int64_t i = 0; i < n_nodes; ++i) inc_ptr[i + 1] += inc_ptr[i];
  std::vector<int32_t>& inc = out.inc_ea;
  inc.resize(n_el * 10);
  {
    std::vector<int64_t> pos(inc_ptr.begin(), inc_ptr.end() - 1);
    for (int64_t e = 0; e < n_el; ++e)
      for (int a = 0; a < 10; ++a) inc[pos[conn[e * 10 + a]]++] = (int32_t)(e * 10 + a);
  }

  // row i columns = sorted unique nodes of incident elements
  std::vector<std::vector<int32_t>> rows(n_nodes);
  parallel_for(n_nodes, nth, [&](int64_t a, int64_t b) {
    std::vector<int32_t> buf;
    for (int64_t i = a; i < b; ++i) {
      buf.clear();
      for (int64_t k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int32_t* c = conn + (int64_t)(inc[k] / 10) * 10;
        buf.insert(buf.end(), c, c + 10);
      }
      if (buf.empty()) buf.push_back((int32_t)i);  // isolated node: keep a diagonal block
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
      rows[i] = buf;
    }
  });
  out.n_nodes = n_nodes;
  out.row_ptr.assign(n_nodes + 1, 0);
  for (int64_t i = 0; i < n_nodes; ++i) out.row_ptr[i + 1] = out.row_ptr[i] + (int32_t)rows[i].size();
  const int64_t nnzb = out.row_ptr[n_nodes];
  if (nnzb >= (int64_t)INT32_MAX) return -8;
  out.nnzb = nnzb;
  out.col_idx.resize(nnzb);
  out.block_row.resize(nnzb);
  out.diag_block.resize(n_nodes);
  parallel_for(n_nodes, nth, [&](int64_t a, int64_t b) {
    for (int64_t i = a; i < b; ++i) {
      int32_t p = out.row_ptr[i];
      for (size_t k = 0; k < rows[i].size(); ++k) {
        out.col_idx[p + k] = rows[i][k];
        out.block_row[p + k] = (int32_t)i;
        if (rows[i][k] == i) out.diag_block[i] = p + (int32_t)k;
      }
      std::vector<int32_t>().swap(rows[i]);
    }
  });

  // element -> block map by binary search in the sorted row
  out.emap.resize(n_el * 100);
  parallel_for(n_el, nth, [&](int64_t a, int64_t b) {
    for (int64_t e = a; e < b; ++e) {
      const int32_t* c = conn + e * 10;
      for (int ia = 0; ia < 10; ++ia) {
        const int32_t r = c[ia];
        const int32_t* beg = out.col_idx.data() + out.row_ptr[r];
        const int32_t* end = out.col_idx.data() + out.row_ptr[r + 1];
        for (int ib = 0; ib < 10; ++ib) {
          const int32_t* f = std::lower_bound(beg, end, c[ib]);
          out.emap[e * 100 + ia * 10 + ib] = (int32_t)(f - out.col_idx.data());
        }
      }
    }
  });

  // inverse map: per block, contributions in (element, a, b) order.  A contribution names a
  // stored upper-triangle element block (tri index of (min(a,b), max(a,b))) and whether it
  // is used transposed (a > b): src = (e * 55 + tri) * 2 + transposed.
  out.gather_ptr.assign(nnzb + 1, 0);
  for (int64_t k = 0; k < n_el * 100; ++k) out.gather_ptr[out.emap[k] + 1]++;
  for (int64_t k = 0; k < nnzb; ++k) out.gather_ptr[k + 1] += out.gather_ptr[k];
  out.gather_src.resize(n_el * 100);
  {
    std::vector<int32_t> pos(out.gather_ptr.begin(), out.gather_ptr.end() - 1);
    for (int64_t e = 0; e < n_el; ++e)
      for (int ia = 0; ia < 10; ++ia)
        for (int ib = 0; ib < 10; ++ib) {
          const int lo = ia < ib ? ia : ib, hi = ia < ib ? ib : ia;
          const int tri = tri_index(lo, hi);
          const int32_t blk = out.emap[e * 100 + ia * 10 + ib];
          out.gather_src[pos[blk]++] = (int32_t)((e * 55 + tri) * 2 + (ia > ib ? 1 : 0));
        }
  }
  return 0;
}

// Tile-owner assembly plan.  Tiles: whole block rows, at most tile_blocks blocks and tile_rows
// rows each, greedy in row order (the tiling of the streamed fine matrix).
int build_assembly_plan(const Bsr3Pattern& pat, int64_t n_el, int tile_blocks, int tile_rows, int ne_cap,
                        AssemblyPlan& out) {
  out = AssemblyPlan();
  const int64_t n = pat.n_nodes;
  const int32_t* rp = pat.row_ptr.data();
  for (int64_t r = 0; r < n;) {
    const int64_t r0 = r;
    if (rp[r + 1] - rp[r] > tile_blocks) return 1;
    while (r < n && r - r0 < tile_rows && rp[r + 1] - rp[r0] <= tile_blocks) ++r;
    out.tiles.push_back({(int32_t)r0, (int32_t)r, rp[r0], rp[r]});
  }
  const int64_t nt = (int64_t)out.tiles.size();
  if (nt >= (int64_t)INT32_MAX || ne_cap > 256) return 1;
  out.n_tiles = (int)nt;
  // incident elements per tile: the elements of the incidence lists of its rows
  std::vector<std::vector<int32_t>> els(nt);
  std::vector<int> over(nt, 0);
  const int nth = host_threads();
  parallel_for(nt, nth, [&](int64_t a, int64_t b) {
    for (int64_t t = a; t < b; ++t) {
      std::vector<int32_t>& v = els[t];
      for (int64_t q = pat.inc_ptr[out.tiles[t].r0]; q < pat.inc_ptr[out.tiles[t].r1]; ++q) v.push_back(pat.inc_ea[q] / 10);
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      if ((int)v.size() > ne_cap) over[t] = 1;
    }
  });
  for (int64_t t = 0; t < nt; ++t) {
    if (over[t]) return 1;
    out.ne_max = std::max(out.ne_max, (int)els[t].size());
  }
  out.el_ptr.assign(nt + 1, 0);
  for (int64_t t = 0; t < nt; ++t) out.el_ptr[t + 1] = out.el_ptr[t] + (int32_t)els[t].size();
  out.el.resize(out.el_ptr[nt]);
  out.contrib.resize(pat.gather_src.size());
  out.perm.resize(pat.nnzb);
  parallel_for(nt, nth, [&](int64_t a, int64_t b) {
    std::vector<std::pair<int32_t, int32_t>> order;
    for (int64_t t = a; t < b; ++t) {
      const std::vector<int32_t>& v = els[t];
      std::copy(v.begin(), v.end(), out.el.begin() + out.el_ptr[t]);
      const AssemblyTile& T = out.tiles[t];
      order.clear();
      for (int32_t blk = T.b0; blk < T.b1; ++blk) {
        for (int32_t q = pat.gather_ptr[blk]; q < pat.gather_ptr[blk + 1]; ++q) {
          const int32_t src = pat.gather_src[q];  // (e * 55 + tri) * 2 + transposed
          const int32_t e = (src >> 1) / 55, tri = (src >> 1) % 55;
          int lo = 0;
          while (tri_index(lo + 1, lo + 1) <= tri) ++lo;  // tri_index(lo, lo) <= tri < tri_index(lo + 1, lo + 1)
          const int hi = lo + (tri - tri_index(lo, lo));
          const int ea = (src & 1) ? hi : lo, eb = (src & 1) ? lo : hi;
          const int slot = (int)(std::lower_bound(v.begin(), v.end(), e) - v.begin());
          out.contrib[q] = (uint16_t)((slot << 8) | (ea << 4) | eb);
        }
        order.push_back({pat.gather_ptr[blk + 1] - pat.gather_ptr[blk], blk - T.b0});
      }
      std::stable_sort(order.begin(), order.end(), [](const std::pair<int32_t, int32_t>& x,
                                                     const std::pair<int32_t, int32_t>& y) { return x.first > y.first; });
      for (size_t k = 0; k < order.size(); ++k) out.perm[T.b0 + k] = (uint16_t)order[k].second;
    }
  });
  // chunk length: the smallest of the candidates whose chunks fit the kernel's slots in every
  // tile (heavy blocks are the diagonal blocks of vertex nodes; 6 on the structured I-beam)
  int32_t max_count = 0;
  for (int64_t blk = 0; blk < pat.nnzb; ++blk)
    max_count = std::max(max_count, pat.gather_ptr[blk + 1] - pat.gather_ptr[blk]);
  if (max_count > 1023) return 1;  // 10-bit chunk offsets
  const int candidates[] = {6, 8, 12, 16, 24, 32, 48, 63};
  out.chunk_len = 1024;  // no split block
  for (int C : candidates) {
    if (C >= max_count) break;
    int worst = 0;
    for (int64_t t = 0; t < nt && worst <= kAsmChunkSlots; ++t) {
      int nc = 0;
      for (int32_t blk = out.tiles[t].b0; blk < out.tiles[t].b1; ++blk) {
        const int32_t c = pat.gather_ptr[blk + 1] - pat.gather_ptr[blk];
        if (c > C) nc += (c + C - 1) / C;
      }
      worst = std::max(worst, nc);
    }
    if (worst <= kAsmChunkSlots) {
      out.chunk_len = C;
      break;
    }
  }
  out.chunk_ptr.assign(nt + 1, 0);
  out.n_split.assign(nt, 0);
  out.chunks.clear();
  for (int64_t t = 0; t < nt; ++t) {
    const AssemblyTile& T = out.tiles[t];
    out.max_codes = std::max(out.max_codes, pat.gather_ptr[T.b1] - pat.gather_ptr[T.b0]);
    int h = 0;
    for (int32_t k = 0; k < T.b1 - T.b0; ++k) {
      const int32_t j = out.perm[T.b0 + k];
      const int32_t c = pat.gather_ptr[T.b0 + j + 1] - pat.gather_ptr[T.b0 + j];
      if (c <= out.chunk_len) break;  // perm is by descending count: the rest are not split
      ++h;
      // c contributions in n near-equal chunks: the first c % n of them one longer
      const int32_t n = (c + out.chunk_len - 1) / out.chunk_len, base = c / n, extra = c % n;
      int32_t off = 0;
      for (int32_t m = 0; m < n; ++m) {
        const int32_t len = base + (m < extra ? 1 : 0);
        out.chunks.push_back((uint32_t)j | ((uint32_t)off << 9) | ((uint32_t)len << 19) | ((m == 0 ? 1u : 0u) << 25));
        off += len;
      }
    }
    out.n_split[t] = h;
    out.chunk_ptr[t + 1] = (int32_t)out.chunks.size();
    out.max_chunks = std::max(out.max_chunks, out.chunk_ptr[t + 1] - out.chunk_ptr[t]);
  }
  if (out.max_chunks > kAsmChunkSlots) return 1;
  return 0;
}

}  // namespace wn
