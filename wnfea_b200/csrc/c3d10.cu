// C3D10 element kernels for sm_100a:
//   * stiffness of every element (upper-triangle 3x3 blocks) into a scratch buffer,
//   * atomic-free gather of those blocks into the BSR3 matrix through the element->block
//     map's inverse, with Dirichlet rows/columns applied in the same pass,
//   * matrix-free internal force / strain energy (adjoint) and Gauss-point stresses.
//
// Element math restates wnfea/elements/c3d10.py:219-318.  Ke entries use the isotropic
// closed form K_ab[i][j] = sum_g w|J| (lam a_i b_j + mu a_j b_i + mu delta_ij a.b) with
// a = dN_a/dx, b = dN_b/dx, which equals (B^T C B)[3a+i][3b+j] of c3d10.py:244-246; only
// a <= b is computed and K_ba = K_ab^T, so Ke is exactly symmetric as after
// c3d10.py:248.
#include <algorithm>

#include "c3d10.cuh"
#include "common.cuh"
#include "kernels.h"
#include "pattern.h"
#include "wnfea_cuda.h"

namespace wn {

// (a, b) of upper-triangle index t (inverse of tri_index: t runs over a = 0..9, b = a..9),
// statically initialised, so no set-up call uploads them
__constant__ unsigned char c_tri_a[55] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 6, 6, 6, 6, 7, 7, 7, 8, 8, 9};
__constant__ unsigned char c_tri_b[55] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 1, 2, 3, 4, 5, 6, 7, 8, 9, 2, 3, 4, 5, 6, 7, 8, 9, 3, 4, 5, 6, 7, 8, 9, 4, 5, 6, 7, 8, 9, 5, 6, 7, 8, 9, 6, 7, 8, 9, 7, 8, 9, 8, 9, 9};

constexpr int KE_TILE = 16;      // elements per CTA
constexpr int KE_THREADS = 256;  // threads per CTA

// Stage one element's coordinates: X[a][j] = nodes[conn[e][a]][j].
__device__ __forceinline__ void load_coords(const double* __restrict__ nodes, const int32_t* __restrict__ conn,
                                            int64_t e, double X[10][3]) {
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    const int64_t n = conn[e * 10 + a];
    X[a][0] = nodes[n * 3 + 0];
    X[a][1] = nodes[n * 3 + 1];
    X[a][2] = nodes[n * 3 + 2];
  }
}

// Ke upper triangle of elements [0, n_el): out[(e * 55 + t) * 9 + 3 i + j].
// Phase 1: one thread per (element, Gauss point) computes dN/dx and w|J| into shared
// memory.  Phase 2: all threads produce the 495 block entries of the tile's elements,
// written contiguously.  An element with det J <= 0 raises bit 0 of *flags; an element with a
// node index outside [0, n_nodes) raises bit 1, reads no coordinates and gets a zero Ke.
__global__ void __launch_bounds__(KE_THREADS) ke_upper_kernel(int64_t n_el, int64_t n_nodes,
                                                              const double* __restrict__ nodes,
                                                              const int32_t* __restrict__ conn,
                                                              const double* __restrict__ props,
                                                              double* __restrict__ out, int* __restrict__ flags) {
  __shared__ double s_dn[KE_TILE][4][3][10];
  __shared__ double s_w[KE_TILE][4];
  __shared__ double s_lam[KE_TILE], s_mu[KE_TILE];
  for (int64_t tile = blockIdx.x; tile * KE_TILE < n_el; tile += gridDim.x) {
    const int64_t e0 = tile * KE_TILE;
    const int ne = (int)((n_el - e0) < KE_TILE ? (n_el - e0) : KE_TILE);
    if (threadIdx.x < KE_TILE * 4) {
      const int le = threadIdx.x >> 2, g = threadIdx.x & 3;
      if (le < ne) {
        bool in_range = true;
#pragma unroll
        for (int a = 0; a < 10; ++a) {
          const int32_t v = conn[(e0 + le) * 10 + a];
          in_range = in_range && v >= 0 && (int64_t)v < n_nodes;
        }
        double dndx[3][10];
        double det = 0.0;
        if (in_range) {
          double X[10][3];
          load_coords(nodes, conn, e0 + le, X);
          det = gp_cartesian(g, X, dndx);
          if (!(det > 0.0)) atomicOr(flags, 1);
        } else {
          atomicOr(flags, 2);
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int a = 0; a < 10; ++a) dndx[i][a] = 0.0;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int a = 0; a < 10; ++a) s_dn[le][g][i][a] = dndx[i][a];
        s_w[le][g] = kWeight * det;
        if (g == 0) {
          double lam, mu;
          lame(props[(e0 + le) * 2], props[(e0 + le) * 2 + 1], lam, mu);
          s_lam[le] = lam;
          s_mu[le] = mu;
        }
      }
    }
    __syncthreads();
    const int n_out = ne * 495;
    double* dst = out + e0 * 495;
    for (int o = threadIdx.x; o < n_out; o += KE_THREADS) {
      const int le = o / 495;
      const int rem = o - le * 495;
      const int t = rem / 9;
      const int ij = rem - t * 9;
      const int i = ij / 3, j = ij - (ij / 3) * 3;
      const int a = c_tri_a[t], b = c_tri_b[t];
      const double lam = s_lam[le], mu = s_mu[le];
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const double ai = s_dn[le][g][i][a], bj = s_dn[le][g][j][b];
        const double aj = s_dn[le][g][j][a], bi = s_dn[le][g][i][b];
        double v = lam * ai * bj + mu * aj * bi;
        if (i == j) {
          const double dot = s_dn[le][g][0][a] * s_dn[le][g][0][b] + s_dn[le][g][1][a] * s_dn[le][g][1][b] +
                             s_dn[le][g][2][a] * s_dn[le][g][2][b];
          v += mu * dot;
        }
        acc += s_w[le][g] * v;
      }
      dst[o] = acc;
    }
    __syncthreads();
  }
}

// Gather-assemble: one thread per 3x3 block.  K[b] = sum over the block's gather list (fixed
// (element, a, b) order) of the stored element block, transposed when a > b.  Dirichlet: an
// entry in a fixed row or column becomes 1 on the diagonal, 0 elsewhere
// (solid_solver.py:105-125).  Output is component-major (entry k of block b at k * nnzb + b)
// in FP64 and, if k32 != nullptr, FP32 -- consecutive threads write consecutive addresses.
__global__ void gather_assemble_kernel(int64_t nnzb, const int32_t* __restrict__ gptr,
                                       const int32_t* __restrict__ gsrc, const double* __restrict__ ke,
                                       const int32_t* __restrict__ block_row, const int32_t* __restrict__ col_idx,
                                       const uint8_t* __restrict__ fixed, double* __restrict__ k64,
                                       float* __restrict__ k32) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nnzb; b += (int64_t)gridDim.x * blockDim.x) {
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    const int32_t s = gptr[b], e = gptr[b + 1];
    for (int32_t q = s; q < e; ++q) {
      const int32_t src = gsrc[q];
      const double* blk = ke + (int64_t)(src >> 1) * 9;
      if (src & 1) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) acc[i * 3 + j] += blk[j * 3 + i];
      } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[k] += blk[k];
      }
    }
    if (fixed) {
      const int64_t r0 = (int64_t)block_row[b] * 3, c0 = (int64_t)col_idx[b] * 3;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          if (fixed[r0 + i] | fixed[c0 + j]) acc[i * 3 + j] = (r0 + i == c0 + j) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      k64[k * nnzb + b] = acc[k];
      if (k32) k32[k * nnzb + b] = (float)acc[k];
    }
  }
}

// ---------------------------------------------------------------------------------------
// Tile-owner assembly (no per-element scratch in global memory).  One CTA per row tile of
// the fine matrix (the tiles of its tile-major packs):
//   phase 0: the tile's contribution codes into shared memory, and each thread's three work
//            items (below) from the plan, loads in flight during phase 1;
//   phase 1: for every element incident to the tile's rows (the plan's list) and every
//            Gauss point, the Cartesian derivatives dN/dx (3 x 10) and w|J| into shared memory,
//            lam and mu beside them.  A warp takes one Gauss point for 32 elements, so the
//            natural derivatives are compile-time constants (gp_cartesian_rel) and the 32
//            lanes store to 32 distinct banks (element stride kAsmElStride: odd in 8-byte words);
//   phase 2: with v = dN/dx at a Gauss point, an element's block is
//            K_ab = lam S + mu S^T + mu tr(S) I for S = sum_g w v_a v_b^T (the isotropic
//            B^T C B of c3d10.py:244-246 summed over the Gauss points); a work item sums
//            A = sum_e lam_e S_e and B = sum_e mu_e S_e over a run of the block's contributions
//            in element order (the gather order), and the block is K = A + B^T + tr(B) I.  S is
//            computed for (p, r) = (min, max) of the element's local node pair and transposed
//            when a > b, and S_pp is mirrored from its upper triangle, so blocks (i, j) and
//            (j, i) add bitwise-transposed terms in the same order, diagonal blocks come out
//            symmetric and K is exactly symmetric.
//            Work items, in three rounds of one item per thread: round 0 gives the chunks of
//            the tile's split blocks (more than the plan's chunk_len contributions: the
//            diagonal blocks of vertex nodes) to threads 0 .. NH-1, which leave their A and B in
//            chunk slots, and the heaviest other blocks to the rest; round 1 the next 256
//            blocks in reverse thread order (a thread with a heavy block in round 0 gets a light
//            one now); round 2 the remainder to threads 0 .. NH-1.  A thread holds at most two
//            finished blocks.  The chunk sums of a split block are then added in chunk order;
//            blocks are cut by their contribution count alone, so (i, j) and (j, i) alike.
//            Then the Dirichlet rows / columns;
//   phase 3: the tile's blocks staged in shared memory and written coalesced: FP64 and FP32
//            component-major values and, when given, the FP64 / FP32 pack segments of the tile.
// ---------------------------------------------------------------------------------------
constexpr int kAsmThreads = 256;
constexpr int kAsmGpStride = 31;                  // 30 derivatives + w|J|
constexpr int kAsmElStride = 4 * kAsmGpStride + 1;  // 125 doubles per element (odd)

// shared-memory layout (doubles): [0, el_area) element data, later the staged blocks;
// [el_area, el_area + 18 kAsmChunkSlots) chunk sums; then the tile's contribution codes
__host__ __device__ constexpr int64_t asm_el_area(int ne_max) {
  return (int64_t)ne_max * (kAsmElStride + 2) > (int64_t)WN_STREAM_TILE_BLOCKS * 9
             ? (int64_t)ne_max * (kAsmElStride + 2)
             : (int64_t)WN_STREAM_TILE_BLOCKS * 9;
}

// doubles of the space shared by the chunk sums (phase 2 on) and the incident elements'
// connectivity (phases 0-1)
__host__ __device__ constexpr int64_t asm_union_doubles(int ne_max) {
  return (int64_t)18 * kAsmChunkSlots > ((int64_t)ne_max * 10 + 1) / 2 ? (int64_t)18 * kAsmChunkSlots
                                                                      : ((int64_t)ne_max * 10 + 1) / 2;
}

struct AsmItem {
  int j = -1;      // local block, -1: none
  int qa = 0, qb = 0;  // contributions [qa, qb) (global indices)
};

// A and B of a work item: sum over contributions q in [qa, qb) of lam S and mu S
__device__ __forceinline__ void asm_item_sums(const double* __restrict__ s_el, const double* __restrict__ s_lm,
                                              const uint16_t* __restrict__ s_codes, int qbase, int qa, int qb,
                                              double (&As)[9], double (&Bs)[9]) {
#pragma unroll
  for (int m = 0; m < 9; ++m) As[m] = Bs[m] = 0.0;
  for (int q = qa; q < qb; ++q) {
    const int code = s_codes[q - qbase];
    const int slot = code >> 8, ea = (code >> 4) & 15, eb = code & 15;
    const int p = min(ea, eb), r = max(ea, eb);
    const double* d = s_el + slot * kAsmElStride;
    double S[9];
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const double* dg = d + g * kAsmGpStride;
      const double w = dg[30];
      const double wp0 = w * dg[p], wp1 = w * dg[10 + p], wp2 = w * dg[20 + p];
      const double vr0 = dg[r], vr1 = dg[10 + r], vr2 = dg[20 + r];
      if (g == 0) {
        S[0] = wp0 * vr0; S[1] = wp0 * vr1; S[2] = wp0 * vr2;
        S[3] = wp1 * vr0; S[4] = wp1 * vr1; S[5] = wp1 * vr2;
        S[6] = wp2 * vr0; S[7] = wp2 * vr1; S[8] = wp2 * vr2;
      } else {
        S[0] = fma(wp0, vr0, S[0]); S[1] = fma(wp0, vr1, S[1]); S[2] = fma(wp0, vr2, S[2]);
        S[3] = fma(wp1, vr0, S[3]); S[4] = fma(wp1, vr1, S[4]); S[5] = fma(wp1, vr2, S[5]);
        S[6] = fma(wp2, vr0, S[6]); S[7] = fma(wp2, vr1, S[7]); S[8] = fma(wp2, vr2, S[8]);
      }
    }
    if (p == r) {  // S_pp symmetric: its lower triangle from the upper
      S[3] = S[1];
      S[6] = S[2];
      S[7] = S[5];
    }
    const double lam = s_lm[2 * slot], mu = s_lm[2 * slot + 1];
    if (ea <= eb) {
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        As[m] = fma(lam, S[m], As[m]);
        Bs[m] = fma(mu, S[m], Bs[m]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
          As[i * 3 + jj] = fma(lam, S[jj * 3 + i], As[i * 3 + jj]);
          Bs[i * 3 + jj] = fma(mu, S[jj * 3 + i], Bs[i * 3 + jj]);
        }
    }
  }
}

// K = A + B^T + tr(B) I, then the Dirichlet rows / columns of block b
__device__ __forceinline__ void asm_finish(const AsmTileArgs& A, const uint8_t* __restrict__ fixed, int64_t b,
                                           const double (&As)[9], const double (&Bs)[9], double (&out)[9]) {
  const double trB = Bs[0] + Bs[4] + Bs[8];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) out[i * 3 + jj] = As[i * 3 + jj] + Bs[jj * 3 + i] + (i == jj ? trB : 0.0);
  if (fixed) {
    const int64_t r0 = (int64_t)A.block_row[b] * 3, c0 = (int64_t)A.col_idx[b] * 3;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int jj = 0; jj < 3; ++jj)
        if (fixed[r0 + i] | fixed[c0 + jj]) out[i * 3 + jj] = (r0 + i == c0 + jj) ? 1.0 : 0.0;
  }
}

__global__ void __launch_bounds__(kAsmThreads, 2) assemble_tiles_kernel(
    const AsmTileArgs A, int el_area, const double* __restrict__ nodes, const int32_t* __restrict__ conn,
    const double* __restrict__ props, const uint8_t* __restrict__ fixed, int64_t nnzb, double* __restrict__ k64,
    float* __restrict__ k32, int* __restrict__ flags) {
  extern __shared__ double s_el[];
  double* s_part = s_el + el_area;                           // kAsmChunkSlots x (A 9, B 9), phase 2 on
  int32_t* s_conn = reinterpret_cast<int32_t*>(s_part);      // the same space, phases 0-1: ne x 10
  uint16_t* s_codes = reinterpret_cast<uint16_t*>(s_el + el_area + asm_union_doubles(A.ne_max));
  __shared__ uint32_t s_chunk[kAsmChunkSlots];
  const int t = blockIdx.x, x = threadIdx.x;
  const int4 T = reinterpret_cast<const int4*>(A.tiles)[t];  // r0, r1, b0, b1
  const int4 H0 = reinterpret_cast<const int4*>(A.hdr)[2 * t];
  const int4 H1 = reinterpret_cast<const int4*>(A.hdr)[2 * t + 1];
  const int e_beg = H0.x, ne = H0.y, c0 = H0.z, NH = H0.w, H = H1.x, qbase = H1.y, ncodes = H1.z;
  double* s_lm = s_el + ne * kAsmElStride;  // lam, mu per element
  const int nb = T.w - T.z, L = nb - H;
  // phase 0: work items, incident elements (connectivity, lam, mu), codes -- loads in flight
  // together, each at most two dependent steps from the tile header
  const int n0 = min(L, kAsmThreads - NH);  // light blocks of round 0
  AsmItem it[3];
  bool first = false;  // round 0 holds the first chunk of a split block
  if (x < NH) {
    const uint32_t c = A.chunks[c0 + x];
    s_chunk[x] = c;
    it[0].j = (int)(c & 511u);
    it[0].qa = A.gptr[T.z + it[0].j] + (int)((c >> 9) & 1023u);
    it[0].qb = it[0].qa + (int)((c >> 19) & 63u);
    first = (c >> 25) & 1u;
  } else if (x - NH < L) {
    it[0].j = A.perm[T.z + H + (x - NH)];
  }
  {
    const int k1 = n0 + (kAsmThreads - 1 - x), k2 = n0 + kAsmThreads + x;
    if (k1 < L) it[1].j = A.perm[T.z + H + k1];
    if (x < NH && k2 < L) it[2].j = A.perm[T.z + H + k2];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
    if (it[r].j >= 0 && !(r == 0 && x < NH)) {
      it[r].qa = A.gptr[T.z + it[r].j];
      it[r].qb = A.gptr[T.z + it[r].j + 1];
    }
  for (int k = x; k < ne; k += kAsmThreads) {
    const int64_t e = A.el[e_beg + k];
    int32_t cn[10];
#pragma unroll
    for (int a = 0; a < 10; ++a) cn[a] = conn[e * 10 + a];
    double lam, mu;
    lame(props[e * 2], props[e * 2 + 1], lam, mu);
#pragma unroll
    for (int a = 0; a < 10; ++a) s_conn[k * 10 + a] = cn[a];
    s_lm[2 * k] = lam;
    s_lm[2 * k + 1] = mu;
  }
  {
    constexpr int kDeep = 8;  // codes per thread loaded before any is stored
    for (int i0 = x; i0 < ncodes; i0 += kAsmThreads * kDeep) {
      uint16_t v[kDeep];
#pragma unroll
      for (int j = 0; j < kDeep; ++j) {
        const int i = i0 + j * kAsmThreads;
        v[j] = i < ncodes ? A.contrib[qbase + i] : (uint16_t)0;
      }
#pragma unroll
      for (int j = 0; j < kDeep; ++j) {
        const int i = i0 + j * kAsmThreads;
        if (i < ncodes) s_codes[i] = v[j];
      }
    }
  }
  __syncthreads();
  // phase 1
  {
    const int warp = x >> 5, lane = x & 31;
    const int n_items = ((ne + 31) >> 5) * 4;  // (32-element group, Gauss point)
    for (int wi = warp; wi < n_items; wi += kAsmThreads / 32) {
      const int g = wi & 3, k = (wi >> 2) * 32 + lane;
      if (k >= ne) continue;
      double Xr[10][3];
#pragma unroll
      for (int a = 0; a < 10; ++a) {
        const int64_t nd = s_conn[k * 10 + a];
        Xr[a][0] = nodes[nd * 3 + 0];
        Xr[a][1] = nodes[nd * 3 + 1];
        Xr[a][2] = nodes[nd * 3 + 2];
      }
#pragma unroll
      for (int a = 1; a < 10; ++a)
#pragma unroll
        for (int j = 0; j < 3; ++j) Xr[a][j] -= Xr[0][j];
      double dndx[3][10];
      double det;
      switch (g) {  // warp-uniform
        case 0: det = gp_cartesian_rel<0>(Xr, dndx); break;
        case 1: det = gp_cartesian_rel<1>(Xr, dndx); break;
        case 2: det = gp_cartesian_rel<2>(Xr, dndx); break;
        default: det = gp_cartesian_rel<3>(Xr, dndx); break;
      }
      if (!(det > 0.0)) atomicOr(flags, 1);
      double* d = s_el + k * kAsmElStride + g * kAsmGpStride;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int a = 0; a < 10; ++a) d[i * 10 + a] = dndx[i][a];
      d[30] = kWeight * det;
    }
  }
  __syncthreads();  // s_conn is dead from here on (its space holds the chunk sums)
  // phase 2: rounds 0 and 2 finish into fin[0], round 1 into fin[1] (a thread has a light
  // block in round 0 or in round 2, not both); split-block chunks leave A and B in slot x
  double fin[2][9];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    if (it[r].j < 0) continue;
    double As[9], Bs[9];
    asm_item_sums(s_el, s_lm, s_codes, qbase, it[r].qa, it[r].qb, As, Bs);
    if (r == 0 && x < NH) {
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        s_part[x * 18 + m] = As[m];
        s_part[x * 18 + 9 + m] = Bs[m];
      }
    } else {
      asm_finish(A, fixed, T.z + it[r].j, As, Bs, fin[r == 1 ? 1 : 0]);
    }
  }
  // phase 3: the tile's blocks staged in shared memory in local order (over the element data,
  // which every thread has finished reading), then written coalesced, component by component
  __syncthreads();
  double* stage = s_el;  // nb x 9 (odd stride: consecutive blocks hit different banks)
  if (first) {  // the chunk sums of this split block, in chunk order
    double As[9], Bs[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) {
      As[m] = s_part[x * 18 + m];
      Bs[m] = s_part[x * 18 + 9 + m];
    }
    for (int y = x + 1; y < NH && !((s_chunk[y] >> 25) & 1u); ++y)
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        As[m] += s_part[y * 18 + m];
        Bs[m] += s_part[y * 18 + 9 + m];
      }
    double out[9];
    asm_finish(A, fixed, T.z + it[0].j, As, Bs, out);
#pragma unroll
    for (int m = 0; m < 9; ++m) stage[it[0].j * 9 + m] = out[m];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
    if (it[r].j >= 0 && !(r == 0 && x < NH))
#pragma unroll
      for (int m = 0; m < 9; ++m) stage[it[r].j * 9 + m] = fin[r == 1 ? 1 : 0][m];
  __syncthreads();
  const int4 d64 = A.p64 ? reinterpret_cast<const int4*>(A.d64)[t] : make_int4(0, 0, 0, 0);  // r0, r1, seg, cntp
  const int4 d32 = A.p64 ? reinterpret_cast<const int4*>(A.d32)[t] : make_int4(0, 0, 0, 0);
  double* v64 = A.p64 ? reinterpret_cast<double*>(A.p64 + (size_t)d64.z * 128) : nullptr;
  float* v32 = A.p64 ? reinterpret_cast<float*>(A.p32 + (size_t)d32.z * 128) : nullptr;
  // nb <= 2 kAsmThreads: two blocks per thread and component, all shared-memory reads first
#pragma unroll
  for (int m = 0; m < 9; ++m) {
    const int j0 = x, j1 = x + kAsmThreads;
    const double a0 = j0 < nb ? stage[j0 * 9 + m] : 0.0, a1 = j1 < nb ? stage[j1 * 9 + m] : 0.0;
    if (j0 < nb) {
      k64[m * nnzb + T.z + j0] = a0;
      k32[m * nnzb + T.z + j0] = (float)a0;
      if (v64) {
        v64[m * d64.w + j0] = a0;
        v32[m * d32.w + j0] = (float)a0;
      }
    }
    if (j1 < nb) {
      k64[m * nnzb + T.z + j1] = a1;
      k32[m * nnzb + T.z + j1] = (float)a1;
      if (v64) {
        v64[m * d64.w + j1] = a1;
        v32[m * d32.w + j1] = (float)a1;
      }
    }
  }
}

// Matrix-free element forces f_e = Ke u_e (= sum_g w|J| B^T C B u_e, c3d10.py:252-283) for
// DOF stride `stride` (3 for the solid path, 6 for the reference's mixed-DOF layout of
// kernels.cpp:244-376).  If fe_out: writes f_e (n_el x 30).  If energy_out: writes
// u_e . f_e per element.  If grad_e: writes -u_e . f_e / E_e (compliance adjoint).
__global__ void element_force_kernel(int64_t n_el, const double* __restrict__ nodes, const int32_t* __restrict__ conn,
                                     const double* __restrict__ props, const double* __restrict__ u, int stride,
                                     double* __restrict__ fe_out, double* __restrict__ energy_out,
                                     double* __restrict__ grad_e, int* __restrict__ flags) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_el; e += (int64_t)gridDim.x * blockDim.x) {
    double X[10][3], ue[10][3];
    load_coords(nodes, conn, e, X);
#pragma unroll
    for (int a = 0; a < 10; ++a) {
      const int64_t n = conn[e * 10 + a];
      ue[a][0] = u[n * stride + 0];
      ue[a][1] = u[n * stride + 1];
      ue[a][2] = u[n * stride + 2];
    }
    const double E = props[e * 2], nu = props[e * 2 + 1];
    const double f = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double c11 = f * (1.0 - nu), c12 = f * nu, G = E / (2.0 * (1.0 + nu));
    double fe[10][3];
#pragma unroll
    for (int a = 0; a < 10; ++a) fe[a][0] = fe[a][1] = fe[a][2] = 0.0;
    bool bad = false;
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
      double d[3][10];
      const double det = gp_cartesian(g, X, d);
      if (!(det > 0.0)) bad = true;
      double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int a = 0; a < 10; ++a) {
        eps[0] += d[0][a] * ue[a][0];
        eps[1] += d[1][a] * ue[a][1];
        eps[2] += d[2][a] * ue[a][2];
        eps[3] += d[1][a] * ue[a][0] + d[0][a] * ue[a][1];
        eps[4] += d[2][a] * ue[a][1] + d[1][a] * ue[a][2];
        eps[5] += d[2][a] * ue[a][0] + d[0][a] * ue[a][2];
      }
      const double s0 = c11 * eps[0] + c12 * eps[1] + c12 * eps[2];
      const double s1 = c12 * eps[0] + c11 * eps[1] + c12 * eps[2];
      const double s2 = c12 * eps[0] + c12 * eps[1] + c11 * eps[2];
      const double s3 = G * eps[3], s4 = G * eps[4], s5 = G * eps[5];
      const double w = kWeight * det;
#pragma unroll
      for (int a = 0; a < 10; ++a) {
        fe[a][0] += w * (d[0][a] * s0 + d[1][a] * s3 + d[2][a] * s5);
        fe[a][1] += w * (d[1][a] * s1 + d[0][a] * s3 + d[2][a] * s4);
        fe[a][2] += w * (d[2][a] * s2 + d[1][a] * s4 + d[0][a] * s5);
      }
    }
    if (bad) flags[0] = 1;
    if (fe_out) {
#pragma unroll
      for (int a = 0; a < 10; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) fe_out[e * 30 + a * 3 + c] = fe[a][c];
    }
    if (energy_out || grad_e) {
      double en = 0.0;
#pragma unroll
      for (int a = 0; a < 10; ++a) en += ue[a][0] * fe[a][0] + ue[a][1] * fe[a][1] + ue[a][2] * fe[a][2];
      if (energy_out) energy_out[e] = en;
      if (grad_e) grad_e[e] = -en / E;
    }
  }
}

// Node gather of element vectors: out[n * stride + c] (+)= sum over the node's incident
// (element, local node) pairs, in ascending element order, of fe[e][a][c].  Atomic-free.
__global__ void node_gather_kernel(int64_t n_nodes, const int64_t* __restrict__ inc_ptr,
                                   const int32_t* __restrict__ inc_ea, const double* __restrict__ fe, int stride,
                                   int accumulate, double* __restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_nodes * 3;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = t / 3;
    const int c = (int)(t - n * 3);
    double s = 0.0;
    for (int64_t q = inc_ptr[n]; q < inc_ptr[n + 1]; ++q) s += fe[(int64_t)inc_ea[q] * 3 + c];
    if (accumulate)
      out[n * stride + c] += s;
    else
      out[n * stride + c] = s;
  }
}

// Cell stresses: mean of the 4 Gauss-point stresses [sxx, syy, szz, sxy, syz, szx] and the
// mean Gauss-point von Mises (solid_solver.py:341-350, c3d10.py:286-318).
// Also, when gp_sig / gp_vm are given, the stresses and von Mises of every Gauss point
// (element_stresses_c3d10, c3d10.py:286-318): gp_sig[(e * 4 + g) * 6 + k], gp_vm[e * 4 + g].
__global__ void stress_kernel(int64_t n_el, const double* __restrict__ nodes, const int32_t* __restrict__ conn,
                              const double* __restrict__ props, const double* __restrict__ u,
                              double* __restrict__ cell_sig, double* __restrict__ cell_vm, double* __restrict__ gp_sig,
                              double* __restrict__ gp_vm) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_el; e += (int64_t)gridDim.x * blockDim.x) {
    double X[10][3], ue[10][3];
    load_coords(nodes, conn, e, X);
#pragma unroll
    for (int a = 0; a < 10; ++a) {
      const int64_t n = conn[e * 10 + a];
      ue[a][0] = u[n * 3 + 0];
      ue[a][1] = u[n * 3 + 1];
      ue[a][2] = u[n * 3 + 2];
    }
    const double E = props[e * 2], nu = props[e * 2 + 1];
    const double f = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double c11 = f * (1.0 - nu), c12 = f * nu, G = E / (2.0 * (1.0 + nu));
    double ssum[6] = {0, 0, 0, 0, 0, 0};
    double vmsum = 0.0;
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
      double d[3][10];
      gp_cartesian(g, X, d);
      double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int a = 0; a < 10; ++a) {
        eps[0] += d[0][a] * ue[a][0];
        eps[1] += d[1][a] * ue[a][1];
        eps[2] += d[2][a] * ue[a][2];
        eps[3] += d[1][a] * ue[a][0] + d[0][a] * ue[a][1];
        eps[4] += d[2][a] * ue[a][1] + d[1][a] * ue[a][2];
        eps[5] += d[2][a] * ue[a][0] + d[0][a] * ue[a][2];
      }
      const double s[6] = {c11 * eps[0] + c12 * eps[1] + c12 * eps[2], c12 * eps[0] + c11 * eps[1] + c12 * eps[2],
                           c12 * eps[0] + c12 * eps[1] + c11 * eps[2], G * eps[3], G * eps[4], G * eps[5]};
#pragma unroll
      for (int k = 0; k < 6; ++k) ssum[k] += s[k];
      const double a0 = s[0] - s[1], a1 = s[1] - s[2], a2 = s[2] - s[0];
      const double vm = sqrt(0.5 * (a0 * a0 + a1 * a1 + a2 * a2 + 6.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5])));
      vmsum += vm;
      if (gp_sig) {
#pragma unroll
        for (int k = 0; k < 6; ++k) gp_sig[(e * 4 + g) * 6 + k] = s[k];
        gp_vm[e * 4 + g] = vm;
      }
    }
    if (cell_sig) {
#pragma unroll
      for (int k = 0; k < 6; ++k) cell_sig[e * 6 + k] = ssum[k] / 4.0;
      cell_vm[e] = vmsum / 4.0;
    }
  }
}

// Nodal von Mises = unweighted mean of incident cells' von Mises (solid_solver.py:352-363).
__global__ void nodal_average_kernel(int64_t n_nodes, const int64_t* __restrict__ inc_ptr,
                                     const int32_t* __restrict__ inc_ea, const double* __restrict__ cell_vm,
                                     double* __restrict__ nodal) {
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = inc_ptr[n], e = inc_ptr[n + 1];
    double acc = 0.0;
    for (int64_t q = s; q < e; ++q) acc += cell_vm[inc_ea[q] / 10];
    nodal[n] = (e > s) ? acc / (double)(e - s) : 0.0;
  }
}

// ---------------------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------------------
size_t assemble_tiles_smem(int ne_max, int max_codes) {
  return (size_t)(asm_el_area(ne_max) + asm_union_doubles(ne_max)) * sizeof(double) +
         ((size_t)max_codes * 2 + 7) / 8 * 8;
}

int launch_assemble_tiles(const AsmTileArgs& A, int n_tiles, int ne_max, int max_codes, const double* nodes,
                          const int32_t* conn, const double* props, const uint8_t* fixed, int64_t nnzb, double* k64,
                          float* k32, int* flags, cudaStream_t st) {
  if (n_tiles == 0) return 0;
  // element data of the tile (derivatives, then lam and mu), later (same space) its finished
  // blocks, at most WN_STREAM_TILE_BLOCKS x 9 doubles; the chunk sums; the contribution codes
  static_assert(WN_STREAM_TILE_BLOCKS <= 2 * kAsmThreads, "two blocks per thread in the assembly");
  const int64_t el_area = asm_el_area(ne_max);
  const size_t smem = assemble_tiles_smem(ne_max, max_codes);
  WN_REQUIRE(smem <= kAsmSmemLimit, WN_ETOOBIG, "assembly: %zu bytes of shared memory per tile", smem);
  static int configured_bytes[64] = {0};  // per device: the largest dynamic size allowed so far
  int dev = 0;
  WN_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) dev = 0;
  if ((int)smem > configured_bytes[dev] && smem > 48 * 1024) {
    WN_CUDA(cudaFuncSetAttribute(assemble_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured_bytes[dev] = (int)smem;
  }
  assemble_tiles_kernel<<<n_tiles, kAsmThreads, smem, st>>>(A, (int)el_area, nodes, conn, props, fixed, nnzb, k64,
                                                            k32, flags);
  WN_CUDA(cudaGetLastError());
  return 0;
}

int launch_ke_upper(int64_t n_el, int64_t n_nodes, const double* nodes, const int32_t* conn, const double* props,
                    double* out, int* flags, cudaStream_t st) {
  if (n_el == 0) return 0;
  const int64_t tiles = (n_el + KE_TILE - 1) / KE_TILE;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)kNumSMs * 8);
  ke_upper_kernel<<<grid, KE_THREADS, 0, st>>>(n_el, n_nodes, nodes, conn, props, out, flags);
  WN_CUDA(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------------------
// node incidence on the device (for the stateless internal-force call)
// ---------------------------------------------------------------------------------------
__global__ void incidence_count_kernel(int64_t n_entries, int64_t nn, const int32_t* __restrict__ conn,
                                       int32_t* __restrict__ counts, int* __restrict__ bad) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n_entries;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = conn[k];
    if (v < 0 || v >= nn) {
      *bad = 1;
      continue;
    }
    atomicAdd(&counts[v], 1);  // integer counts: order-independent
  }
}

// inclusive scan of one value per thread over a 1024-thread CTA
__device__ __forceinline__ int64_t block_scan_1024(int64_t v, int64_t* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    int64_t t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += u;
    }
    sh[lane] = t;
  }
  __syncthreads();
  const int64_t r = v + (w > 0 ? sh[w - 1] : 0);
  __syncthreads();
  return r;
}

// per 1024-entry chunk: out[i] = exclusive prefix inside the chunk, tot[chunk] = chunk sum
__global__ void __launch_bounds__(1024) scan_chunks_kernel(int64_t n, const int32_t* __restrict__ in,
                                                          int64_t* __restrict__ out, int64_t* __restrict__ tot) {
  __shared__ int64_t sh[32];
  const int64_t i = blockIdx.x * 1024 + threadIdx.x;
  const int64_t v = i < n ? in[i] : 0;
  const int64_t inc = block_scan_1024(v, sh);
  if (i < n) out[i] = inc - v;
  if (threadIdx.x == 1023) tot[blockIdx.x] = inc;
}

// one CTA: exclusive scan of the chunk sums in place (any count, in passes of 1024), total to *total
__global__ void __launch_bounds__(1024) scan_totals_kernel(int64_t n_chunks, int64_t* __restrict__ tot,
                                                          int64_t* __restrict__ total) {
  __shared__ int64_t sh[32];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n_chunks; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < n_chunks ? tot[i] : 0;
    const int64_t inc = block_scan_1024(v, sh);
    const int64_t c = carry;
    if (i < n_chunks) tot[i] = c + inc - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = c + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_add_kernel(int64_t n, const int64_t* __restrict__ tot, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] += tot[i >> 10];
}

__global__ void incidence_fill_kernel(int64_t n_entries, int64_t nn, const int32_t* __restrict__ conn,
                                      const int64_t* __restrict__ inc_ptr, int32_t* __restrict__ cursor,
                                      int32_t* __restrict__ inc) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n_entries;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = conn[k];
    if (v < 0 || v >= nn) continue;
    const int32_t p = atomicAdd(&cursor[v], 1);
    inc[inc_ptr[v] + p] = (int32_t)k;
  }
}

// each node's entries in ascending e * 10 + a (insertion sort; ~10-50 entries per node), so
// that the node gather sums in a fixed order whatever order the fill wrote them in
__global__ void incidence_sort_kernel(int64_t nn, const int64_t* __restrict__ inc_ptr, int32_t* __restrict__ inc) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nn; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = inc_ptr[v], e = inc_ptr[v + 1];
    for (int64_t i = s + 1; i < e; ++i) {
      const int32_t key = inc[i];
      int64_t j = i - 1;
      while (j >= s && inc[j] > key) {
        inc[j + 1] = inc[j];
        --j;
      }
      inc[j + 1] = key;
    }
  }
}

int launch_build_incidence(int64_t nn, int64_t ne, const int32_t* conn, int32_t* counts, int64_t* inc_ptr,
                           int32_t* inc, int64_t* scan, int* flags, cudaStream_t st) {
  const int64_t n_entries = ne * 10;
  const int64_t n_chunks = (nn + 1023) / 1024;
  WN_CUDA(cudaMemsetAsync(counts, 0, nn * sizeof(int32_t), st));
  WN_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(int), st));
  incidence_count_kernel<<<grid_for(n_entries, 1, 256, 8), 256, 0, st>>>(n_entries, nn, conn, counts, flags);
  scan_chunks_kernel<<<(int)n_chunks, 1024, 0, st>>>(nn, counts, inc_ptr, scan);
  scan_totals_kernel<<<1, 1024, 0, st>>>(n_chunks, scan, inc_ptr + nn);
  scan_add_kernel<<<grid_for(nn, 1, 256, 8), 256, 0, st>>>(nn, scan, inc_ptr);
  WN_CUDA(cudaMemsetAsync(counts, 0, nn * sizeof(int32_t), st));
  incidence_fill_kernel<<<grid_for(n_entries, 1, 256, 8), 256, 0, st>>>(n_entries, nn, conn, inc_ptr, counts, inc);
  incidence_sort_kernel<<<grid_for(nn, 1, 256, 8), 256, 0, st>>>(nn, inc_ptr, inc);
  WN_CUDA(cudaGetLastError());
  return 0;
}

int launch_gather_assemble(int64_t nnzb, const int32_t* gptr, const int32_t* gsrc, const double* ke,
                           const int32_t* block_row, const int32_t* col_idx, const uint8_t* fixed, double* k64,
                           float* k32, cudaStream_t st) {
  if (nnzb == 0) return 0;
  const int grid = grid_for(nnzb, 1, 256, 16);
  gather_assemble_kernel<<<grid, 256, 0, st>>>(nnzb, gptr, gsrc, ke, block_row, col_idx, fixed, k64, k32);
  WN_CUDA(cudaGetLastError());
  return 0;
}

int launch_element_force(int64_t n_el, const double* nodes, const int32_t* conn, const double* props,
                         const double* u, int stride, double* fe_out, double* energy_out, double* grad_e,
                         int* flags, cudaStream_t st) {
  if (n_el == 0) return 0;
  const int grid = grid_for(n_el, 1, 128, 16);
  element_force_kernel<<<grid, 128, 0, st>>>(n_el, nodes, conn, props, u, stride, fe_out, energy_out, grad_e, flags);
  WN_CUDA(cudaGetLastError());
  return 0;
}

int launch_node_gather(int64_t n_nodes, const int64_t* inc_ptr, const int32_t* inc_ea, const double* fe, int stride,
                       int accumulate, double* out, cudaStream_t st) {
  if (n_nodes == 0) return 0;
  const int grid = grid_for(n_nodes * 3, 1, 256, 16);
  node_gather_kernel<<<grid, 256, 0, st>>>(n_nodes, inc_ptr, inc_ea, fe, stride, accumulate, out);
  WN_CUDA(cudaGetLastError());
  return 0;
}

int launch_stress(int64_t n_el, int64_t n_nodes, const double* nodes, const int32_t* conn, const double* props,
                  const double* u, const int64_t* inc_ptr, const int32_t* inc_ea, double* cell_sig, double* cell_vm,
                  double* nodal_vm, cudaStream_t st) {
  if (n_el > 0) {
    const int grid = grid_for(n_el, 1, 128, 16);
    stress_kernel<<<grid, 128, 0, st>>>(n_el, nodes, conn, props, u, cell_sig, cell_vm, nullptr, nullptr);
    WN_CUDA(cudaGetLastError());
  }
  if (n_nodes > 0) {
    const int grid = grid_for(n_nodes, 1, 256, 16);
    nodal_average_kernel<<<grid, 256, 0, st>>>(n_nodes, inc_ptr, inc_ea, cell_vm, nodal_vm);
    WN_CUDA(cudaGetLastError());
  }
  return 0;
}

int launch_gp_stress(int64_t n_el, const double* nodes, const int32_t* conn, const double* props, const double* u,
                     double* gp_sig, double* gp_vm, cudaStream_t st) {
  if (n_el == 0) return 0;
  const int grid = grid_for(n_el, 1, 128, 16);
  stress_kernel<<<grid, 128, 0, st>>>(n_el, nodes, conn, props, u, nullptr, nullptr, gp_sig, gp_vm);
  WN_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wn
