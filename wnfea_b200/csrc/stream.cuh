// Streamed row engine for block-sparse matrices on sm_100a: BR x BC blocks (3x3 for the fine
// level, 6x6 for the AMG levels too large to stay in L2, 3x6 / 6x3 for the fine level's
// prolongator / restrictor), 32-bit row pointers and column indices, FP32 or FP64 values.
//
// The fine matrix is the one array every fine-level kernel of the solve reads in full (40 B per
// block in FP32, 76 B in FP64, against 12-24 B of x gathers that L2 serves), so its kernels are
// HBM-bound, and a warp-per-row kernel that chains row_ptr -> values -> x gathers leaves HBM
// idle while it waits.  Here the matrix is cut into tiles of whole rows (at most kStreamCap
// blocks and kStreamRowCap rows) and streamed through shared memory:
//   * after each assembly the values are packed tile-major ("pack"): tile t is one 128-byte
//     aligned segment holding its BR * BC value components (component-major, cntp = cnt rounded
//     up to 4 per component), its column indices and its local row starts (uint16), so the whole
//     tile moves with ONE bulk async copy (cp.async.bulk, the TMA's 1-D form) -- a bulk copy
//     costs the issuing thread a fixed ~70-90 ns on B200 whatever its size, so a tile of 11
//     separate copies (9 components of the component-major matrix, columns, row pointers)
//     held one producer to ~1 tile per microsecond;
//   * one producer thread per CTA issues the copies into a ring of stage buffers, with an L2
//     evict-first hint so the streamed matrix does not push the vectors out of L2, and
//     signals completion through an mbarrier per stage (expect_tx bytes); the producer warp
//     holds the next 32 tile descriptors, one per lane, so no copy waits on a descriptor load;
//   * consumer warps wait on the stage, compute their rows from shared memory (G lanes per
//     block row, lane l taking the row's blocks l, l + G, ... -- the assignment of the register
//     kernels in spmv.cuh, with the shape's own G -- with U blocks' gathers in flight per lane),
//     and release the stage through a second mbarrier;
//   * CTAs are persistent and take fixed runs of tiles, so the per-CTA dot partials come out in
//     a fixed order (deterministic two-stage dots);
//   * the first stages' copies are issued before griddepcontrol.wait: under a programmatic
//     dependent launch a kernel's CTAs start streaming their matrix while the previous kernel
//     on the stream finishes, and read vectors, partials and flags only after the wait.
// Every wait is bounded in time: a wait that runs out sets the caller's status word to
// WN_ETIMEOUT and its done flag, the CTA stops issuing, waits (bounded) for its copies in
// flight and returns.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <vector>

#include "wnfea_cuda.h"

namespace wn {

// a tile of the fine matrix: block rows [r0, r1) holding blocks [b0, b1) (the plan)
struct StreamTile {
  int32_t r0, r1, b0, b1;
};
// the device descriptor of a packed tile: rows [r0, r1), segment at byte 128 seg of the pack,
// cntp blocks per value component (the tile's block count rounded up to 4)
struct PackTile {
  int32_t r0, r1, seg, cntp;
};

constexpr int kStreamCap = WN_STREAM_TILE_BLOCKS;   // blocks per tile at most (a multiple of 4)
constexpr int kStreamRowCap = WN_STREAM_TILE_ROWS;  // rows per tile at most
static_assert(kStreamCap % 4 == 0, "tile capacity: a multiple of 4 blocks");
// shared memory ahead of the stage buffers: full / empty mbarriers (<= 8 stages), the abort
// flag at byte 256 and the skip flag at 260, the stage descriptors at byte 384
constexpr int kStreamHeader = 512;

// Byte layout of a packed tile segment of NV = BR * BC values per block (also its stage buffer
// image):
//   [0, NV cntp sizeof(T))     values, component k of local block b at k * cntp + b
//   [col_off, + 4 cntp)        column indices (padding: 0)
//   [row_off, + 2 (nr + 1))    local row starts (uint16), rounded up to 16 bytes
// and the whole segment rounded up to 128 bytes.
__host__ __device__ constexpr int pack_cntp(int cnt) { return (cnt + 3) & ~3; }
template <typename T, int NV>
__host__ __device__ constexpr uint32_t pack_col_off(int cntp) {
  return (uint32_t)NV * (uint32_t)cntp * (uint32_t)sizeof(T);
}
template <typename T, int NV>
__host__ __device__ constexpr uint32_t pack_row_off(int cntp) {
  return pack_col_off<T, NV>(cntp) + 4u * (uint32_t)cntp;
}
template <typename T, int NV>
__host__ __device__ constexpr uint32_t pack_bytes(int cntp, int nr) {
  return (pack_row_off<T, NV>(cntp) + ((2u * (uint32_t)(nr + 1) + 15u) & ~15u) + 127u) & ~127u;
}

// Shape of a streamed kernel: tile capacity (blocks, rows), consumer warps, lanes per block
// row, stage buffers, blocks a lane has in flight per row and rows a lane group computes
// together (their gathers all issued before the first multiply-add).
template <int CAP, int ROWS, int WARPS, int G, int STAGES, int UNROLL, int RPG = 1>
struct StreamCfg {
  static constexpr int kCap = CAP, kRowCap = ROWS, kWarps = WARPS, kG = G, kStages = STAGES, kUnroll = UNROLL;
  static constexpr int kRpg = RPG;
  static constexpr int kThreads = (WARPS + 1) * 32;
  static_assert(CAP % 4 == 0 && ROWS < 65535 && CAP < 65536 && 32 % G == 0 && STAGES >= 2 && STAGES <= 8,
                "stream shape");
  template <typename T, int NV>
  static constexpr uint32_t stage_bytes() {
    return pack_bytes<T, NV>(CAP, ROWS);
  }
};

// The shapes the library launches, per value type and block shape (all 8 consumer warps + 1
// producer warp: kStreamThreads threads).  3x3 (fine level; measured on the 1M-DOF I-beam,
// 17,125 tiles of ~20 rows of ~25 blocks: FP32 SpMV 63 us with 8 consumer warps, 3 stages of
// 20.7 KB and 3 CTAs per SM, against 72-90 us for 12-16 warps at 2 CTAs or 4-8 stages at 1 CTA;
// in FP32, 8 lanes per row with 4 blocks in flight each (four rows per warp: a tile in one pass
// of the 8 warps, three shuffle levels) ran the fused V-cycle passes 12-16 % faster than 16
// lanes x 2 blocks (0.74 vs 0.62 of HBM for the Chebyshev step; 4 x 8 and two rows per group
// were slower); FP64 104 us with 2 stages of 39 KB and 2 CTAs per SM, 8 lanes x 4 blocks
// as well: 3 % off the FP64 solve against 16 x 2).  6x6 (AMG level 1, rows
// of ~54 blocks) and 6x3 (restriction, rows of ~105 blocks): a warp per row (16 lanes with one
// or two blocks each were slower); 3x6 (prolongation, rows of ~5.5 blocks): 4 lanes per row,
// two blocks in flight per lane, two rows per lane group (5 % faster than one).
constexpr int kStreamThreads = 9 * 32;
template <typename T, int BR, int BC>
struct StreamDefault;
template <>
struct StreamDefault<float, 3, 3> {
  using type = StreamCfg<kStreamCap, kStreamRowCap, 8, 8, 3, 4>;
  static constexpr int kCtasPerSm = 3;
};
template <>
struct StreamDefault<double, 3, 3> {
  using type = StreamCfg<kStreamCap, kStreamRowCap, 8, 8, 2, 4>;
  static constexpr int kCtasPerSm = 2;
};
template <typename T>
struct StreamDefault<T, 6, 6> {
  using type = StreamCfg<256, kStreamRowCap, 8, 32, 2, 1>;
  static constexpr int kCtasPerSm = sizeof(T) == 4 ? 2 : 1;
};
// 6x6 operators with short rows (the level-1 and level-2 prolongations: ~5-8 blocks per row):
// 8 lanes per row, 4 rows per warp, on the same tiles and packs as the default 6x6 shape
template <typename T>
struct StreamShort66 {
  using type = StreamCfg<256, kStreamRowCap, 8, 8, 2, 1>;
  static constexpr int kCtasPerSm = sizeof(T) == 4 ? 2 : 1;
  static_assert(type::kCap == StreamDefault<T, 6, 6>::type::kCap &&
                    type::kRowCap == StreamDefault<T, 6, 6>::type::kRowCap,
                "the short-row shape streams the default 6x6 tiles");
};
template <typename T>
struct StreamDefault<T, 6, 3> {
  using type = StreamCfg<512, kStreamRowCap, 8, 32, 2, 2>;
  static constexpr int kCtasPerSm = sizeof(T) == 4 ? 2 : 1;
};
template <typename T>
struct StreamDefault<T, 3, 6> {
  using type = StreamCfg<512, kStreamRowCap, 8, 4, 2, 2, 2>;
  static constexpr int kCtasPerSm = sizeof(T) == 4 ? 2 : 1;
};
// The fine 3x3 level with FP16 values (the equilibrated matrix S A S of the FP16 V-cycle) and
// FP32 arithmetic: the tiles of the FP32 / FP64 packs, stages of half the bytes, so four of them
// per CTA at three CTAs per SM.
struct StreamHalf33 {
  using type = StreamCfg<kStreamCap, kStreamRowCap, 8, 8, 4, 4>;
  using value = __half;
  static constexpr int kCtasPerSm = 3;
  static_assert(type::kCap == StreamDefault<float, 3, 3>::type::kCap &&
                    type::kRowCap == StreamDefault<float, 3, 3>::type::kRowCap,
                "the FP16 shape streams the default 3x3 tiles");
};
// storage type of a shape's matrix values: SHAPE::value when the shape names one, else T
template <typename SHAPE, typename T, typename = void>
struct ShapeValue {
  using type = T;
};
template <typename SHAPE, typename T>
struct ShapeValue<SHAPE, T, std::void_t<typename SHAPE::value>> {
  using type = typename SHAPE::value;
};

template <typename T, int BR, int BC, typename Cfg = typename StreamDefault<T, BR, BC>::type>
constexpr size_t stream_smem_bytes() {
  return kStreamHeader + (size_t)Cfg::kStages * Cfg::template stage_bytes<T, BR * BC>();
}

// Tiles of whole rows, greedy in row order, at most `cap` blocks and `row_cap` rows each.
// False if a row alone exceeds `cap` blocks (the engine then cannot take the matrix).
inline bool build_stream_tiles(const int32_t* rp, int64_t n_rows, std::vector<StreamTile>& out,
                               int cap = kStreamCap, int row_cap = kStreamRowCap) {
  out.clear();
  int64_t r = 0;
  while (r < n_rows) {
    const int64_t r0 = r;
    if (rp[r + 1] - rp[r] > cap) return false;
    while (r < n_rows && r - r0 < row_cap && rp[r + 1] - rp[r0] <= cap) ++r;
    out.push_back({(int32_t)r0, (int32_t)r, rp[r0], rp[r]});
  }
  return true;
}

// Segment descriptors of the pack for value type T; returns the pack size in bytes (-1 when
// it would not be addressable with 32-bit 128-byte segment indices).
template <typename T, int NV>
inline int64_t build_pack_tiles(const std::vector<StreamTile>& plan, std::vector<PackTile>& out) {
  out.resize(plan.size());
  int64_t seg = 0;  // in 128-byte units
  for (size_t t = 0; t < plan.size(); ++t) {
    const StreamTile& p = plan[t];
    const int cntp = pack_cntp(p.b1 - p.b0);
    if (seg > INT32_MAX) return -1;
    out[t] = {p.r0, p.r1, (int32_t)seg, cntp};
    seg += pack_bytes<T, NV>(cntp, p.r1 - p.r0) / 128;
  }
  return seg * 128;
}

#if defined(__CUDACC__)

// Pack a matrix of NV values per block tile-major: source component k of block b at
// v[k * stride + b] (component-major, stride > 0) or v[b * NV + k] (block-contiguous,
// stride == 0).  One CTA per tile, grid-stride; padding is written as zeros.
template <typename T, int NV>
__global__ void __launch_bounds__(256) k_pack_tiles(int n_tiles, const StreamTile* __restrict__ plan,
                                                    const PackTile* __restrict__ desc, const int32_t* __restrict__ rp,
                                                    const int32_t* __restrict__ ci, const T* __restrict__ v,
                                                    int64_t stride, unsigned char* __restrict__ pack) {
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const StreamTile p = plan[t];
    const PackTile d = desc[t];
    const int cnt = p.b1 - p.b0, cntp = d.cntp, nr = p.r1 - p.r0;
    unsigned char* seg = pack + (size_t)d.seg * 128;
    T* sv = reinterpret_cast<T*>(seg);
    if (stride > 0) {
      for (int k = 0; k < NV; ++k)
        for (int b = threadIdx.x; b < cntp; b += blockDim.x)
          sv[k * cntp + b] = b < cnt ? v[(int64_t)k * stride + p.b0 + b] : T(0);
    } else {
      for (int q = threadIdx.x; q < NV * cntp; q += blockDim.x) {  // read coalesced, write strided
        const int b = q / NV, k = q - b * NV;
        sv[k * cntp + b] = b < cnt ? v[((int64_t)p.b0 + b) * NV + k] : T(0);
      }
    }
    int32_t* sc = reinterpret_cast<int32_t*>(seg + pack_col_off<T, NV>(cntp));
    for (int b = threadIdx.x; b < cntp; b += blockDim.x) sc[b] = b < cnt ? ci[p.b0 + b] : 0;
    uint16_t* sr = reinterpret_cast<uint16_t*>(seg + pack_row_off<T, NV>(cntp));
    const int slots = (int)(pack_bytes<T, NV>(cntp, nr) - pack_row_off<T, NV>(cntp)) / 2;
    for (int i = threadIdx.x; i < slots; i += blockDim.x) sr[i] = (uint16_t)(i <= nr ? rp[p.r0 + i] - p.b0 : 0);
  }
}

// The FP16 pack of the equilibrated 3x3 matrix S A S, S = diag(scale): component k = 3 r + c of
// block b (row br, column bc) is v[k stride + b] scale[3 br + r] scale[3 bc + c], formed in FP64
// and rounded to FP16 once.  With scale = diag(A)^-1/2 the matrix has a unit diagonal and, A
// being symmetric positive (semi)definite, entries of magnitude <= 1.  Same tiles and layout as
// k_pack_tiles<__half, 9>.
static __global__ void __launch_bounds__(256) k_pack_half33(int n_tiles, const StreamTile* __restrict__ plan,
                                                     const PackTile* __restrict__ desc, const int32_t* __restrict__ rp,
                                                     const int32_t* __restrict__ ci,
                                                     const int32_t* __restrict__ block_row,
                                                     const double* __restrict__ v, int64_t stride,
                                                     const double* __restrict__ scale, unsigned char* __restrict__ pack) {
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const StreamTile p = plan[t];
    const PackTile d = desc[t];
    const int cnt = p.b1 - p.b0, cntp = d.cntp, nr = p.r1 - p.r0;
    unsigned char* seg = pack + (size_t)d.seg * 128;
    __half* sv = reinterpret_cast<__half*>(seg);
    for (int k = 0; k < 9; ++k) {
      const int r = k / 3, c = k - 3 * (k / 3);
      for (int b = threadIdx.x; b < cntp; b += blockDim.x) {
        double a = 0.0;
        if (b < cnt) {
          const int64_t q = p.b0 + b;
          a = v[(int64_t)k * stride + q] * scale[(int64_t)block_row[q] * 3 + r] * scale[(int64_t)ci[q] * 3 + c];
        }
        sv[k * cntp + b] = __double2half(a);
      }
    }
    int32_t* sc = reinterpret_cast<int32_t*>(seg + pack_col_off<__half, 9>(cntp));
    for (int b = threadIdx.x; b < cntp; b += blockDim.x) sc[b] = b < cnt ? ci[p.b0 + b] : 0;
    uint16_t* sr = reinterpret_cast<uint16_t*>(seg + pack_row_off<__half, 9>(cntp));
    const int slots = (int)(pack_bytes<__half, 9>(cntp, nr) - pack_row_off<__half, 9>(cntp)) / 2;
    for (int i = threadIdx.x; i < slots; i += blockDim.x) sr[i] = (uint16_t)(i <= nr ? rp[p.r0 + i] - p.b0 : 0);
  }
}

// Bounded waits of the pipeline.  ctl.wait_ns bounds every stage wait (consumers waiting for a
// tile, the producer waiting for a free stage); the host sets it per matrix (default 4 s).  After
// a failure the copies still in flight are drained with their own fixed limit, so a short
// ctl.wait_ns never lets a CTA exit before its copies have landed.  ctl.withhold >= 0 is the
// failure-detection test hook: the producer skips that tile's copy (nothing arms its stage), so
// the consumers' wait for it must run out and the call must report WN_ETIMEOUT.
constexpr unsigned long long kStreamWaitLimitNs = 4000000000ull;   // 4 s: default stage-wait limit
constexpr unsigned long long kStreamDrainLimitNs = 4000000000ull;  // 4 s: drain of issued copies
struct StreamCtl {
  unsigned long long wait_ns = kStreamWaitLimitNs;
  int withhold = -1;  // tile index withheld by the producer (tests only), -1: none
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// bulk async copy global -> this CTA's shared memory, completion counted on `bar` (bytes and
// both addresses multiples of 16)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
      : "memory");
}

// one thread: wait for the phase of `parity` to complete; false after limit_ns or when
// `abort_flag` is raised (abort_flag may be null)
__device__ __forceinline__ bool wait_thread(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                            unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t n = 1;; ++n) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((n & 63) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (global_ns() - t0 > limit_ns) return false;
    }
  }
}

// a full warp: every lane polls, the warp leaves together (all lanes saw the phase complete,
// or one lane saw the limit / the abort flag)
__device__ __forceinline__ bool wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned long long limit_ns) {
  if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t n = 1;; ++n) {
    if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
    if ((n & 63) == 0) {
      const bool stop = *abort_flag != 0 || global_ns() - t0 > limit_ns;
      if (__any_sync(0xffffffffu, stop)) return false;
    }
  }
}

// Programmatic dependent launch (griddepcontrol): a kernel launched with programmatic stream
// serialisation may start while its predecessor is still running; pdl_wait() blocks until the
// predecessor has completed and its memory is visible (an immediate return for an ordinary
// launch); pdl_trigger() lets this kernel's dependents be scheduled.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// called by every thread of the CTA once the predecessor's results are visible
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};


// The tile pipeline.  Every thread of a CTA of Cfg::kThreads threads calls it once (dynamic
// shared memory of stream_smem_bytes<T, BR, BC, Cfg>()); the pack was built from a plan with
// Cfg's capacities (NV = BR * BC values per block).  The producer warp streams the CTA's run of
// tiles into the stage ring; every consumer warp calls body(jc, stage, desc, dot) for each tile jc
// of the run (stage = the tile's image in shared memory, desc = rows r0, r1 / segment /
// cntp), adding its dot contributions to the consumer's running sum, which is returned (0 for
// the producer).
// The first stages' copies (the matrix only) are issued before pdl_wait(), so under a
// programmatic dependent launch they overlap the predecessor's tail; then every thread runs
// hook(), and when *done is set (read after the wait) the CTA lets those copies land and
// returns with *skipped = true.  Every warp of the CTA meets once more at the end; if any wait
// ran out, one thread then waits (bounded) for the copies still in flight before the CTA exits.
template <typename T, int NV, typename Cfg, typename BODY, typename HOOK>
__device__ __forceinline__ double stream_pipeline(const PackTile* __restrict__ tiles, int n_tiles,
                                                  const unsigned char* __restrict__ pack, unsigned char* smem,
                                                  int* status, int* done, const StreamCtl ctl, bool* skipped,
                                                  const HOOK& hook, BODY& body) {
  constexpr int STAGES = Cfg::kStages;
  constexpr uint32_t SB = Cfg::template stage_bytes<T, NV>();
  constexpr int NCW = Cfg::kWarps;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + STAGES;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 256);
  volatile int* skip_flag = reinterpret_cast<volatile int*>(smem + 260);
  int4* descs = reinterpret_cast<int4*>(smem + 384);
  unsigned char* stages = smem + kStreamHeader;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this CTA's tiles: a contiguous run [tb, te)
  const int tb = (int)((int64_t)blockIdx.x * n_tiles / gridDim.x);
  const int te = (int)((int64_t)(blockIdx.x + 1) * n_tiles / gridDim.x);
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, NCW);
    }
    *abort_flag = 0;
    mbar_init_fence();
  }
  __syncthreads();
  double dot = 0.0;
  auto fail = [&]() {
    *abort_flag = 1;
    *status = WN_ETIMEOUT;
    if (done) *(volatile int*)done = 1;
  };

  // producer warp: lane 0 issues, the warp holds the tile descriptors of tiles tb + 32 c + lane
  // in chunks (the next chunk loaded while the current one is issued)
  const int n_my = te - tb;
  uint64_t pol = 0;
  int4 cur = make_int4(0, 0, 0, 0), nxt = make_int4(0, 0, 0, 0);
  int j = 0;  // tiles issued
  bool ok = true;
  auto load_chunk = [&](int c) {
    const int t = tb + 32 * c + lane;
    return t < te ? *reinterpret_cast<const int4*>(tiles + t) : make_int4(0, 0, 0, 0);
  };
  auto issue = [&](int j_end) {  // the whole producer warp: issue tiles j .. j_end - 1
    for (; j < j_end; ++j) {
      const int q = j & 31;
      int4 d;
      d.x = __shfl_sync(0xffffffffu, cur.x, q);
      d.y = __shfl_sync(0xffffffffu, cur.y, q);
      d.z = __shfl_sync(0xffffffffu, cur.z, q);
      d.w = __shfl_sync(0xffffffffu, cur.w, q);
      if (q == 31) {
        cur = nxt;
        nxt = load_chunk((j >> 5) + 2);
      }
      if (lane == 0) {
        const int s = j % STAGES;
        if (j >= STAGES && !wait_thread(empty + s, (uint32_t)((j / STAGES - 1) & 1), abort_flag, ctl.wait_ns)) {
          ok = false;
        } else if (tb + j != ctl.withhold) {
          descs[s] = d;
          const uint32_t bytes = pack_bytes<T, NV>(d.w, d.y - d.x);
          mbar_arrive_expect_tx(full + s, bytes);
          bulk_load(stages + (size_t)s * SB, pack + (size_t)d.z * 128, bytes, full + s, pol);
        }
      }
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
    }
  };
  const int pre = n_my < STAGES ? n_my : STAGES;
  if (warp == NCW) {
    pol = l2_evict_first_policy();
    cur = load_chunk(0);
    nxt = load_chunk(1);
    issue(pre);  // free stages: no waits
  }
  pdl_wait();
  if (threadIdx.x == 0) *skip_flag = (done && *(volatile int*)done) ? 1 : 0;
  __syncthreads();
  hook();
  const bool skip = *skip_flag != 0;
  if (skipped) *skipped = skip;
  // the copies issued so far (j tiles processed by the producer) into this CTA's stages: for each
  // stage, wait (bounded) for the phase of the last tile actually copied into it
  auto drain = [&]() {
    for (int s = 0; s < STAGES && s < j; ++s) {
      int t = s + STAGES * ((j - 1 - s) / STAGES);  // last tile processed into stage s
      if (tb + t == ctl.withhold) t -= STAGES;        // withheld: its predecessor was the last copy
      if (t >= 0) wait_thread(full + s, (uint32_t)((t / STAGES) & 1), nullptr, kStreamDrainLimitNs);
    }
  };
  if (skip) {  // let the copies already issued land before the CTA can exit
    if (warp == NCW && lane == 0) drain();
    return 0.0;
  }

  if (warp == NCW) {
    issue(n_my);
    if (lane == 0 && !ok) fail();
    __syncwarp();
  } else {
    // consumer warps
    for (int jc = 0; jc < n_my; ++jc) {
      const int s = jc % STAGES;
      if (!wait_warp(full + s, (uint32_t)((jc / STAGES) & 1), abort_flag, ctl.wait_ns)) {
        if (lane == 0) fail();
        break;
      }
      body(jc, stages + (size_t)s * SB, descs[s], dot);
      __syncwarp();
      if (lane == 0) mbar_arrive(empty + s);
    }
  }
  // every warp meets here; after a failure (some wait ran out, or the abort flag was raised)
  // the producer's lane 0 waits for the copies it issued before the CTA can exit
  __syncthreads();
  if (*abort_flag && warp == NCW && lane == 0) drain();
  return dot;
}

__host__ __device__ constexpr int pow2_ceil(int v) { return v <= 1 ? 1 : 2 * pow2_ceil((v + 1) / 2); }
__host__ __device__ constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v / 2); }

// Sum of a[0 .. BR) over the G lanes of a row group, transposed: with P = BR rounded up to a
// power of two, each of the first log2 P butterfly levels halves the values a lane holds -- it
// keeps one half and trades the other with its partner -- and the remaining levels are plain
// butterflies.  Lane gl ends with the whole sum of value gl >> (log2 G - log2 P): log2 P + P - 1
// shuffles instead of BR log2 G (9 instead of 30 for 6 values over 32 lanes).
template <int BR, int G, typename T>
__device__ __forceinline__ T group_sum_transposed(const T (&a)[BR], int gl) {
  constexpr int P = pow2_ceil(BR), LG = ilog2(G), LP = ilog2(P);
  static_assert(G >= P && (1 << LG) == G, "a power-of-two group of at least P lanes");
  T v[P];
#pragma unroll
  for (int r = 0; r < P; ++r) v[r] = r < BR ? a[r] : T(0);
#pragma unroll
  for (int k = 0; k < LG; ++k) {
    const int o = G >> (k + 1);
    if (k < LP) {
      const int h = P >> (k + 1);
      const bool up = (gl & o) != 0;
#pragma unroll
      for (int j = 0; j < h; ++j) {
        const T send = up ? v[j] : v[j + h];
        const T keep = up ? v[j + h] : v[j];
        v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    }
  }
  return v[0];
}

// a stored matrix value in the arithmetic type
template <typename T, typename TV>
__device__ __forceinline__ T value_as(TV v) {
  if constexpr (std::is_same<TV, __half>::value)
    return (T)__half2float(v);
  else
    return (T)v;
}

// The row engine: y-rows of A x with G lanes per block row (lane l taking the row's blocks
// l, l + G, ...; U blocks in flight per lane, R rows per lane group), for every row DOF
// i = BR row + c of the CTA's tiles the owning lane (c < BR <= G) calls pre = epi.load(i) before
// the row product and dot += epi.store(i, pre, (A x)_i) after it, with x_j = xf(j)
// (j = BC col + c).  Returns the thread's dot sum (0 for the producer).  The pack stores its
// values as TV (T, or FP16 for an FP32 product), the arithmetic is T.
template <typename T, typename TV, int BR, int BC, typename Cfg, typename XF, typename EPI, typename HOOK = NoHook>
__device__ __forceinline__ double stream_rows_v(const PackTile* __restrict__ tiles, int n_tiles,
                                                const unsigned char* __restrict__ pack, const XF& xf, const EPI& epi,
                                                unsigned char* smem, int* status, int* done, const StreamCtl ctl,
                                                bool* skipped = nullptr, const HOOK& hook = HOOK{}) {
  constexpr int NV = BR * BC;
  constexpr int G = Cfg::kG;
  constexpr int U = Cfg::kUnroll;
  constexpr int R = Cfg::kRpg;
  constexpr int GPW = 32 / G;  // row groups per warp
  constexpr int NCW = Cfg::kWarps;
  static_assert(BR <= G, "a lane per row DOF");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gl = lane % G, grp = lane / G;
  // after group_sum_transposed, row DOF r's sum is in lanes r << SH .. ((r + 1) << SH) - 1; the
  // first of them loads the DOF's epilogue operands and stores its result
  constexpr int SH = ilog2(G) - ilog2(pow2_ceil(BR));
  const int my_r = gl >> SH;
  const bool owner = (gl & ((1 << SH) - 1)) == 0 && my_r < BR;
  auto body = [&](int jc, const unsigned char* st, const int4 d, double& dot) {
    const int r0 = d.x, nr = d.y - d.x, cntp = d.w;
    const TV* sv = reinterpret_cast<const TV*>(st);
    const int32_t* scol = reinterpret_cast<const int32_t*>(st + pack_col_off<TV, NV>(cntp));
    const uint16_t* srp = reinterpret_cast<const uint16_t*>(st + pack_row_off<TV, NV>(cntp));
    // warps take the tile's rows round-robin in passes of GPW * R rows (group g of a pass owns
    // rows base + q GPW + g, q < R), starting from a warp that rotates per tile
    const int wslot = (warp + jc) % NCW;
    for (int base = wslot * GPW * R; base < nr; base += NCW * GPW * R) {
      int rs[R], re[R];
      typename EPI::Pre pre[R];
      T acc[R][BR];
      int len = 0;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int lr = base + q * GPW + grp;
        const bool active = lr < nr;
        rs[q] = active ? srp[lr] : 0;
        re[q] = active ? srp[lr + 1] : 0;
        len = max(len, re[q] - rs[q]);
        pre[q] = typename EPI::Pre{};
        if (active && owner) pre[q] = epi.load((int64_t)(r0 + lr) * BR + my_r);
#pragma unroll
        for (int r = 0; r < BR; ++r) acc[q][r] = T(0);
      }
      // U blocks of each of the R rows in flight per lane: their gathers are issued before the
      // first multiply-add; each row's sum still runs over the lane's blocks in order
      // (b, b + G, b + 2G, ...)
      for (int o = gl; o < len; o += G * U) {
        int col[R][U];
        T xv[R][U][BC];
#pragma unroll
        for (int q = 0; q < R; ++q)
#pragma unroll
          for (int u = 0; u < U; ++u) col[q][u] = (rs[q] + o + u * G < re[q]) ? scol[rs[q] + o + u * G] : 0;
#pragma unroll
        for (int q = 0; q < R; ++q)
#pragma unroll
          for (int u = 0; u < U; ++u)
#pragma unroll
            for (int c = 0; c < BC; ++c) xv[q][u][c] = xf((int64_t)col[q][u] * BC + c);
#pragma unroll
        for (int q = 0; q < R; ++q)
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int b = rs[q] + o + u * G;
            if (b < re[q]) {
#pragma unroll
              for (int r = 0; r < BR; ++r)
#pragma unroll
                for (int c = 0; c < BC; ++c)
                  acc[q][r] = fma(value_as<T>(sv[(r * BC + c) * cntp + b]), xv[q][u][c], acc[q][r]);
            }
          }
      }
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const T sum = group_sum_transposed<BR, G>(acc[q], gl);
        const int lr = base + q * GPW + grp;
        if (lr < nr && owner) dot += epi.store((int64_t)(r0 + lr) * BR + my_r, pre[q], sum);
      }
    }
  };
  return stream_pipeline<TV, NV, Cfg>(tiles, n_tiles, pack, smem, status, done, ctl, skipped, hook, body);
}
template <typename T, int BR, int BC, typename Cfg, typename XF, typename EPI, typename HOOK = NoHook>
__device__ __forceinline__ double stream_rows(const PackTile* __restrict__ tiles, int n_tiles,
                                              const unsigned char* __restrict__ pack, const XF& xf, const EPI& epi,
                                              unsigned char* smem, int* status, int* done, const StreamCtl ctl,
                                              bool* skipped = nullptr, const HOOK& hook = HOOK{}) {
  return stream_rows_v<T, T, BR, BC, Cfg>(tiles, n_tiles, pack, xf, epi, smem, status, done, ctl, skipped, hook);
}

#endif  // __CUDACC__

}  // namespace wn
