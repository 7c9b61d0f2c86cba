// extern "C" boundary of libwnfea_cuda: handle management, assembly, SpMV and element-level
// entry points (declared in include/wnfea_cuda.h).
#include <cstdarg>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "wnfea_cuda.h"
#include "common.cuh"
#include "amg.h"
#include "block.h"
#include "kernels.h"
#include "solid.h"

namespace wn {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}
const char* last_error() { return g_last_error.c_str(); }

// CTAs per SM of a kernel with `smem` bytes of dynamic shared memory, after raising the
// kernel's dynamic shared memory limit to `smem` (once per device); 0 if the kernel cannot
// be launched with that much
int stream_ctas_per_sm(const void* kernel, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair(dev, kernel);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n < 0) {
    cudaGetLastError();
    n = 0;
  }
  cache[key] = n;
  return n;
}

int occupancy_per_sm(const void* kernel, int threads) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair(kernel, threads);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess || n < 1) n = 1;
  cache[key] = n;
  return n;
}

__global__ void grad_f_kernel(int64_t n, const double* __restrict__ u, const uint8_t* __restrict__ fixed,
                              double* __restrict__ g) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    g[i] = (fixed && fixed[i]) ? 0.0 : 2.0 * u[i];
}

static Solid* as_solid(void* h) { return reinterpret_cast<Solid*>(h); }

static int select_device(Solid* s) {
  WN_CUDA(cudaSetDevice(s->device));
  return 0;
}

static int read_flag(Solid* s, cudaStream_t st, int* value) {
  WN_CUDA(cudaMemcpyAsync(value, s->flags.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  return 0;
}

__global__ void to_float_kernel(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

int make_bsr6_system(int64_t n, const int32_t* rp, const int32_t* ci, const double* values, bool values_on_device,
                     const double* coords, const uint8_t* fixed, void** out) {
  *out = nullptr;
  WN_REQUIRE(n < (int64_t)INT32_MAX / 6 && rp[0] == 0, WN_EINVAL, "6x6 system: bad row pointer");
  const int64_t nnzb = rp[n];
  std::vector<int32_t> diag(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    WN_REQUIRE(rp[i + 1] >= rp[i], WN_EINVAL, "6x6 system: row pointer not monotone");
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
      WN_REQUIRE(ci[k] >= 0 && ci[k] < n, WN_EINVAL, "6x6 system: column index out of range");
      WN_REQUIRE(k == rp[i] || ci[k] > ci[k - 1], WN_EINVAL, "6x6 system: columns not sorted / unique in row %lld",
                 (long long)i);
      if (ci[k] == i) diag[i] = k;
    }
    WN_REQUIRE(diag[i] >= 0, WN_EINVAL, "6x6 system: row %lld has no diagonal block", (long long)i);
  }
  int dev = 0;
  WN_CUDA(cudaGetDevice(&dev));
  std::unique_ptr<Solid> s(new Solid());
  s->device = dev;
  s->bs = 6;
  s->n_nodes = n;
  s->n_el = 0;
  s->nnzb = nnzb;
  s->h_row_ptr.assign(rp, rp + n + 1);
  s->h_col_idx.assign(ci, ci + nnzb);
  s->h_diag_block = diag;
  s->h_nodes.assign(coords, coords + n * 3);
  s->h_fixed.assign(n * 6, 0);
  if (fixed)
    for (int64_t i = 0; i < n * 6; ++i) s->h_fixed[i] = fixed[i] ? 1 : 0;
  WN_CHECK(s->row_ptr.upload(s->h_row_ptr));
  WN_CHECK(s->col_idx.upload(s->h_col_idx));
  WN_CHECK(s->diag_block.upload(s->h_diag_block));
  WN_CHECK(s->fixed.upload(s->h_fixed));
  WN_CHECK(s->flags.alloc(16));
  WN_CHECK(s->flags.zero());
  WN_CHECK(s->k64.alloc(nnzb * 36));
  WN_CHECK(s->k32.alloc(nnzb * 36));
  WN_CUDA(cudaMemcpy(s->k64.p, values, nnzb * 36 * sizeof(double),
                     values_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
  to_float_kernel<<<grid_for(nnzb * 36, 1, 256, 8), 256>>>(nnzb * 36, s->k64.p, s->k32.p);
  WN_CUDA(cudaGetLastError());
  WN_CHECK(s->fine.make_plan(rp, n, 6, 6));
  WN_CHECK(s->fine.pack(s->row_ptr.p, s->col_idx.p, s->k32.p, s->k64.p, 0, 0));
  WN_CUDA(cudaDeviceSynchronize());
  ++s->values_version;
  s->assembled = true;
  s->bcs_applied = fixed != nullptr;
  *out = s.release();
  return 0;
}

}  // namespace wn

using namespace wn;

namespace {

// Device buffers of the stateless host-buffer internal-force call, kept per device and grown
// on demand (never shrunk) so that repeated calls neither allocate nor free.
struct FintWorkspace {
  DArray<double> nodes, props, u, f, fe;
  DArray<int32_t> conn, counts, inc;
  DArray<int64_t> inc_ptr, scan;
  DArray<int> flags;
  template <typename T>
  static int at_least(DArray<T>& a, int64_t n) {
    return a.n >= n ? 0 : a.alloc(n);
  }
  int grow(int64_t nn, int64_t ne) {
    WN_CHECK(at_least(nodes, nn * 3));
    WN_CHECK(at_least(u, nn * 6));
    WN_CHECK(at_least(f, nn * 6));
    WN_CHECK(at_least(props, ne * 2));
    WN_CHECK(at_least(fe, ne * 30));
    WN_CHECK(at_least(conn, ne * 10));
    WN_CHECK(at_least(counts, nn));
    WN_CHECK(at_least(inc, ne * 10));
    WN_CHECK(at_least(scan, (nn + 1023) / 1024 + 1));
    WN_CHECK(at_least(inc_ptr, nn + 1));
    WN_CHECK(at_least(flags, 2));
    return 0;
  }
};

std::mutex& fint_workspace_mutex() {
  static std::mutex mu;
  return mu;
}

FintWorkspace& fint_workspace(int dev) {
  static std::map<int, std::unique_ptr<FintWorkspace>> ws;
  auto& p = ws[dev];
  if (!p) p.reset(new FintWorkspace());
  return *p;
}

}  // namespace

extern "C" {

const char* wn_last_error_string(void) { return wn::last_error(); }

int wn_version(void) { return 100; }

int wn_device_synchronize(void) {
  WN_CUDA(cudaDeviceSynchronize());
  return 0;
}

int wn_solid_create(int64_t n_nodes, int64_t n_el, const double* nodes, const int32_t* conn, void** out_handle) {
  WN_REQUIRE(out_handle && nodes && (conn || n_el == 0), WN_EINVAL, "wn_solid_create: null argument");
  WN_REQUIRE(n_nodes > 0 && n_el >= 0, WN_EINVAL, "wn_solid_create: bad sizes n_nodes=%lld n_el=%lld",
             (long long)n_nodes, (long long)n_el);
  WN_REQUIRE(n_nodes < (int64_t)INT32_MAX / 6, WN_ETOOBIG, "wn_solid_create: too many nodes");
  *out_handle = nullptr;
  int dev = 0;
  WN_CUDA(cudaGetDevice(&dev));
  Bsr3Pattern pat;
  int rc = build_bsr3_pattern(n_nodes, n_el, conn, pat);
  WN_REQUIRE(rc != -3, WN_EMESH, "wn_solid_create: element node index out of range [0, %lld)", (long long)n_nodes);
  WN_REQUIRE(rc != -8, WN_ETOOBIG, "wn_solid_create: mesh too large for 32-bit block indices");
  WN_REQUIRE(rc == 0, WN_EINVAL, "wn_solid_create: pattern construction failed (%d)", rc);
  auto* s = new Solid();
  s->device = dev;
  s->n_nodes = n_nodes;
  s->n_el = n_el;
  s->nnzb = pat.nnzb;
  s->h_nodes.assign(nodes, nodes + n_nodes * 3);
  int st = 0;
  st = st ? st : s->nodes.upload(nodes, n_nodes * 3);
  st = st ? st : s->conn.upload(conn, n_el * 10);
  st = st ? st : s->row_ptr.upload(pat.row_ptr);
  st = st ? st : s->col_idx.upload(pat.col_idx);
  st = st ? st : s->block_row.upload(pat.block_row);
  st = st ? st : s->diag_block.upload(pat.diag_block);
  st = st ? st : s->emap.upload(pat.emap);
  st = st ? st : s->gptr.upload(pat.gather_ptr);
  {
    // tile-owner assembly when every tile's incident elements and contribution codes fit in
    // shared memory (at most 200 elements); the tiles are those of the streamed fine matrix
    AssemblyPlan plan;
    std::vector<StreamTile> stiles;
    const bool ok = build_assembly_plan(pat, n_el, kStreamCap, kStreamRowCap, 200, plan) == 0 &&
                    assemble_tiles_smem(plan.ne_max, plan.max_codes) <= kAsmSmemLimit &&
                    build_stream_tiles(pat.row_ptr.data(), n_nodes, stiles) && stiles.size() == plan.tiles.size();
    bool same = ok;
    for (size_t t = 0; same && t < stiles.size(); ++t)
      same = stiles[t].r0 == plan.tiles[t].r0 && stiles[t].r1 == plan.tiles[t].r1;
    if (same && plan.n_tiles > 0) {
      s->asm_tiles = plan.n_tiles;
      s->asm_ne_max = plan.ne_max;
      s->asm_max_codes = plan.max_codes;
      std::vector<int32_t> tl(plan.tiles.size() * 4);
      for (size_t t = 0; t < plan.tiles.size(); ++t) {
        tl[4 * t] = plan.tiles[t].r0;
        tl[4 * t + 1] = plan.tiles[t].r1;
        tl[4 * t + 2] = plan.tiles[t].b0;
        tl[4 * t + 3] = plan.tiles[t].b1;
      }
      st = st ? st : s->asm_tile.upload(tl);
      std::vector<int32_t> hdr(plan.tiles.size() * 8, 0);
      for (size_t t = 0; t < plan.tiles.size(); ++t) {
        int32_t* h = &hdr[8 * t];
        h[0] = plan.el_ptr[t];
        h[1] = plan.el_ptr[t + 1] - plan.el_ptr[t];
        h[2] = plan.chunk_ptr[t];
        h[3] = plan.chunk_ptr[t + 1] - plan.chunk_ptr[t];
        h[4] = plan.n_split[t];
        h[5] = pat.gather_ptr[plan.tiles[t].b0];
        h[6] = pat.gather_ptr[plan.tiles[t].b1] - pat.gather_ptr[plan.tiles[t].b0];
      }
      st = st ? st : s->asm_hdr.upload(hdr);
      st = st ? st : s->asm_el.upload(plan.el);
      st = st ? st : s->asm_perm.upload(plan.perm);
      st = st ? st : s->asm_contrib.upload(plan.contrib);
      st = st ? st : s->asm_chunks.upload(plan.chunks);
    } else {
      st = st ? st : s->gsrc.upload(pat.gather_src);
    }
  }
  st = st ? st : s->inc_ptr.upload(pat.inc_ptr);
  st = st ? st : s->inc_ea.upload(pat.inc_ea);
  st = st ? st : s->flags.alloc(16);
  st = st ? st : s->flags.zero();
  st = st ? st : s->fixed.alloc(n_nodes * 3);
  st = st ? st : s->fixed.zero();
  st = st ? st : s->fine.make_plan(pat.row_ptr.data(), n_nodes, 3, 3);
  if (st == 0) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_error("wn_solid_create: %s", cudaGetErrorString(e));
      st = (int)e;
    }
  }
  if (st != 0) {
    delete s;
    return st;
  }
  s->h_row_ptr = std::move(pat.row_ptr);
  s->h_col_idx = std::move(pat.col_idx);
  s->h_diag_block = std::move(pat.diag_block);
  s->h_fixed.assign(n_nodes * 3, 0);
  *out_handle = s;
  return 0;
}

int wn_assembly_plan_host(int64_t n_nodes, int64_t n_el, const int32_t* conn, int64_t* n_tiles, int* ne_max,
                          int64_t* n_el_entries, int32_t* tiles, int32_t* el_ptr, int32_t* el, uint16_t* contrib,
                          uint16_t* perm) {
  WN_REQUIRE(n_tiles && ne_max && n_el_entries && (conn || n_el == 0) && n_nodes > 0 && n_el >= 0, WN_EINVAL,
             "wn_assembly_plan_host: bad argument");
  Bsr3Pattern pat;
  int rc = build_bsr3_pattern(n_nodes, n_el, conn, pat);
  WN_REQUIRE(rc != -3, WN_EMESH, "wn_assembly_plan_host: element node index out of range");
  WN_REQUIRE(rc == 0, WN_EINVAL, "wn_assembly_plan_host: pattern construction failed (%d)", rc);
  AssemblyPlan plan;
  if (build_assembly_plan(pat, n_el, kStreamCap, kStreamRowCap, 200, plan) != 0) {
    *n_tiles = 0;
    *ne_max = 0;
    *n_el_entries = 0;
    return 0;
  }
  *n_tiles = plan.n_tiles;
  *ne_max = plan.ne_max;
  *n_el_entries = (int64_t)plan.el.size();
  if (tiles)
    for (int t = 0; t < plan.n_tiles; ++t) {
      tiles[4 * t] = plan.tiles[t].r0;
      tiles[4 * t + 1] = plan.tiles[t].r1;
      tiles[4 * t + 2] = plan.tiles[t].b0;
      tiles[4 * t + 3] = plan.tiles[t].b1;
    }
  if (el_ptr) std::copy(plan.el_ptr.begin(), plan.el_ptr.end(), el_ptr);
  if (el) std::copy(plan.el.begin(), plan.el.end(), el);
  if (contrib) std::copy(plan.contrib.begin(), plan.contrib.end(), contrib);
  if (perm) std::copy(plan.perm.begin(), plan.perm.end(), perm);
  return 0;
}

int wn_assembly_chunks_host(int64_t n_nodes, int64_t n_el, const int32_t* conn, int* chunk_len, int* max_codes,
                            int64_t* n_chunks, int32_t* chunk_ptr, uint32_t* chunks, int32_t* n_split) {
  WN_REQUIRE(chunk_len && max_codes && n_chunks && (conn || n_el == 0) && n_nodes > 0 && n_el >= 0, WN_EINVAL,
             "wn_assembly_chunks_host: bad argument");
  Bsr3Pattern pat;
  int rc = build_bsr3_pattern(n_nodes, n_el, conn, pat);
  WN_REQUIRE(rc != -3, WN_EMESH, "wn_assembly_chunks_host: element node index out of range");
  WN_REQUIRE(rc == 0, WN_EINVAL, "wn_assembly_chunks_host: pattern construction failed (%d)", rc);
  AssemblyPlan plan;
  if (build_assembly_plan(pat, n_el, kStreamCap, kStreamRowCap, 200, plan) != 0) {
    *chunk_len = 0;
    *max_codes = 0;
    *n_chunks = 0;
    return 0;
  }
  *chunk_len = plan.chunk_len;
  *max_codes = plan.max_codes;
  *n_chunks = (int64_t)plan.chunks.size();
  if (chunk_ptr) std::copy(plan.chunk_ptr.begin(), plan.chunk_ptr.end(), chunk_ptr);
  if (chunks) std::copy(plan.chunks.begin(), plan.chunks.end(), chunks);
  if (n_split) std::copy(plan.n_split.begin(), plan.n_split.end(), n_split);
  return 0;
}

int wn_bsr3_pattern_host(int64_t n_nodes, int64_t n_el, const int32_t* conn, int64_t* nnzb, int32_t* row_ptr,
                         int32_t* col_idx, int32_t* emap) {
  WN_REQUIRE(nnzb && (conn || n_el == 0) && n_nodes > 0 && n_el >= 0, WN_EINVAL, "wn_bsr3_pattern_host: bad argument");
  Bsr3Pattern pat;
  int rc = build_bsr3_pattern(n_nodes, n_el, conn, pat);
  WN_REQUIRE(rc != -3, WN_EMESH, "wn_bsr3_pattern_host: element node index out of range");
  WN_REQUIRE(rc != -8, WN_ETOOBIG, "wn_bsr3_pattern_host: mesh too large for 32-bit block indices");
  WN_REQUIRE(rc == 0, WN_EINVAL, "wn_bsr3_pattern_host: failed (%d)", rc);
  *nnzb = pat.nnzb;
  if (row_ptr) memcpy(row_ptr, pat.row_ptr.data(), sizeof(int32_t) * (n_nodes + 1));
  if (col_idx) memcpy(col_idx, pat.col_idx.data(), sizeof(int32_t) * pat.nnzb);
  if (col_idx && emap) memcpy(emap, pat.emap.data(), sizeof(int32_t) * n_el * 100);
  return 0;
}

int wn_bsr6_system_create(int64_t n_nodes, const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                          const double* coords, const uint8_t* fixed_mask, void** out_handle) {
  WN_REQUIRE(out_handle && row_ptr && col_idx && values && coords && n_nodes > 0, WN_EINVAL,
             "wn_bsr6_system_create: bad argument");
  return make_bsr6_system(n_nodes, row_ptr, col_idx, values, false, coords, fixed_mask, out_handle);
}

int wn_solid_destroy(void* h) {
  if (!h) return 0;
  Solid* s = as_solid(h);
  cudaSetDevice(s->device);
  delete s;
  return 0;
}

int wn_solid_info(void* h, int64_t* n_nodes, int64_t* n_el, int64_t* nnzb) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_info: null handle");
  Solid* s = as_solid(h);
  if (n_nodes) *n_nodes = s->n_nodes;
  if (n_el) *n_el = s->n_el;
  if (nnzb) *nnzb = s->nnzb;
  return 0;
}

int wn_solid_get_pattern(void* h, int32_t* row_ptr, int32_t* col_idx) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_get_pattern: null handle");
  Solid* s = as_solid(h);
  if (row_ptr) memcpy(row_ptr, s->h_row_ptr.data(), sizeof(int32_t) * (s->n_nodes + 1));
  if (col_idx) memcpy(col_idx, s->h_col_idx.data(), sizeof(int32_t) * s->nnzb);
  return 0;
}

int wn_solid_get_map(void* h, int32_t* emap) {
  WN_REQUIRE(h && emap, WN_EINVAL, "wn_solid_get_map: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_solid_get_map: not a C3D10 system");
  WN_CHECK(select_device(s));
  WN_CUDA(cudaMemcpy(emap, s->emap.p, s->emap.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

int wn_solid_set_fixed(void* h, const uint8_t* fixed_mask) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_set_fixed: null handle");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_solid_set_fixed: not a C3D10 system");
  WN_CHECK(select_device(s));
  if (fixed_mask) {
    for (int64_t i = 0; i < s->n_nodes * 3; ++i) s->h_fixed[i] = fixed_mask[i] ? 1 : 0;
  } else {
    std::fill(s->h_fixed.begin(), s->h_fixed.end(), 0);
  }
  WN_CUDA(cudaMemcpy(s->fixed.p, s->h_fixed.data(), s->h_fixed.size(), cudaMemcpyHostToDevice));
  return 0;
}

int wn_assemble_c3d10_device(void* h, const double* d_props, int apply_bcs, uintptr_t stream) {
  WN_REQUIRE(h && (d_props || as_solid(h)->n_el == 0), WN_EINVAL, "wn_assemble_c3d10: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_assemble_c3d10_device: not a C3D10 system");
  WN_CHECK(select_device(s));
  cudaStream_t st = (cudaStream_t)stream;
  WN_CHECK(s->props.alloc(s->n_el * 2));
  if (s->n_el) WN_CUDA(cudaMemcpyAsync(s->props.p, d_props, s->props.bytes(), cudaMemcpyDeviceToDevice, st));
  WN_CHECK(s->k64.alloc(s->nnzb * 9));
  WN_CHECK(s->k32.alloc(s->nnzb * 9));
  WN_CUDA(cudaMemsetAsync(s->flags.p, 0, sizeof(int), st));
  if (s->asm_tiles > 0) {
    // tile-owner assembly: values and, when the packs exist with their structure, the packs'
    // values too, in one kernel with no element scratch
    const bool fused = s->stream_fine && s->fine.n_tiles == s->asm_tiles && s->fine.structure &&
                       s->fine.p64.p && s->fine.p32.p;
    AsmTileArgs A{s->asm_tile.p, s->asm_hdr.p, s->asm_el.p, s->asm_perm.p, s->gptr.p, s->asm_contrib.p,
                  s->block_row.p, s->col_idx.p,
                  fused ? reinterpret_cast<const int32_t*>(s->fine.d64.p) : nullptr,
                  fused ? reinterpret_cast<const int32_t*>(s->fine.d32.p) : nullptr,
                  fused ? s->fine.p64.p : nullptr, fused ? s->fine.p32.p : nullptr,
                  s->asm_chunks.p, s->asm_ne_max};
    WN_CHECK(launch_assemble_tiles(A, s->asm_tiles, s->asm_ne_max, s->asm_max_codes, s->nodes.p, s->conn.p,
                                   s->props.p, apply_bcs ? s->fixed.p : nullptr, s->nnzb, s->k64.p, s->k32.p,
                                   s->flags.p, st));
    if (fused)
      s->fine.packed = true;
    else if (s->stream_fine)  // first assembly: build the packs (structure and values) from the arrays
      WN_CHECK(s->fine.pack(s->row_ptr.p, s->col_idx.p, s->k32.p, s->k64.p, s->nnzb, st));
  } else {
    WN_CHECK(s->ke.alloc(s->n_el * 55 * 9));
    WN_CHECK(launch_ke_upper(s->n_el, s->n_nodes, s->nodes.p, s->conn.p, s->props.p, s->ke.p, s->flags.p, st));
    WN_CHECK(launch_gather_assemble(s->nnzb, s->gptr.p, s->gsrc.p, s->ke.p, s->block_row.p, s->col_idx.p,
                                    apply_bcs ? s->fixed.p : nullptr, s->k64.p, s->k32.p, st));
    // tile-major copies for the streamed fine-level kernels
    if (s->stream_fine) WN_CHECK(s->fine.pack(s->row_ptr.p, s->col_idx.p, s->k32.p, s->k64.p, s->nnzb, st));
  }
  ++s->values_version;
  int flag = 0;
  WN_CHECK(read_flag(s, st, &flag));
  WN_REQUIRE(flag == 0, WN_EMESH, "wn_assemble_c3d10: non-positive Jacobian determinant in a C3D10 element");
  s->assembled = true;
  s->bcs_applied = apply_bcs != 0;
  return 0;
}

int wn_assemble_c3d10(void* h, const double* props, int apply_bcs) {
  WN_REQUIRE(h && (props || as_solid(h)->n_el == 0), WN_EINVAL, "wn_assemble_c3d10: null argument");
  Solid* s = as_solid(h);
  WN_CHECK(select_device(s));
  DArray<double> d;
  WN_CHECK(d.upload(props, s->n_el * 2));
  return wn_assemble_c3d10_device(h, d.p, apply_bcs, 0);
}

int wn_solid_get_values(void* h, double* values) {
  WN_REQUIRE(h && values, WN_EINVAL, "wn_solid_get_values: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_solid_get_values: not a C3D10 system");
  WN_REQUIRE(s->assembled, WN_ESTATE, "wn_solid_get_values: not assembled");
  WN_CHECK(select_device(s));
  // device values are component-major (9 arrays of nnzb); return row-major blocks
  std::vector<double> soa(s->nnzb * 9);
  WN_CUDA(cudaMemcpy(soa.data(), s->k64.p, s->k64.bytes(), cudaMemcpyDeviceToHost));
  for (int64_t b = 0; b < s->nnzb; ++b)
    for (int k = 0; k < 9; ++k) values[b * 9 + k] = soa[k * s->nnzb + b];
  return 0;
}

int wn_solid_device_arrays(void* h, const double** k64, const float** k32, const int32_t** row_ptr,
                           const int32_t** col_idx, const uint8_t** fixed_mask) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_device_arrays: null handle");
  Solid* s = as_solid(h);
  if (k64) *k64 = s->k64.p;
  if (k32) *k32 = s->k32.p;
  if (row_ptr) *row_ptr = s->row_ptr.p;
  if (col_idx) *col_idx = s->col_idx.p;
  if (fixed_mask) *fixed_mask = s->fixed.p;
  return 0;
}

int wn_stream_tiles_host(int64_t n_rows, const int32_t* row_ptr, int32_t* tiles, int64_t capacity, int64_t* n_tiles) {
  WN_REQUIRE(row_ptr && n_tiles && n_rows >= 0, WN_EINVAL, "wn_stream_tiles_host: bad argument");
  std::vector<StreamTile> t;
  if (!build_stream_tiles(row_ptr, n_rows, t)) {
    *n_tiles = 0;
    return 0;
  }
  *n_tiles = (int64_t)t.size();
  if (tiles) {
    WN_REQUIRE(capacity >= (int64_t)t.size(), WN_EINVAL, "wn_stream_tiles_host: capacity %lld < %lld tiles",
               (long long)capacity, (long long)t.size());
    memcpy(tiles, t.data(), t.size() * sizeof(StreamTile));
  }
  return 0;
}

int wn_solid_set_stream(void* h, int enable) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_set_stream: null handle");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_solid_set_stream: not a C3D10 system");
  WN_CHECK(select_device(s));
  WN_CUDA(cudaDeviceSynchronize());
  WN_REQUIRE(enable >= 0 && enable <= 2, WN_EINVAL, "wn_solid_set_stream: enable %d not 0, 1 or 2", enable);
  s->stream_fine = enable != 0;
  s->stream_batched = enable == 2;
  // captured PCG chunks hold the launches (and pack pointers) of the current path: drop them
  // (the batched solver's on the epoch change)
  ++s->fine.epoch;
  if (s->work)
    for (auto& a : s->work->graphs)
      for (auto& g : a) g.reset();
  if (!s->stream_fine) {
    s->fine.clear();
    return 0;
  }
  if (s->fine.n_tiles == 0) WN_CHECK(s->fine.make_plan(s->h_row_ptr.data(), s->n_nodes, 3, 3));
  if (s->assembled && !s->fine.packed) {
    WN_CHECK(s->fine.pack(s->row_ptr.p, s->col_idx.p, s->k32.p, s->k64.p, s->nnzb, 0));
    WN_CUDA(cudaDeviceSynchronize());
  }
  return 0;
}

int wn_solid_set_batch_staging(void* h, int enable) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_set_batch_staging: null handle");
  Solid* s = as_solid(h);
  WN_CHECK(select_device(s));
  WN_CUDA(cudaDeviceSynchronize());
  s->batch_stage_x = enable != 0;
  ++s->fine.epoch;  // captured batched chunks hold the launches of the other path
  return 0;
}

int wn_solid_stream_status(void* h, int reset, int* status) {
  WN_REQUIRE(h && status, WN_EINVAL, "wn_solid_stream_status: null argument");
  Solid* s = as_solid(h);
  WN_CHECK(select_device(s));
  WN_CUDA(cudaDeviceSynchronize());
  WN_CUDA(cudaMemcpy(status, s->flags.p + kStreamStatusWord, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) WN_CUDA(cudaMemset(s->flags.p + kStreamStatusWord, 0, sizeof(int)));
  return 0;
}

int wn_solid_stream_test_hook(void* h, int64_t wait_limit_ns, int withhold_tile) {
  WN_REQUIRE(h, WN_EINVAL, "wn_solid_stream_test_hook: null handle");
  Solid* s = as_solid(h);
  WN_REQUIRE(wait_limit_ns >= 0, WN_EINVAL, "wn_solid_stream_test_hook: negative wait limit");
  WN_CHECK(select_device(s));
  WN_CUDA(cudaDeviceSynchronize());
  s->fine.ctl.wait_ns = wait_limit_ns > 0 ? (unsigned long long)wait_limit_ns : kStreamWaitLimitNs;
  s->fine.ctl.withhold = withhold_tile >= 0 ? withhold_tile : -1;
  // captured PCG chunks (single and batched) carry the old control values as kernel
  // parameters: drop them
  ++s->fine.epoch;
  if (s->work)
    for (auto& a : s->work->graphs)
      for (auto& g : a) g.reset();
  return 0;
}

int wn_spmv_solid_device(void* h, int precision, const void* x, void* y, uintptr_t stream) {
  WN_REQUIRE(h && x && y, WN_EINVAL, "wn_spmv_solid_device: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_spmv_solid_device: not a C3D10 system");
  WN_REQUIRE(s->assembled, WN_ESTATE, "wn_spmv_solid_device: not assembled");
  WN_CHECK(select_device(s));
  if (precision == 0 || precision == 1) {
    if (s->fine.packed) {
      const int rc = launch_solid_spmv_stream(precision, precision == 0 ? s->fine.d64.p : s->fine.d32.p,
                                              s->fine.n_tiles, precision == 0 ? s->fine.p64.p : s->fine.p32.p, x, y,
                                              s->flags.p + kStreamStatusWord, s->fine.ctl.wait_ns,
                                              s->fine.ctl.withhold, (cudaStream_t)stream);
      if (rc != 0) return rc < 0 ? rc : 0;
    }
  }
  if (precision == 0)
    return launch_solid_spmv_f64(s->n_nodes, s->row_ptr.p, s->col_idx.p, s->k64.p, s->nnzb, (const double*)x,
                                 (double*)y, (cudaStream_t)stream);
  if (precision == 1)
    return launch_solid_spmv_f32(s->n_nodes, s->row_ptr.p, s->col_idx.p, s->k32.p, s->nnzb, (const float*)x,
                                 (float*)y, (cudaStream_t)stream);
  set_error("wn_spmv_solid_device: precision must be 0 (FP64) or 1 (FP32)");
  return WN_EINVAL;
}

int wn_spmv_bsr_f64_device(int br, int bc, int64_t n_rows, const int32_t* row_ptr, const int32_t* col_idx,
                           const double* values, const double* x, double* y, double alpha, double beta,
                           uintptr_t stream) {
  WN_REQUIRE(n_rows >= 0 && (n_rows == 0 || (row_ptr && col_idx && values && x && y)), WN_EINVAL,
             "wn_spmv_bsr_f64_device: null argument");
  return launch_bsr_spmv_f64(br, bc, n_rows, row_ptr, col_idx, values, x, y, alpha, beta, (cudaStream_t)stream);
}

int wn_spmv_bsr_f32_device(int br, int bc, int64_t n_rows, const int32_t* row_ptr, const int32_t* col_idx,
                           const float* values, const float* x, float* y, float alpha, float beta, uintptr_t stream) {
  WN_REQUIRE(n_rows >= 0 && (n_rows == 0 || (row_ptr && col_idx && values && x && y)), WN_EINVAL,
             "wn_spmv_bsr_f32_device: null argument");
  return launch_bsr_spmv_f32(br, bc, n_rows, row_ptr, col_idx, values, x, y, alpha, beta, (cudaStream_t)stream);
}

int wn_spmv_bsr_f64(int br, int bc, int64_t n_rows, int64_t n_cols, int64_t nnzb, const int32_t* row_ptr,
                    const int32_t* col_idx, const double* values, const double* x, double* y, double alpha,
                    double beta) {
  WN_REQUIRE(row_ptr && col_idx && values && x && y, WN_EINVAL, "wn_spmv_bsr_f64: null argument");
  WN_REQUIRE(n_rows >= 0 && n_cols >= 0 && nnzb >= 0, WN_EINVAL, "wn_spmv_bsr_f64: negative size");
  WN_REQUIRE(row_ptr[n_rows] == nnzb, WN_EINVAL, "wn_spmv_bsr_f64: row_ptr[n_rows] != nnzb");
  for (int64_t k = 0; k < nnzb; ++k)
    WN_REQUIRE(col_idx[k] >= 0 && col_idx[k] < n_cols, WN_EINVAL, "wn_spmv_bsr_f64: column index out of range");
  DArray<int32_t> rp, ci;
  DArray<double> v, dx, dy;
  WN_CHECK(rp.upload(row_ptr, n_rows + 1));
  WN_CHECK(ci.upload(col_idx, nnzb));
  WN_CHECK(v.upload(values, nnzb * br * bc));
  WN_CHECK(dx.upload(x, n_cols * bc));
  WN_CHECK(dy.upload(y, n_rows * br));
  WN_CHECK(launch_bsr_spmv_f64(br, bc, n_rows, rp.p, ci.p, v.p, dx.p, dy.p, alpha, beta, 0));
  WN_CUDA(cudaMemcpy(y, dy.p, dy.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

int wn_c3d10_element_stresses(int64_t n_el, const double* coords, const double* props, const double* u_e,
                               double* gp_sig, double* gp_vm) {
  WN_REQUIRE(n_el >= 0 && (n_el == 0 || (coords && props && u_e && gp_sig && gp_vm)), WN_EINVAL,
             "wn_c3d10_element_stresses: null argument");
  if (n_el == 0) return 0;
  // each element gets its own 10 nodes: nodes = coords, conn[e][a] = 10 e + a, u = u_e
  std::vector<int32_t> conn(n_el * 10);
  for (int64_t k = 0; k < n_el * 10; ++k) conn[k] = (int32_t)k;
  DArray<double> dn, dp, du, ds, dv;
  DArray<int32_t> dc;
  WN_CHECK(dn.upload(coords, n_el * 30));
  WN_CHECK(dp.upload(props, n_el * 2));
  WN_CHECK(du.upload(u_e, n_el * 30));
  WN_CHECK(dc.upload(conn));
  WN_CHECK(ds.alloc(n_el * 24));
  WN_CHECK(dv.alloc(n_el * 4));
  WN_CHECK(launch_gp_stress(n_el, dn.p, dc.p, dp.p, du.p, ds.p, dv.p, 0));
  WN_CUDA(cudaMemcpy(gp_sig, ds.p, ds.bytes(), cudaMemcpyDeviceToHost));
  WN_CUDA(cudaMemcpy(gp_vm, dv.p, dv.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

int wn_c3d10_element_stiffness(int64_t n_el, const double* coords, const double* props, double* Ke) {
  WN_REQUIRE(n_el >= 0 && (n_el == 0 || (coords && props && Ke)), WN_EINVAL,
             "wn_c3d10_element_stiffness: null argument");
  if (n_el == 0) return 0;
  // each element gets its own 10 nodes: nodes = coords, conn[e][a] = 10 e + a
  std::vector<int32_t> conn(n_el * 10);
  for (int64_t k = 0; k < n_el * 10; ++k) conn[k] = (int32_t)k;
  DArray<double> dn, dp, dke;
  DArray<int32_t> dc;
  DArray<int> flags;
  WN_CHECK(dn.upload(coords, n_el * 30));
  WN_CHECK(dp.upload(props, n_el * 2));
  WN_CHECK(dc.upload(conn));
  WN_CHECK(dke.alloc(n_el * 55 * 9));
  WN_CHECK(flags.alloc(1));
  WN_CHECK(flags.zero());
  WN_CHECK(launch_ke_upper(n_el, n_el * 10, dn.p, dc.p, dp.p, dke.p, flags.p, 0));
  std::vector<double> up(n_el * 55 * 9);
  int flag = 0;
  WN_CUDA(cudaMemcpy(up.data(), dke.p, dke.bytes(), cudaMemcpyDeviceToHost));
  WN_CUDA(cudaMemcpy(&flag, flags.p, sizeof(int), cudaMemcpyDeviceToHost));
  WN_REQUIRE(flag == 0, WN_EMESH, "wn_c3d10_element_stiffness: non-positive Jacobian determinant");
  for (int64_t e = 0; e < n_el; ++e) {
    double* K = Ke + e * 900;
    for (int a = 0; a < 10; ++a)
      for (int b = a; b < 10; ++b) {
        const double* blk = up.data() + (e * 55 + tri_index(a, b)) * 9;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            K[(3 * a + i) * 30 + 3 * b + j] = blk[i * 3 + j];
            K[(3 * b + j) * 30 + 3 * a + i] = blk[i * 3 + j];
          }
      }
  }
  return 0;
}

int wn_c3d10_internal_forces(const double* nodes, const int32_t* solid_elements, const double* props, const double* U,
                             double* F_int, int n_solids, int n_nodes) {
  WN_REQUIRE(nodes && U && F_int && n_nodes > 0 && n_solids >= 0, WN_EINVAL,
             "wn_c3d10_internal_forces: bad argument");
  if (n_solids == 0) return 0;
  WN_REQUIRE(solid_elements && props, WN_EINVAL, "wn_c3d10_internal_forces: null argument");
  int dev = 0;
  WN_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(fint_workspace_mutex());
  FintWorkspace& w = fint_workspace(dev);
  const int64_t ne = n_solids, nn = n_nodes;
  WN_CHECK(w.grow(nn, ne));
  cudaStream_t st = 0;
  WN_CUDA(cudaMemcpyAsync(w.nodes.p, nodes, nn * 3 * sizeof(double), cudaMemcpyHostToDevice, st));
  WN_CUDA(cudaMemcpyAsync(w.conn.p, solid_elements, ne * 10 * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  WN_CUDA(cudaMemcpyAsync(w.props.p, props, ne * 2 * sizeof(double), cudaMemcpyHostToDevice, st));
  WN_CUDA(cudaMemcpyAsync(w.u.p, U, nn * 6 * sizeof(double), cudaMemcpyHostToDevice, st));
  WN_CUDA(cudaMemcpyAsync(w.f.p, F_int, nn * 6 * sizeof(double), cudaMemcpyHostToDevice, st));
  // node -> (element, local node) incidence on the device, in ascending e * 10 + a per node
  WN_CHECK(launch_build_incidence(nn, ne, w.conn.p, w.counts.p, w.inc_ptr.p, w.inc.p, w.scan.p, w.flags.p, st));
  int bad = 0;
  WN_CUDA(cudaMemcpyAsync(&bad, w.flags.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  WN_REQUIRE(bad == 0, WN_EMESH, "wn_c3d10_internal_forces: node index out of range");
  WN_CHECK(launch_element_force(ne, w.nodes.p, w.conn.p, w.props.p, w.u.p, 6, w.fe.p, nullptr, nullptr,
                                w.flags.p + 1, st));
  WN_CHECK(launch_node_gather(nn, w.inc_ptr.p, w.inc.p, w.fe.p, 6, 1, w.f.p, st));
  WN_CUDA(cudaMemcpyAsync(F_int, w.f.p, nn * 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
  WN_CUDA(cudaStreamSynchronize(st));
  return 0;
}

int wn_fint_c3d10_device(void* h, const double* d_u, double* d_fint, uintptr_t stream) {
  WN_REQUIRE(h && d_u && d_fint, WN_EINVAL, "wn_fint_c3d10_device: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_fint_c3d10_device: not a C3D10 system");
  WN_REQUIRE(s->props.n == s->n_el * 2, WN_ESTATE, "wn_fint_c3d10_device: no material properties (assemble first)");
  WN_CHECK(select_device(s));
  cudaStream_t st = (cudaStream_t)stream;
  WN_CHECK(s->fe.alloc(s->n_el * 30));
  WN_CHECK(launch_element_force(s->n_el, s->nodes.p, s->conn.p, s->props.p, d_u, 3, s->fe.p, nullptr, nullptr,
                                s->flags.p, st));
  WN_CHECK(launch_node_gather(s->n_nodes, s->inc_ptr.p, s->inc_ea.p, s->fe.p, 3, 0, d_fint, st));
  return 0;
}

int wn_fint_c3d10(void* h, const double* u, double* fint) {
  WN_REQUIRE(h && u && fint, WN_EINVAL, "wn_fint_c3d10: null argument");
  Solid* s = as_solid(h);
  WN_CHECK(select_device(s));
  DArray<double> du, df;
  WN_CHECK(du.upload(u, s->n_nodes * 3));
  WN_CHECK(df.alloc(s->n_nodes * 3));
  WN_CHECK(wn_fint_c3d10_device(h, du.p, df.p, 0));
  WN_CUDA(cudaMemcpy(fint, df.p, df.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

int wn_stress_c3d10_device(void* h, const double* d_u, double* d_cell_sig, double* d_cell_vm, double* d_nodal_vm,
                           uintptr_t stream) {
  WN_REQUIRE(h && d_u && d_cell_sig && d_cell_vm && d_nodal_vm, WN_EINVAL, "wn_stress_c3d10_device: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_stress_c3d10_device: not a C3D10 system");
  WN_REQUIRE(s->props.n == s->n_el * 2, WN_ESTATE, "wn_stress_c3d10_device: no material properties");
  WN_CHECK(select_device(s));
  return launch_stress(s->n_el, s->n_nodes, s->nodes.p, s->conn.p, s->props.p, d_u, s->inc_ptr.p, s->inc_ea.p,
                       d_cell_sig, d_cell_vm, d_nodal_vm, (cudaStream_t)stream);
}

int wn_stress_c3d10(void* h, const double* u, double* cell_sig, double* cell_vm, double* nodal_vm) {
  WN_REQUIRE(h && u && cell_sig && cell_vm && nodal_vm, WN_EINVAL, "wn_stress_c3d10: null argument");
  Solid* s = as_solid(h);
  WN_CHECK(select_device(s));
  DArray<double> du, dsig, dvm, dnv;
  WN_CHECK(du.upload(u, s->n_nodes * 3));
  WN_CHECK(dsig.alloc(s->n_el * 6));
  WN_CHECK(dvm.alloc(s->n_el));
  WN_CHECK(dnv.alloc(s->n_nodes));
  WN_CHECK(wn_stress_c3d10_device(h, du.p, dsig.p, dvm.p, dnv.p, 0));
  WN_CUDA(cudaMemcpy(cell_sig, dsig.p, dsig.bytes(), cudaMemcpyDeviceToHost));
  WN_CUDA(cudaMemcpy(cell_vm, dvm.p, dvm.bytes(), cudaMemcpyDeviceToHost));
  WN_CUDA(cudaMemcpy(nodal_vm, dnv.p, dnv.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

int wn_adjoint_compliance_device(void* h, const double* d_u, double* d_grad_E, double* d_grad_F, uintptr_t stream) {
  WN_REQUIRE(h && d_u, WN_EINVAL, "wn_adjoint_compliance_device: null argument");
  Solid* s = as_solid(h);
  WN_REQUIRE(s->bs == 3, WN_ESTATE, "wn_adjoint_compliance_device: not a C3D10 system");
  WN_REQUIRE(s->props.n == s->n_el * 2, WN_ESTATE, "wn_adjoint_compliance_device: no material properties");
  WN_CHECK(select_device(s));
  cudaStream_t st = (cudaStream_t)stream;
  if (d_grad_E)
    WN_CHECK(launch_element_force(s->n_el, s->nodes.p, s->conn.p, s->props.p, d_u, 3, nullptr, nullptr, d_grad_E,
                                  s->flags.p, st));
  if (d_grad_F) {
    const int64_t n = s->n_nodes * 3;
    grad_f_kernel<<<grid_for(n, 1, 256, 8), 256, 0, st>>>(n, d_u, s->bcs_applied ? s->fixed.p : nullptr, d_grad_F);
    WN_CUDA(cudaGetLastError());
  }
  return 0;
}

int wn_adjoint_compliance(void* h, const double* u, double* grad_E, double* grad_F) {
  WN_REQUIRE(h && u, WN_EINVAL, "wn_adjoint_compliance: null argument");
  Solid* s = as_solid(h);
  WN_CHECK(select_device(s));
  DArray<double> du, dge, dgf;
  WN_CHECK(du.upload(u, s->n_nodes * 3));
  if (grad_E) WN_CHECK(dge.alloc(s->n_el));
  if (grad_F) WN_CHECK(dgf.alloc(s->n_nodes * 3));
  WN_CHECK(wn_adjoint_compliance_device(h, du.p, dge.p, dgf.p, 0));
  if (grad_E) WN_CUDA(cudaMemcpy(grad_E, dge.p, dge.bytes(), cudaMemcpyDeviceToHost));
  if (grad_F) WN_CUDA(cudaMemcpy(grad_F, dgf.p, dgf.bytes(), cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"

namespace wn {
Solid::~Solid() {
  for (cudaEvent_t e : io_ev) cudaEventDestroy(e);
}
}
