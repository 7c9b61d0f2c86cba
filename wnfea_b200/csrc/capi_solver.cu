// extern "C" boundary of the AMG setup and the PCG / mixed-precision solver.
#include <algorithm>
#include <cstring>
#include <thread>

#include "amg.h"
#include "amg_device.h"
#include "common.cuh"
#include "solid.h"
#include "solver.h"
#include "wnfea_cuda.h"

using namespace wn;

namespace {

struct HostAmgHandle {
  HostHierarchy h;
};

// a hierarchy handle may be a Solid (device + host copy) or a host-only handle; the caller
// says which by the entry point used.  Solid handles carry the hierarchy in s->amg->host.
HostHierarchy* host_of_solid(void* h) {
  Solid* s = reinterpret_cast<Solid*>(h);
  if (!s->amg) return nullptr;
  if (amg_sync_host(*s->amg) != 0) return nullptr;  // device-built levels: copies made on demand
  return &s->amg->host;
}

int export_matrix(HostHierarchy* H, int level, int which, int* br, int* bc, int64_t* n_rows, int64_t* n_cols,
                  int64_t* nnzb, int32_t* rp, int32_t* ci, double* v) {
  WN_REQUIRE(H, WN_ESTATE, "wn_amg_level_matrix: no hierarchy");
  WN_REQUIRE(level >= 0 && level < (int)H->levels.size(), WN_EINVAL, "wn_amg_level_matrix: level out of range");
  WN_REQUIRE(which >= 0 && which <= 2, WN_EINVAL, "wn_amg_level_matrix: which in {0,1,2}");
  WN_REQUIRE(!(which == 0 && level == 0), WN_EINVAL, "wn_amg_level_matrix: A_0 is the assembled matrix");
  const HostLevel& L = H->levels[level];
  const HostBsr& M = which == 0 ? L.A : (which == 1 ? L.P : L.R);
  if (br) *br = M.br;
  if (bc) *bc = M.bc;
  if (n_rows) *n_rows = M.n_rows;
  if (n_cols) *n_cols = M.n_cols;
  if (nnzb) *nnzb = M.nnzb();
  if (rp) memcpy(rp, M.rp.data(), sizeof(int32_t) * M.rp.size());
  if (ci) memcpy(ci, M.ci.data(), sizeof(int32_t) * M.ci.size());
  if (v) memcpy(v, M.v.data(), sizeof(double) * M.v.size());
  return 0;
}

}  // namespace

extern "C" {

int wn_amg_default_params(wn_amg_params* out) {
  WN_REQUIRE(out, WN_EINVAL, "wn_amg_default_params: null argument");
  *out = amg_default_params();
  return 0;
}

int wn_amg_setup(void* h, const wn_amg_params* params) {
  WN_REQUIRE(h, WN_EINVAL, "wn_amg_setup: null handle");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_CUDA(cudaSetDevice(s->device));
  return solver_setup(s, params ? *params : amg_default_params());
}

int wn_amg_vcycle_device(void* h, int precision, const void* d_r, void* d_z, uintptr_t stream) {
  WN_REQUIRE(h && d_r && d_z && (precision == 0 || precision == 1 || precision == 3), WN_EINVAL,
             "wn_amg_vcycle_device: bad argument");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_CUDA(cudaSetDevice(s->device));
  return amg_vcycle(s, precision, d_r, d_z, (cudaStream_t)stream);
}

int wn_amg_info(void* h, int* n_levels, int* bs, int64_t* n_nodes, int64_t* nnzb, int64_t* n_coarse,
                double* setup_seconds) {
  WN_REQUIRE(h, WN_EINVAL, "wn_amg_info: null handle");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_REQUIRE(s->amg, WN_ESTATE, "wn_amg_info: no hierarchy");
  const HostHierarchy& H = s->amg->host;
  const int L = (int)H.levels.size();
  if (n_levels) *n_levels = L + 1;
  for (int l = 0; l < L && l < 16; ++l) {
    if (bs) bs[l] = H.levels[l].bs;
    if (n_nodes) n_nodes[l] = H.levels[l].n_nodes;
    if (nnzb) nnzb[l] = l == 0 ? s->nnzb : s->amg->levels[l].A.nnzb;
  }
  if (n_coarse) *n_coarse = H.n_coarse;
  if (setup_seconds) *setup_seconds = s->amg->setup_seconds;
  return 0;
}

int wn_amg_level_matrix(void* h, int level, int which, int* br, int* bc, int64_t* n_rows, int64_t* n_cols,
                        int64_t* nnzb, int32_t* rp, int32_t* ci, double* v) {
  WN_REQUIRE(h, WN_EINVAL, "wn_amg_level_matrix: null handle");
  HostHierarchy* H = reinterpret_cast<Solid*>(h)->amg ? host_of_solid(h) : nullptr;
  return export_matrix(H, level, which, br, bc, n_rows, n_cols, nnzb, rp, ci, v);
}

int wn_amg_level_data(void* h, int level, double* rho, double* dinv) {
  WN_REQUIRE(h, WN_EINVAL, "wn_amg_level_data: null handle");
  HostHierarchy* H = host_of_solid(h);
  WN_REQUIRE(H && level >= 0 && level < (int)H->levels.size(), WN_EINVAL, "wn_amg_level_data: bad level");
  const HostLevel& L = H->levels[level];
  if (rho) *rho = L.rho;
  if (dinv) memcpy(dinv, L.dinv.data(), sizeof(double) * L.dinv.size());
  return 0;
}

int wn_amg_coarse(void* h, int64_t* n_coarse, double* Ac, double* Ac_inv) {
  WN_REQUIRE(h, WN_EINVAL, "wn_amg_coarse: null handle");
  HostHierarchy* H = host_of_solid(h);
  WN_REQUIRE(H, WN_ESTATE, "wn_amg_coarse: no hierarchy");
  if (n_coarse) *n_coarse = H->n_coarse;
  if (Ac) memcpy(Ac, H->coarse_A.data(), sizeof(double) * H->coarse_A.size());
  if (Ac_inv) memcpy(Ac_inv, H->coarse_inv.data(), sizeof(double) * H->coarse_inv.size());
  return 0;
}

int wn_amg_setup_host(int64_t n_nodes, const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                      const double* coords, const uint8_t* fixed_mask, const wn_amg_params* params, void** out) {
  WN_REQUIRE(out && row_ptr && col_idx && values && coords && n_nodes > 0, WN_EINVAL,
             "wn_amg_setup_host: bad argument");
  auto* hh = new HostAmgHandle();
  int rc = amg_build(params ? *params : amg_default_params(), n_nodes, 3, row_ptr, col_idx, values, coords, fixed_mask,
                     hh->h);
  if (rc != 0) {
    delete hh;
    return rc;
  }
  *out = hh;
  return 0;
}

int wn_amg_host_destroy(void* hier) {
  delete reinterpret_cast<HostAmgHandle*>(hier);
  return 0;
}

int wn_amg_host_level_matrix(void* hier, int level, int which, int* br, int* bc, int64_t* n_rows, int64_t* n_cols,
                             int64_t* nnzb, int32_t* rp, int32_t* ci, double* v) {
  WN_REQUIRE(hier, WN_EINVAL, "wn_amg_host_level_matrix: null handle");
  return export_matrix(&reinterpret_cast<HostAmgHandle*>(hier)->h, level, which, br, bc, n_rows, n_cols, nnzb, rp,
                       ci, v);
}

int wn_amg_host_level_data(void* hier, int level, double* rho, double* dinv, int64_t* n_nodes, int* bs) {
  WN_REQUIRE(hier, WN_EINVAL, "wn_amg_host_level_data: null handle");
  HostHierarchy& H = reinterpret_cast<HostAmgHandle*>(hier)->h;
  if (level == -1) {  // number of levels with P (coarsest excluded)
    if (n_nodes) *n_nodes = (int64_t)H.levels.size();
    return 0;
  }
  WN_REQUIRE(level >= 0 && level < (int)H.levels.size(), WN_EINVAL, "wn_amg_host_level_data: bad level");
  const HostLevel& L = H.levels[level];
  if (rho) *rho = L.rho;
  if (dinv) memcpy(dinv, L.dinv.data(), sizeof(double) * L.dinv.size());
  if (n_nodes) *n_nodes = L.n_nodes;
  if (bs) *bs = L.bs;
  return 0;
}

int wn_amg_host_coarse(void* hier, int64_t* n_coarse, double* Ac, double* Ac_inv) {
  WN_REQUIRE(hier, WN_EINVAL, "wn_amg_host_coarse: null handle");
  HostHierarchy& H = reinterpret_cast<HostAmgHandle*>(hier)->h;
  if (n_coarse) *n_coarse = H.n_coarse;
  if (Ac) memcpy(Ac, H.coarse_A.data(), sizeof(double) * H.coarse_A.size());
  if (Ac_inv) memcpy(Ac_inv, H.coarse_inv.data(), sizeof(double) * H.coarse_inv.size());
  return 0;
}

int wn_solve_device(void* h, const double* d_F, double* d_u, const wn_solve_params* params, wn_solve_stats* stats,
                    uintptr_t stream) {
  WN_REQUIRE(h && d_F && d_u && params, WN_EINVAL, "wn_solve_device: null argument");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_CUDA(cudaSetDevice(s->device));
  return solver_solve(s, d_F, d_u, *params, stats, (cudaStream_t)stream);
}

int wn_solve(void* h, const double* F, double* u, const wn_solve_params* params, wn_solve_stats* stats) {
  WN_REQUIRE(h && F && u && params, WN_EINVAL, "wn_solve: null argument");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_CUDA(cudaSetDevice(s->device));
  const int64_t n = s->n_nodes * s->bs;
  // staged through page-locked memory: a device copy from / into pageable memory (a freshly
  // allocated result array in particular) runs at a fraction of the link's speed.  The copies
  // go in chunks so that each host copy overlaps the DMA of its neighbour: F chunk k + 1 is
  // copied into the staging buffer while chunk k uploads, u chunk k is copied out while chunk
  // k + 1 downloads (on the legacy stream, which the solve's stream is ordered with).
  constexpr int64_t kChunk = 1 << 17;  // doubles (1 MB)
  const int nch = (int)((n + kChunk - 1) / kChunk);
  WN_CHECK(s->io_f.alloc(n));
  WN_CHECK(s->io_u.alloc(n));
  WN_CHECK(s->io_pin.at_least(2 * n));
  while ((int)s->io_ev.size() < nch) {
    cudaEvent_t e = nullptr;
    WN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    s->io_ev.push_back(e);
  }
  for (int c = 0; c < nch; ++c) {
    const int64_t a = c * kChunk, len = std::min(kChunk, n - a);
    std::memcpy(s->io_pin.p + a, F + a, len * sizeof(double));
    WN_CUDA(cudaMemcpyAsync(s->io_f.p + a, s->io_pin.p + a, len * sizeof(double), cudaMemcpyHostToDevice, 0));
  }
  // while the GPU solves, a helper thread touches every page of u (F is staged already, so u may
  // alias it): a freshly allocated result array otherwise takes its page faults in the final copy
  struct Toucher {
    std::thread t;
    ~Toucher() {
      if (t.joinable()) t.join();
    }
  } touch;
  touch.t = std::thread([u, n]() {
    volatile double* v = u;
    for (int64_t i = 0; i < n; i += 512) v[i] = 0.0;
    if (n > 0) v[n - 1] = 0.0;
  });
  WN_CHECK(solver_solve(s, s->io_f.p, s->io_u.p, *params, stats, 0));
  touch.t.join();
  for (int c = 0; c < nch; ++c) {
    const int64_t a = c * kChunk, len = std::min(kChunk, n - a);
    WN_CUDA(cudaMemcpyAsync(s->io_pin.p + n + a, s->io_u.p + a, len * sizeof(double), cudaMemcpyDeviceToHost, 0));
    WN_CUDA(cudaEventRecord(s->io_ev[c], 0));
  }
  for (int c = 0; c < nch; ++c) {
    const int64_t a = c * kChunk, len = std::min(kChunk, n - a);
    WN_CUDA(cudaEventSynchronize(s->io_ev[c]));
    std::memcpy(u + a, s->io_pin.p + n + a, len * sizeof(double));
  }
  return 0;
}

int wn_solve_profile(void* h, int capacity, int* n_rows, char* names, int64_t* counts, double* ms, double* bytes) {
  WN_REQUIRE(h && n_rows && capacity >= 0, WN_EINVAL, "wn_solve_profile: bad argument");
  return solver_profile(reinterpret_cast<Solid*>(h), capacity, n_rows, names, counts, ms, bytes);
}

int wn_solve_multi_device(void* h, int n_rhs, const double* d_F, double* d_U, const wn_solve_params* params,
                          wn_solve_stats* stats, int* case_iters, double* case_rel_res, uintptr_t stream) {
  WN_REQUIRE(h && params && n_rhs >= 0 && (n_rhs == 0 || (d_F && d_U)), WN_EINVAL,
             "wn_solve_multi_device: bad argument");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_CUDA(cudaSetDevice(s->device));
  return solver_solve_multi(s, n_rhs, d_F, d_U, *params, stats, case_iters, case_rel_res, (cudaStream_t)stream);
}

int wn_solve_multi(void* h, int n_rhs, const double* F, double* U, const wn_solve_params* params,
                   wn_solve_stats* stats, int* case_iters, double* case_rel_res) {
  WN_REQUIRE(h && params && n_rhs >= 0 && (n_rhs == 0 || (F && U)), WN_EINVAL, "wn_solve_multi: bad argument");
  Solid* s = reinterpret_cast<Solid*>(h);
  WN_CUDA(cudaSetDevice(s->device));
  const int64_t n = s->n_nodes * 3 * (int64_t)n_rhs;
  DArray<double> dF, dU;
  WN_CHECK(dF.upload(F, n));
  WN_CHECK(dU.alloc(n));
  WN_CHECK(solver_solve_multi(s, n_rhs, dF.p, dU.p, *params, stats, case_iters, case_rel_res, 0));
  if (n) WN_CUDA(cudaMemcpy(U, dU.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"
