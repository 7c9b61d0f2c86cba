// Host-side launchers of the sm_100a kernels (internal; the public boundary is
// include/wnfea_cuda.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wn {

// c3d10.cu
// tile-owner assembly (assemble_tiles_kernel): device arrays of an AssemblyPlan (pattern.h) and,
// when the packs of the streamed fine matrix use the same tiles, their descriptors and buffers
// (p64 == nullptr: no packs written)
struct AsmTileArgs {
  const int32_t* tiles;      // n_tiles x 4: r0, r1, b0, b1
  // n_tiles x 8: first incident element, incident elements, first chunk, chunks; split blocks,
  // first contribution, contributions, 0 (one load per tile for every per-tile scalar)
  const int32_t* hdr;
  const int32_t* el;         // incident elements per tile
  const uint16_t* perm;      // nnzb
  const int32_t* gptr;       // nnzb + 1
  const uint16_t* contrib;   // n_el * 100
  const int32_t* block_row;  // nnzb
  const int32_t* col_idx;    // nnzb
  const int32_t* d64;        // pack descriptors (n_tiles x 4: r0, r1, seg, cntp) or null
  const int32_t* d32;
  unsigned char* p64;        // packs or null
  unsigned char* p32;
  const uint32_t* chunks;    // AssemblyPlan::chunks
  int ne_max;                // most incident elements of a tile (shared-memory layout)
};
// flags bit 0: det J <= 0.  Dynamic shared memory: ne_max elements of 127 doubles (at least
// the tile's 512 x 9 staged blocks); 32 chunk sums of 18 doubles, earlier the incident
// elements' connectivity (ne_max x 10 int32); max_codes 16-bit codes.
size_t assemble_tiles_smem(int ne_max, int max_codes);
constexpr size_t kAsmSmemLimit = 227 * 1024;  // dynamic shared memory of one CTA on sm_100
int launch_assemble_tiles(const AsmTileArgs& A, int n_tiles, int ne_max, int max_codes, const double* nodes,
                          const int32_t* conn, const double* props, const uint8_t* fixed, int64_t nnzb, double* k64,
                          float* k32, int* flags, cudaStream_t st);
// flags: bit 0 = det J <= 0, bit 1 = node index outside [0, n_nodes) (that element: zero Ke)
int launch_ke_upper(int64_t n_el, int64_t n_nodes, const double* nodes, const int32_t* conn, const double* props,
                    double* out, int* flags, cudaStream_t st);
int launch_gather_assemble(int64_t nnzb, const int32_t* gptr, const int32_t* gsrc, const double* ke,
                           const int32_t* block_row, const int32_t* col_idx, const uint8_t* fixed, double* k64,
                           float* k32, cudaStream_t st);
int launch_element_force(int64_t n_el, const double* nodes, const int32_t* conn, const double* props,
                         const double* u, int stride, double* fe_out, double* energy_out, double* grad_e,
                         int* flags, cudaStream_t st);
int launch_node_gather(int64_t n_nodes, const int64_t* inc_ptr, const int32_t* inc_ea, const double* fe, int stride,
                       int accumulate, double* out, cudaStream_t st);
// Node -> (element, local node) incidence of a C3D10 connectivity on the device: inc_ptr (nn + 1)
// and inc (10 ne entries e * 10 + a, ascending within each node).  counts: nn ints, scan:
// ceil(nn / 1024) + 1 int64 scratch; flags[0] is set when a node index is out of range.
int launch_build_incidence(int64_t nn, int64_t ne, const int32_t* conn, int32_t* counts, int64_t* inc_ptr,
                           int32_t* inc, int64_t* scan, int* flags, cudaStream_t st);
// Gauss-point stresses gp_sig (n_el x 4 x 6) and von Mises gp_vm (n_el x 4), u at 3 DOFs per node
int launch_gp_stress(int64_t n_el, const double* nodes, const int32_t* conn, const double* props, const double* u,
                     double* gp_sig, double* gp_vm, cudaStream_t st);
int launch_stress(int64_t n_el, int64_t n_nodes, const double* nodes, const int32_t* conn, const double* props,
                  const double* u, const int64_t* inc_ptr, const int32_t* inc_ea, double* cell_sig, double* cell_vm,
                  double* nodal_vm, cudaStream_t st);

// spmv.cu -- generic matrices are block-contiguous (AoS); the assembled fine-level matrix
// of a solid handle is component-major (SoA, stride nnzb)
int launch_bsr_spmv_f64(int br, int bc, int64_t n_rows, const int32_t* rp, const int32_t* ci, const double* v,
                        const double* x, double* y, double alpha, double beta, cudaStream_t st);
int launch_bsr_spmv_f32(int br, int bc, int64_t n_rows, const int32_t* rp, const int32_t* ci, const float* v,
                        const float* x, float* y, float alpha, float beta, cudaStream_t st);
int launch_solid_spmv_f64(int64_t n_rows, const int32_t* rp, const int32_t* ci, const double* v, int64_t nnzb,
                          const double* x, double* y, cudaStream_t st);
int launch_solid_spmv_f32(int64_t n_rows, const int32_t* rp, const int32_t* ci, const float* v, int64_t nnzb,
                          const float* x, float* y, cudaStream_t st);
// the same product with the matrix streamed through shared memory from its tile-major pack
// (stream.cuh); returns 1 when launched, 0 when the kernel cannot run here, < 0 on error; a
// pipeline wait that runs out of time (wait_ns; withhold >= 0: the failure-test hook of
// stream.cuh) writes WN_ETIMEOUT to *status
struct PackTile;
int launch_solid_spmv_stream(int precision, const PackTile* tiles, int n_tiles, const unsigned char* pack,
                             const void* x, void* y, int* status, unsigned long long wait_ns, int withhold,
                             cudaStream_t st);

// A linear 6-DOF-per-node system (block-contiguous row-major 6x6 values; host pattern arrays,
// values on the host or the device) as a solver handle with bs = 6 (capi.cu).
int make_bsr6_system(int64_t n, const int32_t* rp, const int32_t* ci, const double* values, bool values_on_device,
                     const double* coords, const uint8_t* fixed, void** out);

}  // namespace wn
