/*
 * libwnfea_cuda -- C ABI of the B200 (sm_100a) C3D10 / co-rotational-beam solve path.
 *
 * Conventions (as the reference's ctypes bridge, wnfea/solver/fast_kernels.py:96-222, and
 * its HIP C ABI, wnfea/solver/native/hip_kernels.cpp:1523-3164):
 *   - every function returns int: 0 = OK, < 0 = argument/state error (WN_E* below),
 *     > 0 = CUDA runtime error code; wn_last_error_string() describes the last failure
 *     of the calling thread;
 *   - opaque handles come from *_create and are released by *_destroy (cf. hip_amg_create
 *     / hip_amg_destroy, hip_kernels.cpp:1891, 2541);
 *   - plain entry points take HOST buffers and copy in and out (cf. hip_amg_solve_pcg,
 *     hip_kernels.cpp:2491); *_device entry points take DEVICE pointers and a cudaStream_t
 *     passed as uintptr_t (0 = legacy default stream) (cf. hip_amg_solve_pcg_device,
 *     hip_kernels.cpp:2384);
 *   - the library owns every device buffer inside a handle; caller buffers are borrowed
 *     for the duration of a call.  A handle is not thread-safe: one stream per handle.
 *   - sizes are int64_t, node / element indices int32_t, DOF layout node-major [ux,uy,uz].
 * No entry point falls back to a CPU path: without a usable GPU they return an error.
 */
#ifndef WNFEA_CUDA_H
#define WNFEA_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WN_OK 0
#define WN_EINVAL (-1)
#define WN_ESTATE (-2)
#define WN_EMESH (-3)
#define WN_EBREAKDOWN (-4)
#define WN_ENOCONV (-5)
#define WN_ENOTSPD (-6)
#define WN_EALLOC (-7)
#define WN_ETOOBIG (-8)
/* a bounded device-side wait (the streamed fine-matrix pipeline) ran out of time: the kernel
 * returned early and the results of the call are not valid */
#define WN_ETIMEOUT (-9)

/* ---------------------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------------------- */

/* Message of the calling thread's last failure ("" if none).  Replaces the reference's
 * bare integer codes (HIP_CHECK, hip_kernels.cpp:21-27). */
const char* wn_last_error_string(void);

/* Library version, e.g. 100 for 1.0.0. */
int wn_version(void);

/* ---------------------------------------------------------------------------------------
 * C3D10 system handle: mesh + 3x3-block pattern + element->block map.
 * Replaces the per-element COO template + scipy COO->CSR of assemble_c3d10_sparse_3dof
 * (wnfea/solver/solid_solver.py:50-84) with a pattern built once.
 * ------------------------------------------------------------------------------------- */

/* nodes: n_nodes x 3 FP64 (host); conn: n_el x 10 int32 (host), C3D10 node order 4 corners
 * + mid-edges 1-2, 2-3, 3-1, 1-4, 2-4, 3-4 (wnfea/elements/c3d10.py:52-58).
 * Builds the sorted BSR3 pattern (block (i,j) iff nodes i, j share an element), the
 * element->block map and the per-block gather lists, and uploads everything. */
int wn_solid_create(int64_t n_nodes, int64_t n_el, const double* nodes, const int32_t* conn, void** out_handle);
int wn_solid_destroy(void* h);
/* n_nodes, n_el, nnzb (number of 3x3 blocks) */
int wn_solid_info(void* h, int64_t* n_nodes, int64_t* n_el, int64_t* nnzb);
/* Host copies: row_ptr (n_nodes+1), col_idx (nnzb). */
int wn_solid_get_pattern(void* h, int32_t* row_ptr, int32_t* col_idx);
/* Host copy of the element->block map: map[e*100 + 10a + b] = index of block
 * (conn[e][a], conn[e][b]). */
int wn_solid_get_map(void* h, int32_t* emap);
/* Host-only pattern builder (no device work; usable without a GPU).  Call with
 * col_idx == NULL to get *nnzb (and row_ptr if non-NULL); call again with col_idx
 * (nnzb entries) and optionally emap (n_el*100) to fill them. */
int wn_bsr3_pattern_host(int64_t n_nodes, int64_t n_el, const int32_t* conn, int64_t* nnzb, int32_t* row_ptr,
                         int32_t* col_idx, int32_t* emap);
/* Host-only plan of the tile-owner assembly (no device work; for tests and inspection).  The
 * block rows are cut into the row tiles of the streamed fine matrix (WN_STREAM_TILE_BLOCKS /
 * _ROWS); per tile: its incident elements (ascending), and per block its contributions in the
 * assembly's summation order (element ascending) as slot << 8 | a << 4 | b (slot = index in the
 * tile's element list, (a, b) = element-local node pair), and the tile's blocks by descending
 * contribution count (perm[b0 + k] = local index).  Call with tiles == NULL to get the sizes;
 * *n_tiles = 0 when the mesh takes the element-scratch assembly instead (a tile with more than
 * 200 incident elements, or a row over the tile capacity).  Sizes: tiles 4 n_tiles, el_ptr
 * n_tiles + 1, el *n_el_entries, contrib 100 n_el, perm nnzb. */
int wn_assembly_plan_host(int64_t n_nodes, int64_t n_el, const int32_t* conn, int64_t* n_tiles, int* ne_max,
                          int64_t* n_el_entries, int32_t* tiles, int32_t* el_ptr, int32_t* el, uint16_t* contrib,
                          uint16_t* perm);
/* The work split of the tile-owner assembly (host; chunk_ptr n_tiles + 1, n_split n_tiles,
 * chunks n_chunks; NULL outputs skipped): blocks with more than *chunk_len contributions (the
 * first n_split[t] of tile t's order) are summed in chunks, chunks[k] = local block |
 * first contribution << 9 | length << 19 | first chunk of its block << 25; *max_codes is the
 * most contributions of one tile.  All zero when the mesh takes the element-scratch assembly. */
int wn_assembly_chunks_host(int64_t n_nodes, int64_t n_el, const int32_t* conn, int* chunk_len, int* max_codes,
                            int64_t* n_chunks, int32_t* chunk_ptr, uint32_t* chunks, int32_t* n_split);
/* Dirichlet mask over the 3*n_nodes DOFs (host, 1 = FIXED, NULL = none).  FIXED DOFs get
 * zero rows/columns and diagonal 1 and a zero load (solid_solver.py:95-127). */
int wn_solid_set_fixed(void* h, const uint8_t* fixed_mask);

/* Assemble K = sum_e Ke (c3d10.py:219-249, solid_solver.py:26-129) into the handle's BSR3
 * values (FP64, plus an FP32 copy for the mixed-precision solver), atomic-free through the
 * element->block map; apply_bcs != 0 applies the Dirichlet mask in the same pass.
 * props: n_el x 2 [E, nu] (host for wn_assemble_c3d10, device for the _device variant).
 * Returns WN_EMESH if an element has det J <= 0 (c3d10.py:129-134). */
int wn_assemble_c3d10(void* h, const double* props, int apply_bcs);
int wn_assemble_c3d10_device(void* h, const double* d_props, int apply_bcs, uintptr_t stream);
/* Host copy of the FP64 values: nnzb x 9 (row-major 3x3 blocks). */
int wn_solid_get_values(void* h, double* values);
/* Device pointers of the assembled values, pattern and Dirichlet mask (owned by h).  The
 * device values are component-major: entry (i, j) of block b at k64[(3 i + j) * nnzb + b]
 * (wn_solid_get_values returns row-major blocks). */
int wn_solid_device_arrays(void* h, const double** k64, const float** k32, const int32_t** row_ptr,
                           const int32_t** col_idx, const uint8_t** fixed_mask);

/* y = K x for the assembled matrix: precision 0 = FP64 values/accumulation, 1 = FP32
 * values/accumulation (x, y are float then).  Device pointers. */
int wn_spmv_solid_device(void* h, int precision, const void* x, void* y, uintptr_t stream);
/* Streamed fine-level kernels: enable 1 (the default) streams the fine level of single-case
 * solves from the tile-major packs, 2 also that of the batched (wn_solve_multi) solves, 0 turns
 * streaming off: it drops the tile plan and the FP32 / FP64 packs (about 1 GB per million DOFs)
 * and runs the fine level on the register row kernels; 1 or 2 rebuild them (and pack the
 * current values).  The batched solves default to the register kernels: with 32 cases per
 * block a row's cost is the gather of the x rows it touches, not the block values the packs
 * save.  Synchronises. */
int wn_solid_set_stream(void* h, int enable);
/* Batched solves (wn_solve_multi*): the FP32 fine-level passes with each row tile's x slice
 * (the 32 cases of the tile's column nodes) staged in shared memory (enable != 0), or the
 * register row kernels gathering x through L1/L2 (0, the default: on the 1M-DOF I-beam the
 * staged passes are slower, 312 vs 270 ms per 32-case batch).  The same arithmetic in the same
 * order: the row products are bitwise the same.  Synchronises. */
int wn_solid_set_batch_staging(void* h, int enable);
/* Status word of the streamed fine-matrix products of wn_spmv_solid_device: WN_OK, or
 * WN_ETIMEOUT when a bounded pipeline wait of a call since the last reset ran out of time (the
 * y of that call is not valid).  Synchronises the device; reset != 0 clears the word. */
int wn_solid_stream_status(void* h, int reset, int* status);
/* Failure-detection hook of the streamed fine-matrix kernels (for tests; no reference
 * counterpart).  wait_limit_ns bounds each pipeline wait (0 restores the default of 4 s).
 * withhold_tile >= 0 makes the producer skip that tile's copy, so the consumers' wait for it
 * runs out: the call reports WN_ETIMEOUT (wn_solid_stream_status for wn_spmv_solid_device,
 * stats.status for the solves) and every kernel still waits, bounded, for the copies it did
 * issue before it exits; -1 turns it off.  Synchronises; drops the handle's captured graphs. */
int wn_solid_stream_test_hook(void* h, int64_t wait_limit_ns, int withhold_tile);
/* The row tiles the streamed fine-matrix kernels cut a 3x3 block-row pattern into (host only):
 * tiles[4 t .. 4 t + 3] = (first row, end row, first block, end block) of tile t, whole rows
 * in order, at most WN_STREAM_TILE_BLOCKS blocks and WN_STREAM_TILE_ROWS rows per tile.
 * *n_tiles = 0 when a row alone exceeds the block capacity (those matrices use the register
 * row kernels).  tiles may be null to query the count. */
#define WN_STREAM_TILE_BLOCKS 512
#define WN_STREAM_TILE_ROWS 120
int wn_stream_tiles_host(int64_t n_rows, const int32_t* row_ptr, int32_t* tiles, int64_t capacity, int64_t* n_tiles);

/* ---------------------------------------------------------------------------------------
 * Smoothed-aggregation AMG + PCG solver (no reference counterpart for C3D10: the reference's
 * AMG, wnfea/solver/amg_preconditioner.py:147-661, aggregates 6-DOF beam nodes only).  The
 * near-null space is the 6 rigid-body modes; coarse levels carry 6 DOFs per aggregate.
 * ------------------------------------------------------------------------------------- */
typedef struct wn_amg_params {
  double strength_theta;   /* strong if |A_ij|_F >= theta sqrt(|A_ii|_F |A_jj|_F)      (0.08) */
  int max_levels;          /* including the coarsest                                   (10)   */
  int coarse_size;         /* stop coarsening at <= this many scalar DOFs               (1500) */
  int smoother_degree;     /* Chebyshev degree per pre-/post-smoothing                  (1)    */
  double cheb_lower;       /* lambda_min = cheb_lower * lambda_max                      (1/16) */
  double cheb_safety;      /* lambda_max = cheb_safety * rho(D^-1 A) estimate          (1.1)  */
  double prolong_omega;    /* P = (I - prolong_omega / rho * D^-1 A) P_tent             (4/3)  */
  int smooth_prolongator;  /* 1 = smoothed aggregation, 0 = plain (tentative) aggregation      */
  int power_iters;         /* power iterations for rho(D^-1 A)                          (15)   */
  double stream_min_mb;    /* level matrices / transfer operators of at least this many MB
                              in FP32 are streamed from tile-major packs, smaller ones stay
                              L2-resident on the register row kernels; < 0: none     (4)    */
  int setup_on_device;     /* 1: diagonal, power iterations, prolongator and Galerkin
                              products on the GPU (aggregation and the per-aggregate QR on
                              the host); 0: the whole setup on the host               (1)    */
  int coarse_block_smoother; /* 1: the 6-DOF levels (all but the finest) are smoothed with
                              6 x 6 block Jacobi in place of point Jacobi, by a change of
                              basis per aggregate made on the GPU after the build (the
                              exported levels are those of the new basis); 0: point
                              Jacobi on every level                                   (1)    */
} wn_amg_params;

/* Defaults above. */
int wn_amg_default_params(wn_amg_params* out);

/* Build the hierarchy of the assembled matrix of h (host setup in C++, FP64, then upload of
 * FP64 and FP32 copies).  params NULL = defaults.  Re-run after every re-assembly. */
int wn_amg_setup(void* h, const wn_amg_params* params);

/* One V-cycle z = M^-1 r at the finest level (precision 0: double r/z, 1: float r/z, 3: float
 * r/z through the FP16 fine level of solve precision 3).
 * Device pointers (the preconditioner apply of hip_amg_apply_vcycle_device,
 * hip_kernels.cpp:2080-2340). */
int wn_amg_vcycle_device(void* h, int precision, const void* d_r, void* d_z, uintptr_t stream);

/* Hierarchy shape: *n_levels counts the coarsest (dense) level; per level l < n_levels-1:
 * bs[l] DOFs per node, n_nodes[l], nnzb[l] blocks of A_l (arrays of 16, may be NULL). */
int wn_amg_info(void* h, int* n_levels, int* bs, int64_t* n_nodes, int64_t* nnzb, int64_t* n_coarse,
                double* setup_seconds);

/* Host copy of a hierarchy matrix: which = 0 (A_l, l >= 1), 1 (P_l), 2 (R_l = P_l^T).
 * Call with rp == NULL to get the sizes, then with buffers (rp: n_rows+1, ci: nnzb,
 * v: nnzb*br*bc). */
int wn_amg_level_matrix(void* h, int level, int which, int* br, int* bc, int64_t* n_rows, int64_t* n_cols,
                        int64_t* nnzb, int32_t* rp, int32_t* ci, double* v);
/* Level data: rho (spectral radius estimate of D^-1 A_l) and 1/diag(A_l) (n_nodes*bs). */
int wn_amg_level_data(void* h, int level, double* rho, double* dinv);
/* Coarsest level: dense A_c and A_c^-1 (n_coarse^2 each, row-major, may be NULL). */
int wn_amg_coarse(void* h, int64_t* n_coarse, double* Ac, double* Ac_inv);

/* Host-only setup (no GPU needed): same algorithm on a caller-supplied BSR3 matrix;
 * returns a host hierarchy handle usable with the three export calls above. */
int wn_amg_setup_host(int64_t n_nodes, const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                      const double* coords, const uint8_t* fixed_mask, const wn_amg_params* params, void** out);
int wn_amg_host_destroy(void* hier);
/* Exports of a host-only hierarchy (as wn_amg_level_matrix / _level_data / _coarse);
 * wn_amg_host_level_data with level == -1 returns the number of levels with a prolongator
 * in *n_nodes. */
int wn_amg_host_level_matrix(void* hier, int level, int which, int* br, int* bc, int64_t* n_rows, int64_t* n_cols,
                             int64_t* nnzb, int32_t* rp, int32_t* ci, double* v);
int wn_amg_host_level_data(void* hier, int level, double* rho, double* dinv, int64_t* n_nodes, int* bs);
int wn_amg_host_coarse(void* hier, int64_t* n_coarse, double* Ac, double* Ac_inv);

/* PCG solve of K u = F (solid_solver.py:197-308; GPU-resident like hip_amg_solve_pcg,
 * hip_kernels.cpp:2384-2517). */
typedef struct wn_solve_params {
  double rtol;        /* stop when ||F - K u|| <= rtol ||F||                          */
  int max_iter;       /* total PCG iterations (inner iterations for mixed)            */
  int precond;        /* 0 none, 1 point Jacobi (solid_solver.py:228-236), 2 AMG,
                         3 block Jacobi: pseudo-inverses of the diagonal node blocks
                         (solid_solver.py:237-258)                                    */
  int precision;      /* 0 FP64 throughout;
                         1 FP64 PCG (FP64 SpMV, x, r, q and dots; on the streamed fine level
                           the search directions p are rounded to FP32 once formed) with the
                           preconditioner in FP32 (AMG: FP32 V-cycle values, vectors and
                           accumulation, FP64 coarsest inverse), inside the FP64
                           true-residual loop;
                         2 FP32 PCG (FP32 SpMV and preconditioner, FP64 dots) inside FP64
                           iterative refinement (the scheme of solid_solver.py:271-300);
                         3 as 1, with the V-cycle's fine level on the equilibrated matrix
                           S K S, S = diag(K)^-1/2, stored in FP16 (FP32 arithmetic and
                           vectors; the FP16 preconditioner of the reference's TRI_PRECISION,
                           mixed_precision.py:96-103, used on every iteration).  AMG on a
                           C3D10 system with the streamed fine level only (else WN_EINVAL /
                           WN_ESTATE)                                                   */
  double inner_rtol;  /* mixed: inner relative tolerance (<= 0: max(1e-4, rtol))      */
  int max_outer;      /* mixed: refinement steps (<= 0: 10)                           */
  int chunk;          /* iterations per CUDA-graph replay / host convergence check    */
  int use_graph;      /* 1 = replay captured chunks as a CUDA graph                   */
  int profile;        /* 1 = time every kernel of this solve with CUDA events (graphs
                         off; read back with wn_solve_profile); 0 = normal          */
} wn_solve_params;

typedef struct wn_solve_stats {
  int iterations;        /* PCG iterations (sum of inner iterations for mixed)      */
  int outer_iterations;  /* refinement steps (0 for FP64)                            */
  int status;            /* 0 converged, WN_ENOCONV, WN_EBREAKDOWN                   */
  int n_levels;          /* AMG levels including the coarsest (0 without AMG)        */
  double rel_res;        /* final true ||F - K u|| / ||F|| (FP64 matrix) of the refined
                            solution, kept as a double-double pair; the FP64 u returned
                            is its rounding, whose own residual is at most about
                            max(rel_res, eps64 || |K| |u| || / ||F||)                */
  double solve_seconds;  /* device time of the solve (CUDA events)                   */
  double setup_seconds;  /* wall time of the last AMG setup                          */
  int64_t kernel_launches; /* kernels issued by the solve (graph replays counted per kernel) */
  double algorithmic_bytes; /* unique bytes read + written by the kernels that did their work
                               (matrices, vectors; single-RHS solves): divided by
                               solve_seconds, the solve's achieved memory bandwidth       */
} wn_solve_stats;

/* Device pointers F, u (3 n_nodes).  Returns 0 even when not converged: check
 * stats->status.  Builds the AMG hierarchy with defaults if precond == 2 and none exists. */
int wn_solve_device(void* h, const double* d_F, double* d_u, const wn_solve_params* params, wn_solve_stats* stats,
                    uintptr_t stream);
/* Host buffers F, u (copies in and out). */
int wn_solve(void* h, const double* F, double* u, const wn_solve_params* params, wn_solve_stats* stats);
/* Per kernel class of the last solve run with params.profile = 1 (e.g. "l0.pre_smooth" for the
 * fine-level first smoothing step, "pcg_spmv_dot", "coarse"): launches that did their work,
 * their summed CUDA-event durations (ms) and algorithmic bytes.  names: capacity x 48 chars
 * (NUL-terminated); *n_rows = number of classes (may exceed capacity). */
int wn_solve_profile(void* h, int capacity, int* n_rows, char* names, int64_t* counts, double* ms, double* bytes);

/* Linear 6-DOF-per-node systems (beam frames; the reference's GPU AMG-PCG of
 * BlockBeamAMGPreconditioner.solve_pcg -> hip_solve_pcg_amg, fast_kernels.py:598-663 and
 * hip_kernels.cpp:1746-2546): a solver handle with 6x6 blocks (row-major, block-contiguous)
 * that wn_amg_setup, wn_solve / wn_solve_device, wn_solid_info / _get_pattern and
 * wn_solid_destroy accept; the C3D10-only entry points return WN_ESTATE for it.  The AMG's
 * near-null space is the 6 rigid-body modes of 6-DOF nodes (translations; rotations w moving a
 * node by w x X and turning it by w), zero on fixed DOFs.  Columns sorted and unique per row,
 * a diagonal block in every row; fixed_mask (6 n_nodes, optional) marks Dirichlet DOFs whose
 * rows/columns the caller has already made identity. */
int wn_bsr6_system_create(int64_t n_nodes, const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                          const double* coords, const uint8_t* fixed_mask, void** out_handle);
/* The same from a beam handle's last assembled tangent (wn_beam_evaluate with
 * assemble_tangent = 1; apply_bcs = 1 for a constrained frame), values copied on the device. */
int wn_beam_linear_system(void* beam, void** out_handle);

/* Multi-right-hand-side solve (no reference counterpart: the reference solves load cases one
 * solve_c3d10_pcg call at a time, solid_solver.py:197-308).  F, U: row-major n x n_rhs
 * (n = 3 n_nodes, load case j in column j).  Cases are solved in batches of 32 sharing every
 * matrix read; each case keeps its own PCG recurrence and stops at its own
 * ||F_j - K U_j|| <= rtol ||F_j|| (FP64 true residual).  precision 0: FP64 V-cycle; 1: FP32
 * V-cycle inside the FP64 PCG.  stats: iterations = batched iterations summed over batches,
 * status = worst case, rel_res = largest case residual.  case_iters / case_rel_res: optional
 * host arrays of n_rhs entries. */
int wn_solve_multi_device(void* h, int n_rhs, const double* d_F, double* d_U, const wn_solve_params* params,
                          wn_solve_stats* stats, int* case_iters, double* case_rel_res, uintptr_t stream);
int wn_solve_multi(void* h, int n_rhs, const double* F, double* U, const wn_solve_params* params,
                   wn_solve_stats* stats, int* case_iters, double* case_rel_res);

/* ---------------------------------------------------------------------------------------
 * Generic block SpMV, y = alpha*A*x + beta*y (cf. hip_spmv_bsr6x6_fp32/_fp64,
 * hip_kernels.cpp:2975-3087, whose CPU reference is bsr6x6_spmv_cpu, bsr_matrix.py:155-193).
 * Block shapes (br x bc): 3x3, 6x6, 3x6, 6x3.  n_rows = number of block rows.
 * ------------------------------------------------------------------------------------- */
int wn_spmv_bsr_f64_device(int br, int bc, int64_t n_rows, const int32_t* row_ptr, const int32_t* col_idx,
                           const double* values, const double* x, double* y, double alpha, double beta,
                           uintptr_t stream);
int wn_spmv_bsr_f32_device(int br, int bc, int64_t n_rows, const int32_t* row_ptr, const int32_t* col_idx,
                           const float* values, const float* x, float* y, float alpha, float beta, uintptr_t stream);
/* Host-buffer variant (allocates, copies, launches, copies back, frees) -- the calling
 * convention of hip_spmv_bsr6x6_fp64 (hip_kernels.cpp:3032). n_cols = block columns. */
int wn_spmv_bsr_f64(int br, int bc, int64_t n_rows, int64_t n_cols, int64_t nnzb, const int32_t* row_ptr,
                    const int32_t* col_idx, const double* values, const double* x, double* y, double alpha,
                    double beta);

/* ---------------------------------------------------------------------------------------
 * Element-level kernels
 * ------------------------------------------------------------------------------------- */

/* Ke (n_el x 30 x 30, row-major, DOF order node-major) of elements given by coordinates
 * coords (n_el x 10 x 3) and props (n_el x 2) -- host buffers.  Batched form of
 * element_stiffness_c3d10 (c3d10.py:219-249).  WN_EMESH on det J <= 0. */
int wn_c3d10_element_stiffness(int64_t n_el, const double* coords, const double* props, double* Ke);
/* Gauss-point Cauchy stresses gp_sig (n_el x 4 x 6: sxx, syy, szz, sxy, syz, szx) and von Mises
 * gp_vm (n_el x 4) of elements given by coordinates coords (n_el x 10 x 3), props (n_el x 2)
 * and element displacements u_e (n_el x 30, node-major) -- host buffers.  Batched form of
 * element_stresses_c3d10 (c3d10.py:286-318). */
int wn_c3d10_element_stresses(int64_t n_el, const double* coords, const double* props, const double* u_e,
                              double* gp_sig, double* gp_vm);

/* Element stiffness for callers that must not allocate device memory (no counterpart in the
 * reference).  Code whose device memory belongs to another allocator -- a framework's caching
 * allocator, or a pool sized once at start-up -- cannot let a library call cudaMalloc behind
 * its back (the allocation can fail or fragment the pool), and latency-bound loops cannot
 * absorb the device-wide synchronisation of cudaFree.  wn_c3d10_element_stiffness allocates
 * on every call; this variant takes device pointers from the caller -- nodes (n_nodes x 3),
 * conn (n_el x 10), props (n_el x 2), Ke out (n_el x 30 x 30) -- and keeps its scratch (the
 * upper-triangle blocks of each element plus a status word) in a fixed device array that
 * every GPU loading the library holds until exit (about 8.1 MB).  It calls no cudaMalloc,
 * cudaFree or allocating library routine.
 *   - n_el > WN_NOALLOC_MAX_ELEMENTS returns WN_ETOOBIG (split the batch);
 *   - a conn entry outside [0, n_nodes) returns WN_EINVAL: the kernel checks every index
 *     before it reads coordinates, and that element's Ke is zero;
 *   - the first call on a device looks up the scratch address (cudaGetSymbolAddress, with
 *     that device current): make that first call before any stream capture;
 *   - all calls share the scratch, so calls that overlap on the GPU (other streams, other
 *     threads) race: serialise them;
 *   - the call synchronises `stream` to report WN_EMESH for det J <= 0. */
#define WN_NOALLOC_MAX_ELEMENTS 2048
int wn_c3d10_element_stiffness_noalloc(int64_t n_el, int64_t n_nodes, const double* d_nodes, const int32_t* d_conn,
                                       const double* d_props, double* d_Ke, uintptr_t stream);

/* Internal forces F_int = sum_e f_e(u) with f_e = sum_g w|J| B^T C B u_e (c3d10.py:252-283),
 * atomic-free (node gather in element order).  Same argument list and U/F_int stride of 6
 * as the reference's compute_c3d10_internal_forces_native (kernels.cpp:244-252); host
 * buffers; F_int is accumulated into (the reference's += scatter).  The node incidence is
 * built on the GPU each call; the device buffers are a per-device workspace kept between
 * calls (grown when a larger mesh arrives, held until exit), and calls are serialised. */
int wn_c3d10_internal_forces(const double* nodes, const int32_t* solid_elements, const double* props, const double* U,
                             double* F_int, int n_solids, int n_nodes);
/* Handle variant on device pointers: f_int (3 n_nodes, overwritten) from u (3 n_nodes). */
int wn_fint_c3d10_device(void* h, const double* d_u, double* d_fint, uintptr_t stream);

/* Host-buffer variant of wn_fint_c3d10_device. */
int wn_fint_c3d10(void* h, const double* u, double* fint);

/* Stresses (compute_c3d10_stress_field, solid_solver.py:311-365): cell_sig n_el x 6
 * [sxx,syy,szz,sxy,syz,szx] (mean of the 4 Gauss points), cell_vm n_el, nodal_vm n_nodes
 * (unweighted mean over incident elements).  Uses the props of the last assembly. */
int wn_stress_c3d10(void* h, const double* u, double* cell_sig, double* cell_vm, double* nodal_vm);
int wn_stress_c3d10_device(void* h, const double* d_u, double* d_cell_sig, double* d_cell_vm, double* d_nodal_vm,
                           uintptr_t stream);

/* Compliance adjoint (no reference counterpart): for C = F^T u with K(E) u = F,
 * grad_E[e] = dC/dE_e = -u_e^T Ke u_e / E_e (self-adjoint: reuses u, no extra solve) and
 * grad_F = dC/dF = 2u on free DOFs, 0 on FIXED DOFs.  Either output may be NULL. */
int wn_adjoint_compliance_device(void* h, const double* d_u, double* d_grad_E, double* d_grad_F, uintptr_t stream);
int wn_adjoint_compliance(void* h, const double* u, double* grad_E, double* grad_F);

/* ---------------------------------------------------------------------------------------
 * Co-rotational 3D beam frames (6 DOFs per node [ux, uy, uz, rx, ry, rz]).
 * Element data as prepare_batch_data builds it (wnfea/solver/fast_kernels.py:263-306):
 * elements n_el x 2, props n_el x 6 [E, G, A, Iy, Iz, J], e_ref n_el x 9 (reference triad
 * rows e1, e2, e3), L0 n_el.
 * ------------------------------------------------------------------------------------- */

/* F_int += f_int(U) -- same argument list as the reference's
 * compute_beam_internal_forces_native (wnfea/solver/native/kernels.cpp:19-29); host
 * buffers, computed on the GPU with an atomic-free node gather. */
int wn_beam_internal_forces(const double* nodes, const int32_t* elements, const double* props, const double* e_ref,
                            const double* L0_arr, const double* U, double* F_int, int n_elements, int n_nodes);

/* Frame handle: element data on the device plus the 6x6-block pattern of the tangent (block
 * (i, j) iff i == j or a beam joins i and j) and its gather lists. */
int wn_beam_create(int64_t n_nodes, int64_t n_el, const double* nodes, const int32_t* elements, const double* props,
                   const double* e_ref, const double* L0, void** out);
int wn_beam_destroy(void* h);
int wn_beam_info(void* h, int64_t* n_nodes, int64_t* n_el, int64_t* nnzb);
int wn_beam_get_pattern(void* h, int32_t* row_ptr, int32_t* col_idx);
/* Dirichlet mask over the 6 n DOFs (1 = constrained; NULL clears). */
int wn_beam_set_fixed(void* h, const uint8_t* fixed_mask);
/* f_int(U) into fint (6 n, overwritten; NULL to skip) and, if assemble_tangent, the
 * consistent tangent K_t = d f_int / d U (exact derivative of the force code, not a finite
 * difference; cf. the JFNK operator, wnfea/solver/jfnk_operator.py:98-134) into the
 * handle's BSR6 values; apply_bcs != 0 turns constrained rows/columns into identity. */
int wn_beam_evaluate_device(void* h, const double* d_U, double* d_fint, int assemble_tangent, int apply_bcs,
                            uintptr_t stream);
int wn_beam_evaluate(void* h, const double* U, double* fint, int assemble_tangent, int apply_bcs);
/* Host copy of the tangent values: nnzb x 36, row-major 6x6 blocks. */
int wn_beam_get_tangent(void* h, double* values);
/* Solve K_t x = b (K_t is not symmetric away from U = 0).  method 1: dense blocked LU with
 * partial pivoting (frames up to WN_BEAM_DENSE_MAX DOFs); 2: BiCGStab preconditioned by
 * the inverse 6x6 diagonal blocks (rtol, max_iter); 0: dense when it fits, else BiCGStab.
 * Returns WN_ENOCONV / WN_EBREAKDOWN (singular) as status; rel_res = ||b - K x|| / ||b||. */
#define WN_BEAM_DENSE_MAX 3072
int wn_beam_solve_device(void* h, const double* d_b, double* d_x, int method, double rtol, int max_iter, int* iters,
                         double* rel_res, uintptr_t stream);
int wn_beam_solve(void* h, const double* rhs, double* x, int method, double rtol, int max_iter, int* iters,
                  double* rel_res);

/* Block until all work of the calling thread's device is done. */
int wn_device_synchronize(void);

#ifdef __cplusplus
}
#endif

#endif /* WNFEA_CUDA_H */
