// Solver entry points used by the C ABI (solver.cu).
#pragma once

#include <cuda_runtime.h>

#include "amg.h"
#include "solid.h"
#include "wnfea_cuda.h"

namespace wn {

int solver_setup(Solid* s, const wn_amg_params& prm);
int solver_solve(Solid* s, const double* F, double* u, const wn_solve_params& prm, wn_solve_stats* stats,
                 cudaStream_t st);
int amg_vcycle(Solid* s, int precision, const void* r, void* z, cudaStream_t st);
int solver_profile(Solid* s, int capacity, int* n_rows, char* names, int64_t* counts, double* ms, double* bytes);
int solver_solve_multi(Solid* s, int n_rhs, const double* F, double* U, const wn_solve_params& prm,
                       wn_solve_stats* stats, int* case_iters, double* case_rel, cudaStream_t st);

}  // namespace wn
