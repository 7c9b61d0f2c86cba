// Error-free transformations for extra-precise residuals: Knuth's TwoSum (a + b = s + e
// exactly) and TwoProduct by fused multiply-add (a * b = p + e exactly), as used by Ogita,
// Rump and Oishi, "Accurate sum and dot product", SIAM J. Sci. Comput. 26 (2005).  The _rn
// intrinsics are never contracted or reordered by the compiler.
#pragma once

#include <cuda_runtime.h>

namespace wn {

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = __dmul_rn(a, b);
  e = __fma_rn(a, b, -p);
}

}  // namespace wn
