// Fixed-popcount closed-form DP levels for Int64 inputs (Int128 states) and the mixed forms
// (FP32 multiplies, FP64 accumulation) of Float64 and ComplexF64.
#include "egg_dp_fixed.cuh"

namespace egg {
EGG_INSTANTIATE_FIXED(IntOp, int64_t, __int128, __int128)
EGG_INSTANTIATE_FIXED(MixedOp, float, float, double)
EGG_INSTANTIATE_FIXED(MixedOp, cf, cf, cd)
}  // namespace egg
