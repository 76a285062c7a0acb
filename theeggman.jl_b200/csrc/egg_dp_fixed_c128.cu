// Fixed-popcount closed-form DP levels for ComplexF64 (EGG_PREC_EXACT and EGG_PREC_FMA).
#include "egg_dp_fixed.cuh"

namespace egg {
EGG_INSTANTIATE_FIXED(ExactOp, cd, cd, cd)
EGG_INSTANTIATE_FIXED(FmaOp, cd, cd, cd)
}  // namespace egg
