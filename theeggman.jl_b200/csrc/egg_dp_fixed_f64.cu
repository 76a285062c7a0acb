// Fixed-popcount closed-form DP levels for Float64 (EGG_PREC_EXACT and EGG_PREC_FMA).
#include "egg_dp_fixed.cuh"

namespace egg {
EGG_INSTANTIATE_FIXED(ExactOp, double, double, double)
EGG_INSTANTIATE_FIXED(FmaOp, double, double, double)
}  // namespace egg
