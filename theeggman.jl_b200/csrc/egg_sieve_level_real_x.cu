// egg_sieve_level_real_x.cu -- popcount-level sieve kernels for Float64 terms, m = 2 .. 32, in the
// reference's arithmetic (each term bit-identical to _glynn_term!, src/hafnian.jl:528-602).
#include "egg_sieve_level_real.cuh"

namespace egg {

template int level_launch_real_lo<true>(const SieveArgs &, const int64_t *, int, int, bool, dd *, int, cudaStream_t);
template int level_launch_all_real_lo<true>(const SieveArgs &, int, bool, dd *, int, cudaStream_t);
template int level_shape_real_lo<true>(int, int, bool, bool, int *, int *);

}  // namespace egg
