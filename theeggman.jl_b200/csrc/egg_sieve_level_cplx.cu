// egg_sieve_level_cplx.cu -- popcount-level sieve kernels for ComplexF64 terms, m = 2 .. 32, with
// fused multiply-adds, and the dispatch over the complex levels (the reference-arithmetic form is
// in egg_sieve_level_cplx_x.cu).
#include "egg_sieve_level_cplx.cuh"

namespace egg {

template int level_launch_cplx_lo<false>(const SieveArgs &, const int64_t *, int, int, bool, dd *, int, cudaStream_t);
template int level_launch_all_cplx_lo<false>(const SieveArgs &, int, bool, dd *, int, cudaStream_t);
template int level_shape_cplx_lo<false>(int, int, bool, bool, int *, int *);
extern template int level_launch_cplx_lo<true>(const SieveArgs &, const int64_t *, int, int, bool, dd *, int, cudaStream_t);
extern template int level_launch_all_cplx_lo<true>(const SieveArgs &, int, bool, dd *, int, cudaStream_t);
extern template int level_shape_cplx_lo<true>(int, int, bool, bool, int *, int *);

int level_launch_cplx(const SieveArgs &a, const int64_t *strides, int B, int k, bool narrow, bool exact, dd *partial,
                      int blocks_x, cudaStream_t st)
{
    return exact ? level_launch_cplx_lo<true>(a, strides, B, k, narrow, partial, blocks_x, st)
                 : level_launch_cplx_lo<false>(a, strides, B, k, narrow, partial, blocks_x, st);
}

int level_launch_all_cplx(const SieveArgs &a, int k, bool narrow, bool exact, dd *partial, int blocks_x, cudaStream_t st)
{
    return exact ? level_launch_all_cplx_lo<true>(a, k, narrow, partial, blocks_x, st)
                 : level_launch_all_cplx_lo<false>(a, k, narrow, partial, blocks_x, st);
}

int level_shape_cplx(int nmax, int k, bool narrow, bool exact, bool all, int *warps_per_block, int *blocks_per_sm)
{
    return exact ? level_shape_cplx_lo<true>(nmax, k, narrow, all, warps_per_block, blocks_per_sm)
                 : level_shape_cplx_lo<false>(nmax, k, narrow, all, warps_per_block, blocks_per_sm);
}

}  // namespace egg
