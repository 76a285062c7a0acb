// egg_sieve_level_real.cu -- popcount-level sieve kernels for Float64 terms, m = 2 .. 32, with fused
// multiply-adds, and the dispatch over every real level (levels 17-24 are in
// egg_sieve_level_real_hi.cu, the reference-arithmetic form in egg_sieve_level_real_x.cu).
#include "egg_sieve_level_real.cuh"

namespace egg {

size_t fast_ws_bytes(int nmax, int cplx, int mhi) { return fast_ws_doubles(nmax, cplx, mhi) * sizeof(double); }

size_t level_ws_bytes(int nmax, int cplx, int k, bool exact)
{
    if (exact && k <= 16) return (cplx ? ctile_ws_doubles(nmax, 2 * k) : tile_ws_doubles(nmax, 2 * k, true)) * sizeof(double);
    return fast_ws_doubles(nmax, cplx, 2 * k) * sizeof(double);
}

template int level_launch_real_lo<false>(const SieveArgs &, const int64_t *, int, int, bool, dd *, int, cudaStream_t);
template int level_launch_all_real_lo<false>(const SieveArgs &, int, bool, dd *, int, cudaStream_t);
template int level_shape_real_lo<false>(int, int, bool, bool, int *, int *);
extern template int level_launch_real_lo<true>(const SieveArgs &, const int64_t *, int, int, bool, dd *, int, cudaStream_t);
extern template int level_launch_all_real_lo<true>(const SieveArgs &, int, bool, dd *, int, cudaStream_t);
extern template int level_shape_real_lo<true>(int, int, bool, bool, int *, int *);

int level_launch_real(const SieveArgs &a, const int64_t *strides, int B, int k, bool narrow, bool exact, dd *partial,
                      int blocks_x, cudaStream_t st)
{
    if (k > 16) {
        if (exact) return fail(EGG_ERR_ARGUMENT, "the reference-arithmetic tiles hold up to 32 rows");
        return level_launch_real_hi(a, strides, B, k, narrow, partial, blocks_x, st);
    }
    return exact ? level_launch_real_lo<true>(a, strides, B, k, narrow, partial, blocks_x, st)
                 : level_launch_real_lo<false>(a, strides, B, k, narrow, partial, blocks_x, st);
}

int level_launch_all_real(const SieveArgs &a, int k, bool narrow, bool exact, dd *partial, int blocks_x, cudaStream_t st)
{
    return exact ? level_launch_all_real_lo<true>(a, k, narrow, partial, blocks_x, st)
                 : level_launch_all_real_lo<false>(a, k, narrow, partial, blocks_x, st);
}

int level_shape_real(int nmax, int k, bool narrow, bool exact, bool all, int *warps_per_block, int *blocks_per_sm)
{
    if (k > 16) {
        if (exact) return fail(EGG_ERR_ARGUMENT, "the reference-arithmetic tiles hold up to 32 rows");
        return level_shape_real_hi(nmax, k, narrow, warps_per_block, blocks_per_sm);
    }
    return exact ? level_shape_real_lo<true>(nmax, k, narrow, all, warps_per_block, blocks_per_sm)
                 : level_shape_real_lo<false>(nmax, k, narrow, all, warps_per_block, blocks_per_sm);
}

}  // namespace egg
