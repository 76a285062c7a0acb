// egg_sieve_level_cplx.cuh -- dispatch over the complex popcount levels 1..16 (m = 2 .. 32) for one
// arithmetic form, instantiated once per form (egg_sieve_level_cplx.cu: fused multiply-adds on the
// relabelled tiles, egg_sieve_level_cplx_x.cu: the reference's arithmetic on the logical-order
// tiles) so that the two compile in parallel.
#pragma once
#include <mutex>

#include "egg_sieve_level.cuh"

namespace egg {

#define EGG_LVLC_LAUNCH(CPLX, K)                                                                              \
    case K:                                                                                                    \
        return narrow ? level_launch_k<CPLX, K, level_group<K>(true), EXACT>(a, strides, B, partial, blocks_x, st) \
                      : level_launch_k<CPLX, K, 32, EXACT>(a, strides, B, partial, blocks_x, st);
#define EGG_LVLC_SHAPE(CPLX, K)                                                                                  \
    case K:                                                                                                      \
        rc = narrow ? level_shape_k<CPLX, K, level_group<K>(true), EXACT>(nmax, warps_per_block, blocks_per_sm)   \
                    : level_shape_k<CPLX, K, 32, EXACT>(nmax, warps_per_block, blocks_per_sm);                   \
        break;

template <bool EXACT>
int level_launch_cplx_lo(const SieveArgs &a, const int64_t *strides, int B, int k, bool narrow, dd *partial, int blocks_x,
                         cudaStream_t st)
{
    switch (k) {
        EGG_LEVEL_CASES(true, EGG_LVLC_LAUNCH)
    }
    return fail(EGG_ERR_ARGUMENT, "no such sieve level");
}

template <bool EXACT>
int level_launch_all_cplx_lo(const SieveArgs &a, int k, bool narrow, dd *partial, int blocks_x, cudaStream_t st)
{
    static_assert(kFusedMaxE == 10, "EGG_FUSED_CASES lists the levels 1..kFusedMaxE");
    switch (k) {
        EGG_FUSED_CASES(true, EGG_ALL_LAUNCH)
    }
    return fail(EGG_ERR_ARGUMENT, "no all-levels sieve launch for this edge count");
}

template <bool EXACT>
int level_shape_cplx_lo(int nmax, int k, bool narrow, bool all, int *warps_per_block, int *blocks_per_sm)
{
    static std::mutex mu;  // the entry point that allocates nothing reaches this without the library's lock
    std::lock_guard<std::mutex> lk(mu);
    // Occupancy figures, the same on every device of one model; they depend on the largest term
    // size n (the workspaces' buffered series), hence nmax in the key.
    static int cache[kLevelMaxCplx + 1][2][2][33][2];
    int *slot = (k >= 1 && k <= kLevelMaxCplx && nmax >= 0 && nmax <= 32) ? cache[k][narrow ? 1 : 0][all ? 1 : 0][nmax] : nullptr;
    if (slot && slot[1] > 0) {
        *warps_per_block = slot[0];
        *blocks_per_sm = slot[1];
        return EGG_OK;
    }
    int rc = fail(EGG_ERR_ARGUMENT, all ? "no all-levels sieve launch for this edge count" : "no such sieve level");
    if (all) {
        switch (k) {
            EGG_FUSED_CASES(true, EGG_ALL_SHAPE)
        }
    } else {
        switch (k) {
            EGG_LEVEL_CASES(true, EGG_LVLC_SHAPE)
        }
    }
    if (rc) return rc;
    if (slot) {
        slot[0] = *warps_per_block;
        slot[1] = *blocks_per_sm;
    }
    return EGG_OK;
}

}  // namespace egg
