// egg_sieve.cuh -- structures shared by the exact and the fast sieve kernels.
#pragma once

#include "egg_internal.cuh"

namespace egg {

struct SieveInst {
    int64_t ax_off;     // element offset of this instance's matrix (ld = lda)
    int64_t steps;      // number of sieve terms
    int64_t reps_off;   // offset into the reps / strides arrays
    int E, n, glynn, lda;
    int subset;         // all multiplicities 1 under inclusion-exclusion: term j is the edge subset j
    int pattern;        // >= 0: the instance's terms are listed per level (SieveArgs::lists), else -1
};

struct SieveArgs {
    const void *Ax;
    const int *reps;
    const double *binoms;  // (maxrep+1) x (maxrep+1), binoms[a + b*(maxrep+1)] = C(a, b)
    const uint32_t *binom32;  // C(x, k) at [x * 65 + k], exact for x <= 32
    const SieveInst *inst;
    dd *partial;           // exact kernel: [B][warps_per_inst][2]
    double *terms;         // if set (one instance, exact kernel only): term j's value at j (complex: 2j, 2j+1)
    int maxrep, warps_per_inst, Emax, nmax;
    int block_warps;       // level launches: warps per block when below the shape's own (0: the shape's)
    int skip_le;           // the exact kernel leaves terms with m <= skip_le to the fast kernels
    // Term lists of repeated multiplicity patterns: the digits of each term of pattern p and level k
    // (4 bits per edge, edge i at bits 4i..4i+3) at lists[list_off[p * list_stride + k] ..
    // list_off[p * list_stride + k + 1]), in odometer order.
    const uint64_t *lists;
    const int64_t *list_off;
    int list_stride;
    // The all-levels launch (level_launch_all_*): its last block to finish sums the blocks'
    // partials into fused_out; done counts finished blocks and starts at zero.
    void *fused_out;
    unsigned *done;
};

constexpr int kFusedMaxE = 10;

// Register-tile path (egg_sieve_fast.cuh, egg_sieve_level*.cu): level k evaluates the terms with
// k surviving edges, m = 2k <= 48 (real) or 32 (complex), for any multiplicities.
constexpr int kLevelMaxReal = 24, kLevelMaxCplx = 16;
constexpr int kMaxPartials = 26;  // the exact kernel and up to 25 level launches
size_t fast_ws_bytes(int nmax, int cplx, int mhi);  // one warp's scratch for a tile of mhi columns
// One group's shared workspace of level k's kernel (the real tiles of up to 32 rows hold the
// reference-arithmetic form's term buffer too when `exact`).
size_t level_ws_bytes(int nmax, int cplx, int k, bool exact);
// Launches level k on a grid of blocks_x x B blocks; a.warps_per_inst must be blocks_x times the
// level's warps per block.  Each block writes one partial (re, im) per instance.  `narrow` puts
// two terms in each warp for tiles of up to 16 rows (odometer instances then need E <= 16).
// `exact` (levels 1..16 only) evaluates every term in the reference's arithmetic; with
// a.terms set those kernels write each term's signed value at its index instead of summing.
int level_launch_real(const SieveArgs &a, const int64_t *strides, int B, int k, bool narrow, bool exact, dd *partial,
                      int blocks_x, cudaStream_t st);
int level_launch_real_hi(const SieveArgs &a, const int64_t *strides, int B, int k, bool narrow, dd *partial, int blocks_x,
                         cudaStream_t st);
// One distinct-row instance (B = 1) of k <= kFusedMaxE edges in one launch: every nonzero edge
// subset, each on the tile of m = 2k columns, the blocks' partials summed inside the launch into
// a.fused_out (when set).  A separate instantiation of the level kernel, so the level launches are
// unchanged.
int level_launch_all_real(const SieveArgs &a, int k, bool narrow, bool exact, dd *partial, int blocks_x, cudaStream_t st);
int level_launch_all_cplx(const SieveArgs &a, int k, bool narrow, bool exact, dd *partial, int blocks_x, cudaStream_t st);
int level_launch_cplx(const SieveArgs &a, const int64_t *strides, int B, int k, bool narrow, bool exact, dd *partial,
                      int blocks_x, cudaStream_t st);
// The level's block size in warps and how many of its blocks one SM holds.
int level_shape_real(int nmax, int k, bool narrow, bool exact, bool all, int *warps_per_block, int *blocks_per_sm);
int level_shape_real_hi(int nmax, int k, bool narrow, int *warps_per_block, int *blocks_per_sm);
int level_shape_cplx(int nmax, int k, bool narrow, bool exact, bool all, int *warps_per_block, int *blocks_per_sm);

}  // namespace egg
