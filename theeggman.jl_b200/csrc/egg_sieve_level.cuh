// egg_sieve_level.cuh -- the popcount-level kernels of the register-resident sieve.
//
// A term's size is m = 2k for its k surviving edges (multiplicity nonzero after the Glynn
// substitution).  One kernel per level k evaluates exactly the terms with k surviving edges, on a
// register tile of exactly m columns: no slot, step or La Budde order is spent on sizes the level
// does not have, and each level's block count follows its own register need.
//
//   * Distinct rows under inclusion-exclusion (every multiplicity 1: hafnian(A; method=:sieve)'s
//     variant for distinct rows, src/hafnian.jl:1139-1146): term j is the subset of edges whose
//     digit is 1, so the level's terms are the k-subsets.  Every warp takes an equal share of them
//     (one colex unrank, then Gosper successors), and the level runs as one balanced wave.
//   * Any other multiplicities (hafnian_repeated, Glynn): when instances of the batch share a small
//     pattern, its terms come listed per level (digits packed 4 bits per edge) and are dealt in
//     equal shares; otherwise each group walks runs of 16 consecutive odometer indices, dealt round
//     robin, and evaluates the terms of its level among them.
//
// Each block writes one partial (re, im) per instance: its warps' double-double sums added in a
// fixed order.
#pragma once
#include "egg_sieve_fast.cuh"

namespace egg {

// 128-thread blocks; resident blocks per SM from the tile's register need (65536 / (128 * blocks)
// registers per thread): a real tile holds m doubles per row, a complex one 2m.
template <bool CPLX, int K, int G = 32>
struct LevelShape {
    static constexpr int MW = 2 * K;
    static constexpr int threads = 128;
    static constexpr int full =
        CPLX ? (MW <= 8 ? 6 : (MW <= 10 ? 5 : (MW <= 16 ? 4 : (MW <= 24 ? 3 : 2))))
             : (MW <= 8 ? 8 : (MW <= 12 ? 7 : (MW <= 18 ? 6 : (MW <= 26 ? 5 : (MW <= 32 ? 4 : 2)))));
    // Two terms per warp need more registers per thread (the series holds two coefficients per
    // lane); one block fewer still keeps more terms in flight.
    static constexpr int min_blocks = G == 32 ? full : (full > 2 ? full - 1 : 1);
};

// Lanes per term: tiles of up to 16 rows (m <= 16) run two terms per warp, one per half-warp group
// of 16 lanes, so that the lanes beyond m are not left idle.  Every shuffle, vote, reduction and
// warp barrier of a term names only its group's lanes.
template <int K>
constexpr int level_group(bool narrow)
{
    return (narrow && 2 * K <= 16) ? 16 : 32;
}

// ALL: the all-levels mode of one small distinct-row instance (level_launch_all_*), a separate
// instantiation.
template <bool CPLX, int K, int G, bool ALL = false>
__global__ void __launch_bounds__(LevelShape<CPLX, K, G>::threads, LevelShape<CPLX, K, G>::min_blocks)
    sieve_level_kernel(SieveArgs a, const int64_t *__restrict__ strides, dd *partial)
{
    constexpr int MW = 2 * K;
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    constexpr int NG = 32 / G;   // groups per warp
    constexpr int GB = cw * NG;  // groups per block
    extern __shared__ double smem[];
    const int grp = threadIdx.x / G, gl = threadIdx.x & (G - 1);
    const int gbase = (threadIdx.x & 31) & ~(G - 1);  // the group's first lane within its warp
    const unsigned gm = G == 32 ? FULL : (0xFFFFu << gbase);
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    const int E = in.E, n = in.n;
    const FastWs w = fast_carve(smem + (size_t)grp * fast_ws_doubles(a.nmax, CPLX, MW), a.nmax, CPLX, MW);
    const int gslot = blockIdx.x * GB + grp;
    const uint64_t W = (uint64_t)a.warps_per_inst * NG;  // groups per instance
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    // One term: the surviving edges are compacted into w.eidx / w.kval (mE of them, mE = K except
    // in the all-levels mode) by the caller.
    auto eval_term = [&](double prefac, int mE) {
        if constexpr (!CPLX) {
            const double val = term_real<MW, (MW > 32 ? 2 : 1), G>((const double *)a.Ax + in.ax_off, in.lda, E,
                                                                   ALL ? mE : K, n, w, gl, gm);
            if (gl == 0) dd_add(acc_re, prefac * val);
        } else {
            const cd val = term_cplx<MW, G>((const cd *)a.Ax + in.ax_off, in.lda, E, ALL ? mE : K, n, w, gl, gm);
            if (gl == 0) {
                dd_add(acc_re, prefac * val.re);
                dd_add(acc_im, prefac * val.im);
            }
        }
    };
    // The group's lanes of a warp vote, as bits 0..G-1.
    auto group_ballot = [&](bool p) -> unsigned {
        const unsigned v = __ballot_sync(gm, p);
        return G == 32 ? v : (v >> gbase) & 0xFFFFu;
    };
    // Each round every group first finds its next term, then the warp evaluates them together (the
    // groups of a warp stay converged through the term), until no group of the warp has one left.
    if constexpr (ALL) {
        // Every nonzero edge subset of the one instance (E <= K): subset r + 1 for r = gslot,
        // gslot + W, ...; a term of k edges has m = 2k <= MW rows.
        const uint64_t cnt = ((uint64_t)1 << E) - 1;
        for (uint64_t r = gslot;; r += W) {
            const bool has = r < cnt;
            if (!__any_sync(FULL, has)) break;
            if (has) {
                const uint32_t S = (uint32_t)r + 1u;
                const int k = __popc(S);
                const double prefac = ((n - k) & 1) ? -1.0 : 1.0;
                for (int e = gl; e < E; e += G)
                    if ((S >> e) & 1u) {
                        const int pos = __popc(S & ((1u << e) - 1u));
                        w.eidx[pos] = e;
                        w.kval[pos] = 1.0;
                    }
                __syncwarp(gm);
                eval_term(prefac, k);
                __syncwarp(gm);
            }
        }
    } else if (in.subset && K <= E) {
        const uint64_t cnt = c_fast.binom[E * 33 + K];
        const uint64_t lo = (uint64_t)gslot * cnt / W, hi = ((uint64_t)gslot + 1) * cnt / W;
        const double prefac = ((n - K) & 1) ? -1.0 : 1.0;  // (-1)^(n - k), every binomial factor 1
        uint32_t S = lo < hi ? subset_unrank(E, K, (uint32_t)lo) : 0u;
        for (uint64_t rk = lo;; ++rk) {
            const bool has = rk < hi;
            if (!__any_sync(FULL, has)) break;
            if (has) {
                if (rk > lo) S = subset_next(S);
                for (int e = gl; e < E; e += G)
                    if ((S >> e) & 1u) {
                        const int pos = __popc(S & ((1u << e) - 1u));
                        w.eidx[pos] = e;
                        w.kval[pos] = 1.0;
                    }
                __syncwarp(gm);
                eval_term(prefac, K);
                __syncwarp(gm);
            }
        }
    } else if (in.pattern >= 0 && K <= E) {
        // The level's terms listed by digits (a multiplicity pattern shared by instances of the
        // batch): every group takes an equal share of the list, as for subsets.  Lane i of the group
        // takes digit i (E <= 16 here), and the term is set up as on the odometer below.
        const int64_t lrow = (int64_t)in.pattern * a.list_stride + K;
        const int64_t lb = a.list_off[lrow];
        const uint64_t cnt = (uint64_t)(a.list_off[lrow + 1] - lb);
        const uint64_t lo = (uint64_t)gslot * cnt / W, hi = ((uint64_t)gslot + 1) * cnt / W;
        const int *reps = a.reps + in.reps_off;
        const int mr1 = a.maxrep + 1;
        const bool unit = a.maxrep <= 1;
        const int r = gl < E ? reps[gl] : 0;
        for (uint64_t rk = lo;; ++rk) {
            const bool has = rk < hi;
            if (!__any_sync(FULL, has)) break;
            if (has) {
                const uint64_t word = a.lists[lb + (int64_t)rk];
                const int digit = gl < E ? (int)((word >> (4 * gl)) & 15u) : 0;
                const int kk = gl < E ? (in.glynn ? 2 * digit - r : digit) : 0;
                const bool nz = gl < E && kk != 0;
                const unsigned mask = group_ballot(nz);
                const int esum = __reduce_add_sync(gm, gl < E ? digit : 0);
                double bp = 1.0;
                if (!unit) {
                    bp = gl < E ? a.binoms[r + digit * mr1] : 1.0;
                    for (int off = G / 2; off > 0; off >>= 1) bp *= __shfl_xor_sync(gm, bp, off, G);
                }
                double prefac = ((n - esum) & 1) ? -bp : bp;
                const int k0 = __shfl_sync(gm, kk, 0, G);
                if (in.glynn && k0 == 0) prefac *= 0.5;  // the mirror's fixed point (:570-573)
                if (nz) {
                    const int pos = __popc(mask & ((1u << gl) - 1u));
                    w.eidx[pos] = gl;
                    w.kval[pos] = (double)kk;
                }
                __syncwarp(gm);
                eval_term(prefac, K);
                __syncwarp(gm);
            }
        }
    } else if (K <= E) {
        // Mixed-radix odometer (src/hafnian.jl:542-580): lane i of the group holds digit i (edge
        // E-1 least significant; E <= G here), digit 0 clipped to its lower half under Glynn.  Runs
        // of kRunTerms consecutive indices are dealt round robin: a term's size is set by its
        // digits, and a long contiguous range fixes the high digits, so contiguous ranges would hand
        // some groups most of a level and others none of it.
        const int *reps = a.reps + in.reps_off;
        const int mr1 = a.maxrep + 1;
        const bool unit = a.maxrep <= 1;  // all multiplicities <= 1: every binomial factor is 1
        int r = 0, base = 1, digit = 0;
        if (gl < E) {
            r = reps[gl];
            base = (in.glynn && gl == 0) ? (r + 2) / 2 : r + 1;
        }
        constexpr int64_t kRunTerms = 16;
        int64_t j0 = (int64_t)gslot * kRunTerms;
        int64_t j = j0, j1 = j0 < in.steps ? (j0 + kRunTerms < in.steps ? j0 + kRunTerms : in.steps) : j0;
        if (gl < E && j0 < in.steps) digit = (int)((j0 / strides[in.reps_off + gl]) % base);
        for (;;) {
            bool has = false;
            double prefac = 0.0;
            while (j < j1) {
                const int kk = gl < E ? (in.glynn ? 2 * digit - r : digit) : 0;
                const bool nz = gl < E && kk != 0;
                const unsigned mask = group_ballot(nz);
                const bool hit = __popc(mask) == K;
                if (hit) {
                    const int esum = __reduce_add_sync(gm, gl < E ? digit : 0);
                    double bp = 1.0;
                    if (!unit) {
                        bp = gl < E ? a.binoms[r + digit * mr1] : 1.0;
                        for (int off = G / 2; off > 0; off >>= 1) bp *= __shfl_xor_sync(gm, bp, off, G);
                    }
                    prefac = ((n - esum) & 1) ? -bp : bp;
                    const int k0 = __shfl_sync(gm, kk, 0, G);
                    if (in.glynn && k0 == 0) prefac *= 0.5;  // the mirror's fixed point (:570-573)
                    if (nz) {
                        const int pos = __popc(mask & ((1u << gl) - 1u));
                        w.eidx[pos] = gl;
                        w.kval[pos] = (double)kk;
                    }
                    has = true;
                }
                // Move to index j + 1: the next odometer value, or the start of the group's next run.
                ++j;
                if (j < j1) {
                    const unsigned notmax = group_ballot(gl < E && digit != base - 1);
                    const int h = 31 - __clz(notmax);
                    if (gl == h) ++digit;
                    else if (gl > h && gl < E) digit = 0;
                } else {
                    j0 += (int64_t)W * kRunTerms;
                    if (j0 < in.steps) {
                        j = j0;
                        j1 = j0 + kRunTerms < in.steps ? j0 + kRunTerms : in.steps;
                        if (gl < E) digit = (int)((j0 / strides[in.reps_off + gl]) % base);
                    }
                }
                if (hit) break;
            }
            if (!__any_sync(FULL, has)) break;
            if (has) {
                __syncwarp(gm);
                eval_term(prefac, K);
                __syncwarp(gm);
            }
        }
    }
    // The block's groups summed in a fixed order: one partial per block.
    __shared__ dd red[2 * GB];
    if (gl == 0) {
        red[2 * grp] = acc_re;
        red[2 * grp + 1] = acc_im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dd re = red[0], im = red[1];
#pragma unroll
        for (int q = 1; q < GB; ++q) {
            dd_add(re, red[2 * q]);
            dd_add(im, red[2 * q + 1]);
        }
        dd *out = partial + ((size_t)b * gridDim.x + blockIdx.x) * 2;
        out[0] = re;
        out[1] = im;
    }
    if constexpr (ALL) {
        // The last block to finish sums all blocks' partials in a fixed order (thread t takes
        // partials t, t + 128, ...; then the warps' lanes pairwise; then the warps in order) and
        // writes the value, so no reduction launch follows.
        __shared__ bool last;
        if (threadIdx.x == 0) {
            __threadfence();
            last = atomicAdd(a.done, 1u) == gridDim.x - 1;
        }
        __syncthreads();
        if (last) {
            __threadfence();
            dd re{0.0, 0.0}, im{0.0, 0.0};
            for (unsigned p = threadIdx.x; p < gridDim.x; p += blockDim.x) {
                const dd *q = partial + (size_t)p * 2;
                dd_add(re, dd{__ldcg(&q[0].hi), __ldcg(&q[0].lo)});
                if (CPLX) dd_add(im, dd{__ldcg(&q[1].hi), __ldcg(&q[1].lo)});
            }
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            for (int off = 16; off > 0; off >>= 1) {
                const dd ro{__shfl_down_sync(FULL, re.hi, off), __shfl_down_sync(FULL, re.lo, off)};
                const dd io{__shfl_down_sync(FULL, im.hi, off), __shfl_down_sync(FULL, im.lo, off)};
                if (lane < off) {
                    dd_add(re, ro);
                    if (CPLX) dd_add(im, io);
                }
            }
            __syncthreads();  // red[] is free again
            if (lane == 0) {
                red[2 * wid] = re;
                red[2 * wid + 1] = im;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                dd fr = red[0], fi = red[1];
                for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                    dd_add(fr, red[2 * w]);
                    if (CPLX) dd_add(fi, red[2 * w + 1]);
                }
                const double hr = __dadd_rn(fr.hi, fr.lo);
                if (CPLX) ((cd *)a.fused_out)[0] = cd{hr, __dadd_rn(fi.hi, fi.lo)};
                else ((double *)a.fused_out)[0] = hr;
            }
        }
    }
}

template <bool CPLX, int K, int G>
static int level_launch_k(const SieveArgs &a, const int64_t *strides, int B, dd *partial, int blocks_x, cudaStream_t st)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * (32 / G) * fast_ws_doubles(a.nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K, G>;
    int rc = smem_limit_at_least((const void *)k, smem);
    if (rc) return rc;
    k<<<dim3((unsigned)blocks_x, (unsigned)B), cw * 32, smem, st>>>(a, strides, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int K, int G>
static int level_launch_all_k(const SieveArgs &a, dd *partial, int blocks_x, cudaStream_t st)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * (32 / G) * fast_ws_doubles(a.nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K, G, true>;
    int rc = smem_limit_at_least((const void *)k, smem);
    if (rc) return rc;
    k<<<dim3((unsigned)blocks_x, 1u), cw * 32, smem, st>>>(a, nullptr, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int K, int G>
static int level_shape_k(int nmax, int *warps_per_block, int *blocks_per_sm)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * (32 / G) * fast_ws_doubles(nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K, G>;
    int nb = 0;
    int rc = smem_limit_at_least((const void *)k, smem);
    if (!rc) rc = egg::blocks_per_sm((const void *)k, cw * 32, smem, &nb);
    if (rc) return rc;
    *warps_per_block = cw;
    *blocks_per_sm = nb;
    return EGG_OK;
}

}  // namespace egg

// Case K of a switch over levels: launch or shape the level-K kernel of the given variant.
#define EGG_LEVEL_CASES(CPLX, X)                                                                   \
    X(CPLX, 1) X(CPLX, 2) X(CPLX, 3) X(CPLX, 4) X(CPLX, 5) X(CPLX, 6) X(CPLX, 7) X(CPLX, 8) X(CPLX, 9) \
    X(CPLX, 10) X(CPLX, 11) X(CPLX, 12) X(CPLX, 13) X(CPLX, 14) X(CPLX, 15) X(CPLX, 16)
// Case K of a switch over the all-levels launches (groups as for the level launch).
#define EGG_ALL_LAUNCH(CPLX, K)                                                                      \
    case K:                                                                                          \
        return narrow ? level_launch_all_k<CPLX, K, level_group<K>(true)>(a, partial, blocks_x, st)  \
                      : level_launch_all_k<CPLX, K, 32>(a, partial, blocks_x, st);
#define EGG_FUSED_CASES(CPLX, X)                                                                    \
    X(CPLX, 1) X(CPLX, 2) X(CPLX, 3) X(CPLX, 4) X(CPLX, 5) X(CPLX, 6) X(CPLX, 7) X(CPLX, 8) X(CPLX, 9) \
    X(CPLX, 10)
#define EGG_LEVEL_CASES_HI(CPLX, X)                                                                 \
    X(CPLX, 17) X(CPLX, 18) X(CPLX, 19) X(CPLX, 20) X(CPLX, 21) X(CPLX, 22) X(CPLX, 23) X(CPLX, 24)
