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
//   * Any other multiplicities (hafnian_repeated, Glynn): each warp walks runs of 16 consecutive
//     odometer indices, dealt round robin, and evaluates the terms of its level among them.
//
// Each block writes one partial (re, im) per instance: its warps' double-double sums added in a
// fixed order.
#pragma once
#include "egg_sieve_fast.cuh"

namespace egg {

// 128-thread blocks; resident blocks per SM from the tile's register need (65536 / (128 * blocks)
// registers per thread): a real tile holds m doubles per row, a complex one 2m.
template <bool CPLX, int K>
struct LevelShape {
    static constexpr int MW = 2 * K;
    static constexpr int threads = 128;
    static constexpr int min_blocks =
        CPLX ? (MW <= 8 ? 6 : (MW <= 10 ? 5 : (MW <= 16 ? 4 : (MW <= 24 ? 3 : 2))))
             : (MW <= 8 ? 8 : (MW <= 12 ? 7 : (MW <= 18 ? 6 : (MW <= 26 ? 5 : (MW <= 32 ? 4 : 2)))));
};

template <bool CPLX, int K>
__global__ void __launch_bounds__(LevelShape<CPLX, K>::threads, LevelShape<CPLX, K>::min_blocks)
    sieve_level_kernel(SieveArgs a, const int64_t *__restrict__ strides, dd *partial)
{
    constexpr int MW = 2 * K;
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    const int E = in.E, n = in.n;
    const FastWs w = fast_carve(smem + (size_t)wib * fast_ws_doubles(a.nmax, CPLX, MW), a.nmax, CPLX, MW);
    const int wslot = blockIdx.x * cw + wib;
    const uint64_t W = (uint64_t)a.warps_per_inst;
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    // One term: the surviving edges are compacted into w.eidx / w.kval (K of them) by the caller.
    auto eval_term = [&](double prefac) {
        if constexpr (!CPLX) {
            const double val = term_real<MW, (MW > 32 ? 2 : 1)>((const double *)a.Ax + in.ax_off, in.lda, E, K, n, w,
                                                                lane);
            if (lane == 0) dd_add(acc_re, prefac * val);
        } else {
            const cd val = term_cplx<MW>((const cd *)a.Ax + in.ax_off, in.lda, E, K, n, w, lane);
            if (lane == 0) {
                dd_add(acc_re, prefac * val.re);
                dd_add(acc_im, prefac * val.im);
            }
        }
    };
    if (in.subset && K <= E) {
        const uint64_t cnt = c_binom[E * 33 + K];
        const uint64_t lo = (uint64_t)wslot * cnt / W, hi = ((uint64_t)wslot + 1) * cnt / W;
        const double prefac = ((n - K) & 1) ? -1.0 : 1.0;  // (-1)^(n - k), every binomial factor 1
        uint32_t S = lo < hi ? subset_unrank(E, K, (uint32_t)lo) : 0u;
        for (uint64_t rk = lo; rk < hi; ++rk) {
            if (rk > lo) S = subset_next(S);
            if (lane < E && ((S >> lane) & 1u)) {
                const int pos = __popc(S & ((1u << lane) - 1u));
                w.eidx[pos] = lane;
                w.kval[pos] = 1.0;
            }
            __syncwarp();
            eval_term(prefac);
            __syncwarp();
        }
    } else if (K <= E) {
        // Mixed-radix odometer (src/hafnian.jl:542-580): lane i holds digit i (edge E-1 least
        // significant), digit 0 clipped to its lower half under Glynn.  Runs of kRunTerms
        // consecutive indices are dealt round robin: a term's size is set by its digits, and a long
        // contiguous range fixes the high digits, so contiguous ranges would hand some warps most of
        // a level and others none of it.
        const int *reps = a.reps + in.reps_off;
        const int mr1 = a.maxrep + 1;
        const bool unit = a.maxrep <= 1;  // all multiplicities <= 1: every binomial factor is 1
        int r = 0, base = 1, digit = 0;
        if (lane < E) {
            r = reps[lane];
            base = (in.glynn && lane == 0) ? (r + 2) / 2 : r + 1;
        }
        constexpr int64_t kRunTerms = 16;
        for (int64_t j0 = (int64_t)wslot * kRunTerms; j0 < in.steps; j0 += (int64_t)W * kRunTerms) {
            const int64_t j1 = j0 + kRunTerms < in.steps ? j0 + kRunTerms : in.steps;
            if (lane < E) digit = (int)((j0 / strides[in.reps_off + lane]) % base);
            for (int64_t j = j0; j < j1; ++j) {
                if (j > j0) {
                    const unsigned notmax = __ballot_sync(FULL, lane < E && digit != base - 1);
                    const int h = 31 - __clz(notmax);
                    if (lane == h) ++digit;
                    else if (lane > h && lane < E) digit = 0;
                }
                const int kk = lane < E ? (in.glynn ? 2 * digit - r : digit) : 0;
                const bool nz = lane < E && kk != 0;
                const unsigned mask = __ballot_sync(FULL, nz);
                if (__popc(mask) != K) continue;  // another level
                const int esum = __reduce_add_sync(FULL, lane < E ? digit : 0);
                double bp = 1.0;
                if (!unit) {
                    bp = lane < E ? a.binoms[r + digit * mr1] : 1.0;
                    for (int off = 16; off > 0; off >>= 1) bp *= __shfl_xor_sync(FULL, bp, off);
                }
                double prefac = ((n - esum) & 1) ? -bp : bp;
                const int k0 = __shfl_sync(FULL, kk, 0);
                if (in.glynn && k0 == 0) prefac *= 0.5;  // the mirror's fixed point (:570-573)
                if (nz) {
                    const int pos = __popc(mask & ((1u << lane) - 1u));
                    w.eidx[pos] = lane;
                    w.kval[pos] = (double)kk;
                }
                __syncwarp();
                eval_term(prefac);
                __syncwarp();
            }
        }
    }
    // The block's warps summed in a fixed order: one partial per block.
    __shared__ dd red[2 * cw];
    if (lane == 0) {
        red[2 * wib] = acc_re;
        red[2 * wib + 1] = acc_im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dd r = red[0], i = red[1];
#pragma unroll
        for (int q = 1; q < cw; ++q) {
            dd_add(r, red[2 * q]);
            dd_add(i, red[2 * q + 1]);
        }
        dd *out = partial + ((size_t)b * gridDim.x + blockIdx.x) * 2;
        out[0] = r;
        out[1] = i;
    }
}

template <bool CPLX, int K>
static int level_launch_k(const SieveArgs &a, const int64_t *strides, int B, dd *partial, int blocks_x, cudaStream_t st)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * fast_ws_doubles(a.nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K>;
    int rc = smem_limit_at_least((const void *)k, smem);
    if (rc) return rc;
    k<<<dim3((unsigned)blocks_x, (unsigned)B), cw * 32, smem, st>>>(a, strides, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int K>
static int level_shape_k(int nmax, int *warps_per_block, int *blocks_per_sm)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * fast_ws_doubles(nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K>;
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
#define EGG_LEVEL_CASES_HI(CPLX, X)                                                                 \
    X(CPLX, 17) X(CPLX, 18) X(CPLX, 19) X(CPLX, 20) X(CPLX, 21) X(CPLX, 22) X(CPLX, 23) X(CPLX, 24)
