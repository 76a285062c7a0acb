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
#include "egg_sieve_tile.cuh"

namespace egg {

// 128-thread blocks; resident blocks per SM from the tile's register need (65536 / (128 * blocks)
// registers per thread): a real tile holds m doubles per row, a complex one 2m.
// The real reference-arithmetic tiles keep more values live per step (separately rounded products,
// the buffered term series) and run fewer blocks, whose larger register share spills less (the
// N = 40 sieve 9.25 -> 8.91 ms against the fused tiles' block counts).
template <bool CPLX, int K, int G = 32, bool EXACT = false, bool ALL = false>
struct LevelShape {
    static constexpr int MW = 2 * K;
    static constexpr int full =
        CPLX    ? (MW <= 8 ? 6 : (MW <= 10 ? 5 : (MW <= 16 ? 4 : (MW <= 24 ? 3 : 2))))
        : EXACT ? (MW <= 8 ? 8 : (MW <= 12 ? 6 : (MW <= 20 ? 5 : (MW <= 32 ? 4 : 2))))
                : (MW <= 8 ? 8 : (MW <= 12 ? 7 : (MW <= 18 ? 6 : (MW <= 26 ? 5 : (MW <= 32 ? 4 : 2)))));
    // Two terms per warp need more registers per thread (the series holds two coefficients per
    // lane); one block fewer still keeps more terms in flight.
    static constexpr int per_sm = G == 32 ? full : (full > 2 ? full - 1 : 1);
    // Lockstep: the reference-arithmetic tiles of 17..32 rows run as ONE block per SM holding all
    // of its warps, which take their terms in rounds separated by a block barrier.  Each term runs
    // about 5 k instructions of straight-line code (every Hessenberg step is its own code), and
    // warps spread over different parts of it stall on instruction fetch; in lockstep the warps of
    // an SM run the same part at the same time.  The real N = 40 sieve took 10.52 -> 9.67 ms.  The
    // launch planner may instead launch such a kernel in blocks of four warps (SieveArgs::
    // block_warps): a level with few rounds of terms (egg_sieve.cu, kLockstepMinRounds*).
    static constexpr bool lockstep = !ALL && EXACT && G == 32 && MW > 16 && MW <= 32;
    static constexpr int threads = lockstep ? 128 * per_sm : 128;
    static constexpr int min_blocks = lockstep ? 1 : per_sm;
};

// Lanes per term: tiles of up to 16 rows (m <= 16) run two terms per warp, one per half-warp group
// of 16 lanes, so that the lanes beyond m are not left idle.  Every shuffle, vote, reduction and
// warp barrier of a term names only its group's lanes.
template <int K>
constexpr int level_group(bool narrow)
{
    return (narrow && 2 * K <= 16) ? 16 : 32;
}

// In the reference's arithmetic, terms of up to 32 rows (real or complex) run on the tiles whose
// columns stay in logical order (egg_sieve_tile.cuh).  With fused multiply-adds every term runs on
// the relabelled tiles of egg_sieve_fast.cuh, which move no data on a pivot swap and so keep their
// code compact.
template <bool CPLX, int K, bool EXACT>
constexpr bool level_tile() { return EXACT && 2 * K <= 32; }

// One group's shared workspace, in doubles.
template <bool CPLX, int K, bool EXACT>
__host__ __device__ inline size_t level_ws_doubles(int nmax)
{
    if constexpr (level_tile<CPLX, K, EXACT>()) return CPLX ? ctile_ws_doubles(nmax, 2 * K) : tile_ws_doubles(nmax, 2 * K, EXACT);
    else return fast_ws_doubles(nmax, CPLX, 2 * K);
}

// Term value of one lane's buffered term (EXACT): the series of its q vector, times its prefactor.
// Deterministic sum of a group's buffered terms: a fixed shuffle tree of double-double values.
__device__ __forceinline__ dd group_tree_sum(dd v, unsigned gm, int G)
{
    for (int off = G / 2; off > 0; off >>= 1) {
        const dd o{__shfl_down_sync(gm, v.hi, off, G), __shfl_down_sync(gm, v.lo, off, G)};
        dd_add(v, o);
    }
    return v;
}

// ALL: the all-levels mode of one small distinct-row instance (level_launch_all_*), a separate
// instantiation.  EXACT: every term in the reference's arithmetic (logical-order tiles); the term
// series are evaluated in batches of G terms, one term per lane, and with a.terms set each term's
// signed value is written at its index instead of being summed.
template <bool CPLX, int K, int G, bool ALL = false, bool EXACT = false>
__global__ void __launch_bounds__(LevelShape<CPLX, K, G, EXACT, ALL>::threads, LevelShape<CPLX, K, G, EXACT, ALL>::min_blocks)
    sieve_level_kernel(SieveArgs a, const int64_t *__restrict__ strides, dd *partial)
{
    constexpr int MW = 2 * K;
    constexpr bool TILE = level_tile<CPLX, K, EXACT>();
    static_assert(!EXACT || TILE, "the exact form runs on the logical-order tiles");
    constexpr int NG = 32 / G;   // groups per warp
    constexpr int GB_MAX = LevelShape<CPLX, K, G, EXACT, ALL>::threads / 32 * NG;
    const int GB = (int)(blockDim.x >> 5) * NG;  // groups per block (a lockstep block may hold fewer warps)
    extern __shared__ double smem[];
    const int grp = threadIdx.x / G, gl = threadIdx.x & (G - 1);
    const int gbase = (threadIdx.x & 31) & ~(G - 1);  // the group's first lane within its warp
    const unsigned gm = G == 32 ? FULL : (0xFFFFu << gbase);
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    const int E = in.E, n = in.n;
    double *wbase = smem + (size_t)grp * level_ws_doubles<CPLX, K, EXACT>(a.nmax);
    FastWs wf{};
    const TileWs<MW> wt{wbase};
    const CTileWs<MW> wc{wbase};
    if constexpr (!TILE) wf = fast_carve(wbase, a.nmax, CPLX, MW);
    int *const eidx = TILE ? (CPLX ? wc.eidx() : wt.eidx()) : wf.eidx;
    double *const kval = TILE ? (CPLX ? wc.kval() : wt.kval()) : wf.kval;
    const int gslot = blockIdx.x * GB + grp;
    const uint64_t W = (uint64_t)a.warps_per_inst * NG;  // groups per instance
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    // EXACT: the group's buffered terms (slot s: q vector at qbuf + s * (nmax + 1), prefactor,
    // index and size at pre[s], jx[s], mx[s]).
    int nbuf = 0;
    auto flush = [&]() {
        if constexpr (EXACT && !CPLX) {
            __syncwarp(gm);
            double v = 0.0;
            if (gl < nbuf) {
                double f[32];
                const double val = series_exact(wt.qbuf() + (size_t)gl * (a.nmax + 1), f, wt.mx()[gl], n);
                v = __dmul_rn(wt.pre()[gl], val);
                if (a.terms) a.terms[wt.jx()[gl]] = v;
            }
            if (!a.terms) {
                const dd t = group_tree_sum(dd{v, 0.0}, gm, G);
                if (gl == 0) dd_add(acc_re, t);
            }
            nbuf = 0;
            __syncwarp(gm);
        } else if constexpr (EXACT) {
            __syncwarp(gm);
            double vr = 0.0, vi = 0.0;
            if (gl < nbuf) {
                cd f[32];
                const cd val = series_cplx_exact(wc.qbuf() + (size_t)gl * (a.nmax + 1), f, wc.mx()[gl], n);
                const double pf = wc.pre()[gl];
                vr = __dmul_rn(pf, val.re);
                vi = __dmul_rn(pf, val.im);
                if (a.terms) {
                    a.terms[2 * wc.jx()[gl]] = vr;
                    a.terms[2 * wc.jx()[gl] + 1] = vi;
                }
            }
            if (!a.terms) {
                const dd tr = group_tree_sum(dd{vr, 0.0}, gm, G);
                const dd ti = group_tree_sum(dd{vi, 0.0}, gm, G);
                if (gl == 0) {
                    dd_add(acc_re, tr);
                    dd_add(acc_im, ti);
                }
            }
            nbuf = 0;
            __syncwarp(gm);
        }
    };
    // One term: the surviving edges are compacted into eidx / kval (mE of them, mE = K except in
    // the all-levels mode) by the caller; jidx is the term's index (used with a.terms).
    auto eval_term = [&](double prefac, int mE, int64_t jidx) {
        if constexpr (CPLX && TILE) {
            const int mm = 2 * (ALL ? mE : K);
            term_cplx_tile<MW, G>((const cd *)a.Ax + in.ax_off, in.lda, E, ALL ? mE : K, n, wc, gl, gm);
            cd *dst = wc.qbuf() + (size_t)nbuf * (a.nmax + 1);
            const int jm = mm < n ? mm : n;
            for (int j = 1 + gl; j <= jm; j += G) dst[j] = wc.q()[j];
            if (gl == 0) {
                wc.pre()[nbuf] = prefac;
                wc.mx()[nbuf] = mm;
                wc.jx()[nbuf] = jidx;
            }
            if (++nbuf == G) flush();
            __syncwarp(gm);
        } else if constexpr (CPLX) {
            const cd val = term_cplx<MW, G>((const cd *)a.Ax + in.ax_off, in.lda, E, ALL ? mE : K, n, wf, gl, gm);
            if (gl == 0) {
                dd_add(acc_re, prefac * val.re);
                dd_add(acc_im, prefac * val.im);
            }
        } else if constexpr (TILE) {
            const int mm = 2 * (ALL ? mE : K);
            term_real_tile<MW, G, EXACT>((const double *)a.Ax + in.ax_off, in.lda, E, ALL ? mE : K, n, wt, gl, gm);
            {
                // Buffer q_1..q_min(m,n) in slot nbuf; the lane of that slot keeps the rest.
                double *dst = wt.qbuf() + (size_t)nbuf * (a.nmax + 1);
                const int jm = mm < n ? mm : n;
                for (int j = 1 + gl; j <= jm; j += G) dst[j] = wt.q()[j];
                if (gl == 0) {
                    wt.pre()[nbuf] = prefac;
                    wt.mx()[nbuf] = mm;
                    wt.jx()[nbuf] = jidx;
                }
                if (++nbuf == G) flush();
                __syncwarp(gm);
            }
        } else {
            const double val = term_real<MW, (MW > 32 ? 2 : 1), G>((const double *)a.Ax + in.ax_off, in.lda, E,
                                                                   ALL ? mE : K, n, wf, gl, gm);
            if (gl == 0) dd_add(acc_re, prefac * val);
        }
    };
    // The index of the term whose edge subset is S (edge i at bit E-1-i of the index, as the
    // odometer's edge E-1 is least significant).
    auto subset_index = [&](uint32_t S) -> int64_t { return E ? (int64_t)(__brev(S) >> (32 - E)) : 0; };
    // The group's lanes of a warp vote, as bits 0..G-1.
    auto group_ballot = [&](bool p) -> unsigned {
        const unsigned v = __ballot_sync(gm, p);
        return G == 32 ? v : (v >> gbase) & 0xFFFFu;
    };
    // Each round every group first finds its next term, then the warp evaluates them together (the
    // groups of a warp stay converged through the term), until no group of the warp has one left.
    // Every way of dealing terms feeds the one evaluation below, so that it is compiled once.
    //
    //   * ALL: every nonzero edge subset of the one instance (E <= K): subset r + 1 for
    //     r = gslot, gslot + W, ...; a term of k edges has m = 2k <= MW rows.
    //   * subsets: all multiplicities 1 under inclusion-exclusion, so the level's terms are the
    //     K-subsets of the edges; the group takes an equal share of them (one colex unrank, then
    //     successors).
    //   * lists: the level's terms listed by digits (a multiplicity pattern shared by instances of
    //     the batch); the group takes an equal share of the list.  Lane i of the group takes digit i
    //     (E <= 16 here), and the term is set up as on the odometer.
    //   * odometer: the mixed-radix odometer (src/hafnian.jl:542-580): lane i of the group holds
    //     digit i (edge E-1 least significant; E <= G here), digit 0 clipped to its lower half under
    //     Glynn.  Runs of kRunTerms consecutive indices are dealt round robin: a term's size is set
    //     by its digits, and a long contiguous range fixes the high digits, so contiguous ranges
    //     would hand some groups most of a level and others none of it.
    enum { kAll, kSubset, kList, kOdometer, kNone };
    const int mode = ALL ? kAll : (K > E ? kNone : (in.subset ? kSubset : (in.pattern >= 0 ? kList : kOdometer)));
    const int *reps = a.reps + in.reps_off;
    const int mr1 = a.maxrep + 1;
    const bool unit = a.maxrep <= 1;  // all multiplicities <= 1: every binomial factor is 1
    constexpr int64_t kRunTerms = 16;
    // ALL: rk is the next subset; subsets and lists: the group's share is [lo, hi), rk the next;
    // odometer: the current run is [lo, hi), rk the next index.
    int64_t rk = 0, lo = 0, hi = 0;
    uint32_t S = 0;
    int64_t lb = 0;
    int r = 0, base = 1, digit = 0;  // odometer and lists: this lane's multiplicity, radix and digit
    if (mode == kAll) {
        rk = gslot;
    } else if (mode == kSubset) {
        const uint64_t cnt = c_fast.binom[E * 33 + K];
        lo = (int64_t)((uint64_t)gslot * cnt / W);
        hi = (int64_t)(((uint64_t)gslot + 1) * cnt / W);
        rk = lo;
        S = lo < hi ? subset_unrank(E, K, (uint32_t)lo) : 0u;
    } else if (mode == kList) {
        const int64_t lrow = (int64_t)in.pattern * a.list_stride + K;
        lb = a.list_off[lrow];
        const uint64_t cnt = (uint64_t)(a.list_off[lrow + 1] - lb);
        lo = (int64_t)((uint64_t)gslot * cnt / W);
        hi = (int64_t)(((uint64_t)gslot + 1) * cnt / W);
        rk = lo;
        r = gl < E ? reps[gl] : 0;
    } else if (mode == kOdometer) {
        if (gl < E) {
            r = reps[gl];
            base = (in.glynn && gl == 0) ? (r + 2) / 2 : r + 1;
        }
        lo = (int64_t)gslot * kRunTerms;
        rk = lo;
        hi = lo < in.steps ? (lo + kRunTerms < in.steps ? lo + kRunTerms : in.steps) : lo;
        if (gl < E && lo < in.steps) digit = (int)((lo / strides[in.reps_off + gl]) % base);
    }
    // Sets this group's next term up (eidx/kval, prefactor, surviving edges, index) for a digit
    // vector held one digit per lane: the Glynn substitution, the binomial product and the sign.
    auto setup_digits = [&](int dg, double &prefac, int64_t &jidx, bool want_index) -> void {
        const int kk = gl < E ? (in.glynn ? 2 * dg - r : dg) : 0;
        const bool nz = gl < E && kk != 0;
        const unsigned mask = group_ballot(nz);
        const int esum = __reduce_add_sync(gm, gl < E ? dg : 0);
        double bp = 1.0;
        if (!unit) {
            bp = gl < E ? a.binoms[r + dg * mr1] : 1.0;
            for (int off = G / 2; off > 0; off >>= 1) bp *= __shfl_xor_sync(gm, bp, off, G);
        }
        prefac = ((n - esum) & 1) ? -bp : bp;
        const int k0 = __shfl_sync(gm, kk, 0, G);
        if (in.glynn && k0 == 0) prefac *= 0.5;  // the mirror's fixed point (:570-573)
        if (nz) {
            const int pos = __popc(mask & ((1u << gl) - 1u));
            eidx[pos] = gl;
            kval[pos] = (double)kk;
        }
        if (EXACT && want_index && a.terms) {
            // The term's index: its digits in the mixed-radix place values.
            int64_t part = gl < E ? (int64_t)dg * strides[in.reps_off + gl] : 0;
            for (int off = G / 2; off > 0; off >>= 1) part += __shfl_xor_sync(gm, part, off, G);
            jidx = part;
        }
    };
    // Edges of subset S into eidx/kval (every multiplicity 1).
    auto setup_subset = [&](uint32_t Sv) -> void {
        for (int e = gl; e < E; e += G)
            if ((Sv >> e) & 1u) {
                const int pos = __popc(Sv & ((1u << e) - 1u));
                eidx[pos] = e;
                kval[pos] = 1.0;
            }
    };
    for (;;) {
        bool has = false;
        double prefac = 0.0;
        int mE = K;
        int64_t jidx = 0;
        if (mode == kAll) {
            const int64_t cnt = ((int64_t)1 << E) - 1;
            if (rk < cnt) {
                const uint32_t Sv = (uint32_t)rk + 1u;
                mE = __popc(Sv);
                prefac = ((n - mE) & 1) ? -1.0 : 1.0;
                setup_subset(Sv);
                jidx = subset_index(Sv);
                rk += W;
                has = true;
            }
        } else if (mode == kSubset) {
            if (rk < hi) {
                if (rk > lo) S = subset_next(S);
                prefac = ((n - K) & 1) ? -1.0 : 1.0;  // (-1)^(n - k), every binomial factor 1
                setup_subset(S);
                jidx = subset_index(S);
                ++rk;
                has = true;
            }
        } else if (mode == kList) {
            const bool more = rk < hi;
            if (more) {
                const uint64_t word = a.lists[lb + rk];
                const int dg = gl < E ? (int)((word >> (4 * gl)) & 15u) : 0;
                setup_digits(dg, prefac, jidx, true);
                ++rk;
                has = true;
            }
        } else if (mode == kOdometer) {
            while (rk < hi) {
                const int kk = gl < E ? (in.glynn ? 2 * digit - r : digit) : 0;
                const bool hit = __popc(group_ballot(gl < E && kk != 0)) == K;
                if (hit) {
                    setup_digits(digit, prefac, jidx, false);
                    jidx = rk;
                    has = true;
                }
                // Move to index rk + 1: the next odometer value, or the start of the group's next run.
                ++rk;
                if (rk < hi) {
                    const unsigned notmax = group_ballot(gl < E && digit != base - 1);
                    const int h = 31 - __clz(notmax);
                    if (gl == h) ++digit;
                    else if (gl > h && gl < E) digit = 0;
                } else {
                    lo += (int64_t)W * kRunTerms;
                    if (lo < in.steps) {
                        rk = lo;
                        hi = lo + kRunTerms < in.steps ? lo + kRunTerms : in.steps;
                        if (gl < E) digit = (int)((lo / strides[in.reps_off + gl]) % base);
                    }
                }
                if (hit) break;
            }
        }
        if constexpr (LevelShape<CPLX, K, G, EXACT, ALL>::lockstep) {
            if (!__syncthreads_or(has)) break;  // the block's warps take their terms in rounds
        } else {
            if (!__any_sync(FULL, has)) break;
        }
        if (has) {
            __syncwarp(gm);
            eval_term(prefac, mE, jidx);
            __syncwarp(gm);
        }
    }
    flush();
    // The block's groups summed in a fixed order: one partial per block.
    __shared__ dd red[2 * GB_MAX];
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
                if (!a.fused_out) {
                    // term output: nothing to sum
                } else if (CPLX) {
                    ((cd *)a.fused_out)[0] = cd{hr, __dadd_rn(fi.hi, fi.lo)};
                } else {
                    ((double *)a.fused_out)[0] = hr;
                }
            }
        }
    }
}

// Warps per block of a level kernel: the shape's, except that a lockstep block takes only as many
// warps as their workspaces fit in shared memory (the buffered series grow with the order n: the
// 17..20-row tiles keep their 20 warps up to n = 25, the 21..32-row tiles their 16 up to n = 26;
// at n = 32 the 20-row tile holds 17 warps and the 32-row tile 14).
template <bool CPLX, int K, int G, bool EXACT, bool ALL>
inline int level_warps(int nmax)
{
    using S = LevelShape<CPLX, K, G, EXACT, ALL>;
    constexpr int cw_max = S::threads / 32;
    if constexpr (!S::lockstep) {
        return cw_max;
    } else {
        const size_t per_warp = (size_t)(32 / G) * level_ws_doubles<CPLX, K, EXACT>(nmax) * sizeof(double);
        const int fit = (int)((size_t)(218 * 1024) / per_warp);
        return fit < 1 ? 1 : (fit < cw_max ? fit : cw_max);
    }
}

template <bool CPLX, int K, int G, bool EXACT = false>
static int level_launch_k(const SieveArgs &a, const int64_t *strides, int B, dd *partial, int blocks_x, cudaStream_t st)
{
    int cw = level_warps<CPLX, K, G, EXACT, false>(a.nmax);
    if (a.block_warps > 0 && a.block_warps < cw) cw = a.block_warps;  // the planner's smaller blocks
    const size_t smem = (size_t)cw * (32 / G) * level_ws_doubles<CPLX, K, EXACT>(a.nmax) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K, G, false, EXACT>;
    int rc = smem_limit_at_least((const void *)k, smem);
    if (rc) return rc;
    k<<<dim3((unsigned)blocks_x, (unsigned)B), cw * 32, smem, st>>>(a, strides, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int K, int G, bool EXACT = false>
static int level_launch_all_k(const SieveArgs &a, dd *partial, int blocks_x, cudaStream_t st)
{
    const int cw = level_warps<CPLX, K, G, EXACT, true>(a.nmax);
    const size_t smem = (size_t)cw * (32 / G) * level_ws_doubles<CPLX, K, EXACT>(a.nmax) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K, G, true, EXACT>;
    int rc = smem_limit_at_least((const void *)k, smem);
    if (rc) return rc;
    k<<<dim3((unsigned)blocks_x, 1u), cw * 32, smem, st>>>(a, nullptr, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int K, int G, bool EXACT = false, bool ALL = false>
static int level_shape_k(int nmax, int *warps_per_block, int *blocks_per_sm)
{
    const int cw = level_warps<CPLX, K, G, EXACT, ALL>(nmax);
    const size_t smem = (size_t)cw * (32 / G) * level_ws_doubles<CPLX, K, EXACT>(nmax) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K, G, ALL, EXACT>;
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
        return narrow ? level_launch_all_k<CPLX, K, level_group<K>(true), EXACT>(a, partial, blocks_x, st)  \
                      : level_launch_all_k<CPLX, K, 32, EXACT>(a, partial, blocks_x, st);
// Case K of a switch over the all-levels launches' shapes.
#define EGG_ALL_SHAPE(CPLX, K)                                                                         \
    case K:                                                                                            \
        rc = narrow ? level_shape_k<CPLX, K, level_group<K>(true), EXACT, true>(nmax, warps_per_block, blocks_per_sm) \
                    : level_shape_k<CPLX, K, 32, EXACT, true>(nmax, warps_per_block, blocks_per_sm);   \
        break;
#define EGG_FUSED_CASES(CPLX, X)                                                                    \
    X(CPLX, 1) X(CPLX, 2) X(CPLX, 3) X(CPLX, 4) X(CPLX, 5) X(CPLX, 6) X(CPLX, 7) X(CPLX, 8) X(CPLX, 9) \
    X(CPLX, 10)
#define EGG_LEVEL_CASES_HI(CPLX, X)                                                                 \
    X(CPLX, 17) X(CPLX, 18) X(CPLX, 19) X(CPLX, 20) X(CPLX, 21) X(CPLX, 22) X(CPLX, 23) X(CPLX, 24)
