// egg_dp_fixed.cuh -- closed-form DP levels with the popcount c a compile-time constant.
//
// The walk of a state (egg_dp.cu, walk_state) becomes straight-line code when c is known: every
// loop over the state's elements unrolls, the table offsets of each step are immediates, and
// there are no trip-count tests or predicated remainder steps.  That is most of the instructions
// of the runtime-c walk, which is issue-bound.  One instance (B == 1) only: for a batch the
// lanes of a warp share a state and the index work is already spread over the instances.
// Included by the egg_dp_fixed_*.cu files, which instantiate fixed_level per type.
#pragma once

#include <type_traits>

#include "egg_dp_common.cuh"

namespace egg {

// How the child level is read: kLoadPlain (the level kernels: the level was written by an earlier
// launch), kLoadL2 (through L2 only) or kLoadCA (weak loads cached in L1, for a level that other
// blocks of the same launch wrote before a grid-wide barrier; see ld_ca).
constexpr int kLoadPlain = 0, kLoadL2 = 1, kLoadCA = 2;
template <int C, class Op, class M, class PT, class HT, class AT, int LOAD = kLoadPlain>
__device__ __forceinline__ AT walk_fixed(M m, const uint2 *__restrict__ TP, int K, int m0, const PT *__restrict__ Ps,
                                         const HT *__restrict__ Hprev)
{
    static_assert(C >= 4 && C % 2 == 0, "levels c >= 4");
    constexpr int ld = C + 1;
    const int e1 = low_bit<M>(m);
    m &= m - 1;
    const int e2 = low_bit<M>(m);
    M r = m & (m - 1);
    uint32_t suf = 0;  // suf_2 = sum_{x=3}^{C} C(e_x - 1, x - 2)
#pragma unroll
    for (int x = 3; x <= C; ++x) {
        const int e = low_bit<M>(r);
        r &= r - 1;
        suf += TP[(e - 1) * ld + (x - 2)].x;
    }
    // Pairs of the minimum e1: 0-based _pair_index(e1 + m0 + 1, ej + m0 + 1, K) - 1 = row + ej.
    const int ib = e1 + m0 + 1;
    const PT *Prow = Ps + ((ib - 1) * K - (ib * (ib + 1)) / 2 + m0);
    uint32_t pre = 0;
    uint32_t padd = TP[(e2 - 1) * ld].y;  // C(e2 - 1, 1)
    int ej = e2;
    r = m & (m - 1);
    AT acc = zero_of<AT>();
#pragma unroll
    for (int x0 = 2; x0 <= C; x0 += kBatch) {
        HT hv[kBatch];
        PT pv[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int x = x0 + u;
            if (x <= C) {
                if constexpr (LOAD == kLoadL2) hv[u] = ld_l2(Hprev + pre + suf);
                else if constexpr (LOAD == kLoadCA) hv[u] = ld_ca(Hprev + pre + suf);
                else hv[u] = Hprev[pre + suf];
                pv[u] = Prow[ej];
                pre += padd;
                if (x < C) {
                    const int en = low_bit<M>(r);
                    r &= r - 1;
                    const uint2 t = TP[(en - 1) * ld + (x - 1)];
                    suf -= t.x;
                    padd = t.y;
                    ej = en;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (x0 + u <= C) acc = madd(Op{}, acc, pv[u], hv[u]);
    }
    return acc;
}

// Same phases as dpc_level_kernel with B == 1 (masks of `run` consecutive states per thread, then
// one state per thread and step), with walk_fixed<C>.  blockIdx.y selects one of several
// independent instances stored instance-major: pairs at P + y * ldp, the level read at
// Hprev + y * ldhp and the level written at Hcur + y * ldhc.
// Blocks of kLevelThreads per SM the level kernel is compiled for.  The child gathers are latency
// bound (long-scoreboard stalls dominate), so more resident warps help, as long as the walk's
// registers still fit: 4 blocks (64 registers) through c = 14, 3 (80) through c = 24, 2 (128)
// through c = 38.  Int128 states, and the 64-bit-mask levels from c = 40, spill under those caps and
// keep the compiler's own allocation.  Measured on the 4096 mix 45.5 -> 42.9 ms, N = 40 FP64
// 3.46 -> 3.33 ms, N = 36 complex 0.83 -> 0.79 ms.
template <int C, class HT>
constexpr int fixed_min_blocks()
{
    if (std::is_same<HT, __int128>::value) return 1;
    return C <= 14 ? 4 : (C <= 24 ? 3 : (C <= 38 ? 2 : 1));
}

template <int C, class Op, class M, class PT, class HT, class AT>
__global__ void __launch_bounds__(kLevelThreads, (fixed_min_blocks<C, HT>())) dpc_fixed_kernel(const uint32_t *__restrict__ binom, const PT *__restrict__ P,
                                                                  const HT *__restrict__ Hprev, HT *__restrict__ Hcur, int K,
                                                                  int64_t n, int run, int64_t ldp, int64_t ldhp, int64_t ldhc)
{
    P += blockIdx.y * ldp;
    Hprev += blockIdx.y * ldhp;
    Hcur += blockIdx.y * ldhc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int ld = C + 1;
    const int m0 = (K - C) / 2, U = K - m0;
    M *masks = reinterpret_cast<M *>(smem_raw);
    uint2 *TP = reinterpret_cast<uint2 *>(smem_raw + (size_t)kRun * kLevelThreads * sizeof(M));
    PT *Ps = reinterpret_cast<PT *>(smem_raw + level_pairs_offset<M>(U, ld));
    fill_pair_table(TP, binom, U, ld, threadIdx.x, kLevelThreads);
    const int npairs = K * (K - 1) / 2;
    for (int q = threadIdx.x; q < npairs; q += kLevelThreads) Ps[q] = P[q];
    __syncthreads();
    const int64_t chunk = (int64_t)run * kLevelThreads;
    for (int64_t s0 = blockIdx.x * chunk; s0 < n; s0 += (int64_t)gridDim.x * chunk) {
        const int cnt = (int)(n - s0 < chunk ? n - s0 : chunk);
        const int r0 = threadIdx.x * run;
        if (r0 < cnt) {
            M m = colex_unrank<M>(TP, ld, U, C, (uint32_t)(s0 + r0));
            masks[r0] = m;
            for (int r = 1; r < run && r0 + r < cnt; ++r) {
                m = colex_next<M>(m);
                masks[r0 + r] = m;
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += kLevelThreads)
            store(Hcur[s0 + i], walk_fixed<C, Op, M, PT, HT, AT>(masks[i], TP, K, m0, Ps, Hprev));
        __syncthreads();
    }
}

template <int C, class Op, class M, class PT, class HT, class AT>
static bool launch_fixed(const uint32_t *binom, const PT *P, const HT *prev, HT *cur, int K, int64_t n, int run, int blocks,
                         int G, int64_t ldp, int64_t ldhp, int64_t ldhc, cudaStream_t st)
{
    auto k = dpc_fixed_kernel<C, Op, M, PT, HT, AT>;
    static bool attr_set = false;  // per instantiation; callers hold the library's lock
    if (!attr_set) {
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024) != cudaSuccess) return false;
        attr_set = true;
    }
    const int U = (K + C) / 2;
    const size_t sm = level_pairs_offset<M>(U, C + 1) + (size_t)K * (K - 1) / 2 * sizeof(PT);
    k<<<dim3((unsigned)blocks, (unsigned)G), kLevelThreads, sm, st>>>(binom, P, prev, cur, K, n, run, ldp, ldhp, ldhc);
    count_launch();
    return true;
}

#define EGG_FIXED_CASE(CC, MT) \
    case CC: return launch_fixed<CC, Op, MT, PT, HT, AT>(binom, P, prev, cur, K, n, run, blocks, G, ldp, ldhp, ldhc, st);

// 32-bit masks for levels whose positions fit (U <= 32, c <= 32); 64-bit masks for c = 26..46.
template <class Op, class PT, class HT, class AT>
bool fixed_level(const uint32_t *binom, const PT *P, const HT *prev, HT *cur, int K, int c, int64_t n, int run, int blocks,
                 int G, int64_t ldp, int64_t ldhp, int64_t ldhc, cudaStream_t st)
{
    const int U = (K + c) / 2;
    if (U <= 32) {
        switch (c) {
            EGG_FIXED_CASE(4, uint32_t) EGG_FIXED_CASE(6, uint32_t) EGG_FIXED_CASE(8, uint32_t)
            EGG_FIXED_CASE(10, uint32_t) EGG_FIXED_CASE(12, uint32_t) EGG_FIXED_CASE(14, uint32_t)
            EGG_FIXED_CASE(16, uint32_t) EGG_FIXED_CASE(18, uint32_t) EGG_FIXED_CASE(20, uint32_t)
            EGG_FIXED_CASE(22, uint32_t) EGG_FIXED_CASE(24, uint32_t) EGG_FIXED_CASE(26, uint32_t)
            EGG_FIXED_CASE(28, uint32_t) EGG_FIXED_CASE(30, uint32_t) EGG_FIXED_CASE(32, uint32_t)
        default: return false;
        }
    }
    switch (c) {
        EGG_FIXED_CASE(26, uint64_t) EGG_FIXED_CASE(28, uint64_t) EGG_FIXED_CASE(30, uint64_t)
        EGG_FIXED_CASE(32, uint64_t) EGG_FIXED_CASE(34, uint64_t) EGG_FIXED_CASE(36, uint64_t)
        EGG_FIXED_CASE(38, uint64_t) EGG_FIXED_CASE(40, uint64_t) EGG_FIXED_CASE(42, uint64_t)
        EGG_FIXED_CASE(44, uint64_t) EGG_FIXED_CASE(46, uint64_t)
    default: return false;
    }
}

#undef EGG_FIXED_CASE

#define EGG_INSTANTIATE_FIXED(OP, PT, HT, AT)                                                                         \
    template bool fixed_level<OP, PT, HT, AT>(const uint32_t *, const PT *, const HT *, HT *, int, int, int64_t, int, int, \
                                              int, int64_t, int64_t, int64_t, cudaStream_t);

}  // namespace egg
