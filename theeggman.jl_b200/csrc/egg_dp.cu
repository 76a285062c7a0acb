// egg_dp.cu -- the subset DP (src/dp.jl:344-363 _dp_states!, :408-442 _haf_dp) on the device.
//
// Layout in HBM.  State values live in two ping-pong buffers, each sized for the largest level:
// every transition out of a level lands in the level immediately below (two subset sizes down,
// src/dp.jl:146-148), so level L only ever reads level L-1 and the full `H` of the reference
// (1.3 GB at K = 40 in FP64) is never materialised.  Within a buffer values are instance-fastest,
// (state - level_lo) * B + b, the reference device layout (ext/TheEggmanKernelAbstractionsExt.jl:
// 13-20, :56-62) restricted to one level.
//
// Plans.  The plan of _build_dp_plan has a closed form (egg_plan.cu), so a resident plan of that
// layout is evaluated without its transition array: each thread derives its state's children from
// the state's rank (dpc_* kernels below).  At K = 40 that removes 22.7 GB of reads per evaluation.
// An uploaded plan that differs from that layout keeps its array and runs through the dp_* kernels
// that read it.
//
// Arithmetic.  Each state is accumulated by one thread in plan order, as the reference does.
// EGG_PREC_EXACT rounds every product and sum separately (__dmul_rn/__dadd_rn), which is how Julia
// evaluates the CPU loop, so results are bit-identical to the reference's _haf_dp.  EGG_PREC_FMA
// contracts each multiply-add as the reference's GPU kernel does.  EGG_PREC_MIXED multiplies in
// FP32 and accumulates each state in FP64.  Integer inputs run exactly in Int128.
#include <cooperative_groups.h>
#include <cstring>
#include <map>
#include <type_traits>
#include <utility>

#include "egg_dp_common.cuh"

namespace cg = cooperative_groups;

namespace egg {

// One level: states [0, n) of the level, out-degree deg, transitions from toff.  Hprev holds
// level L-1 (child numbers are 1-based global, child_lo1 = first state of L-1, 1-based).
template <class Op, class I, class PT, class HT, class AT, bool B1>
__global__ void __launch_bounds__(256) dp_level_kernel(const I *__restrict__ trans, const PT *__restrict__ P,
                                                       const HT *__restrict__ Hprev, HT *__restrict__ Hcur, int64_t n,
                                                       int deg, int64_t toff, int64_t child_lo1, int64_t B, int bits)
{
    const int64_t total = n * B;
    const I mask = ((I)1 << bits) - 1;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        int64_t s, b;
        if (B1) {
            s = g;
            b = 0;
        } else {
            s = g / B;
            b = g - s * B;
        }
        const I *tr = trans + toff + s * deg;
        AT acc = zero_of<AT>();
        for (int k0 = 0; k0 < deg; k0 += kBatch) {
            I tv[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                if (k0 + u < deg) tv[u] = __ldg(tr + k0 + u);
            PT pv[kBatch];
            HT hv[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                if (k0 + u < deg) {
                    const int64_t pi = (int64_t)(tv[u] & mask) - 1;
                    const int64_t ci = (int64_t)(tv[u] >> bits) - child_lo1;
                    pv[u] = P[pi * B + b];
                    hv[u] = Hprev[ci * B + b];
                }
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                if (k0 + u < deg) acc = madd(Op{}, acc, pv[u], hv[u]);
        }
        store(Hcur[s * B + b], acc);
    }
}

// Whole instances in one launch, for degrees whose two largest adjacent levels fit in shared
// memory (N <= 22 in FP64): one CTA per instance (grid-strided over the batch), the level loop
// inside the kernel with a barrier between levels, both level buffers and the instance's pairs in
// shared memory, the plan streamed from global memory (it is L2-resident at these sizes, 0.36 MB
// at N = 20).  Same per-state arithmetic and order as dp_level_kernel.
static constexpr int kSmallMaxDeg = 23;  // out-degree |S|-1 of the largest level handled (N <= 24)

struct SmallLevels {
    int64_t toff[33];
    int n[33];
    int deg[33];
    int nlev;
};

template <class Op, class I, class PT, class HT, class AT>
__global__ void __launch_bounds__(512) dp_small_kernel(const I *__restrict__ trans, SmallLevels lv, const PT *__restrict__ P,
                                                       HT *__restrict__ out, int64_t B, int npairs, int maxlev, int bits)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HT *H0 = reinterpret_cast<HT *>(smem_raw);
    HT *H1 = H0 + maxlev;
    PT *Ps = reinterpret_cast<PT *>(H1 + maxlev);
    const I mask = ((I)1 << bits) - 1;
    for (int64_t b = blockIdx.x; b < B; b += gridDim.x) {
        for (int q = threadIdx.x; q < npairs; q += blockDim.x) Ps[q] = P[(int64_t)q * B + b];
        if (threadIdx.x == 0) H0[0] = one_of<HT>();
        __syncthreads();
        int64_t child_lo1 = 1;  // first state of the previous level, 1-based
        int64_t lo1 = 2;        // first state of the current level, 1-based
        for (int L = 1; L < lv.nlev; ++L) {
            const HT *prev = (L & 1) ? H0 : H1;
            HT *cur = (L & 1) ? H1 : H0;
            const int n = lv.n[L], deg = lv.deg[L];
            const I *tl = trans + lv.toff[L];
            for (int s = threadIdx.x; s < n; s += blockDim.x) {
                // Issue all of this state's transition loads before using any (one L2 round trip),
                // then accumulate in plan order.
                const I *tr = tl + (int64_t)s * deg;
                I tv[kSmallMaxDeg];
#pragma unroll
                for (int k = 0; k < kSmallMaxDeg; ++k)
                    if (k < deg) tv[k] = __ldg(tr + k);
                AT acc = zero_of<AT>();
#pragma unroll
                for (int k = 0; k < kSmallMaxDeg; ++k)
                    if (k < deg) acc = madd(Op{}, acc, Ps[(int)(tv[k] & mask) - 1], prev[(int64_t)(tv[k] >> bits) - child_lo1]);
                store(cur[s], acc);
            }
            __syncthreads();
            child_lo1 = lo1;
            lo1 += n;
        }
        if (threadIdx.x == 0) out[b] = ((lv.nlev - 1) & 1) ? H1[0] : H0[0];
        __syncthreads();
    }
}

// ---- closed-form plans ---------------------------------------------------------------------------
//
// A plan with the layout of _build_dp_plan (src/dp.jl:223-304) needs no transition array.  Level c
// (popcount c) is every c-subset of the top U = K - m0 positions (m0 = (K - c) / 2), numbered in
// colex order, which is increasing mask order.  A state S with shifted elements e1 < ... < ec has
// out-degree c - 1; its j-th transition (j = 2..c, the order of the plan) pairs e1 with ej and
// lands on S - {e1, ej}, whose rank in the level below is
//     pre_j + suf_j,  pre_j = sum_{x=2}^{j-1} C(e_x - 1, x - 1),  suf_j = sum_{x=j+1}^{c} C(e_x - 1, x - 2).
// Both sums are carried along the walk.  A table entry holds C(x, k) and C(x, k + 1) side by side,
// so stepping to the next element takes one 8-byte shared-memory load: its C(e - 1, j - 1) leaves
// suf now and its C(e - 1, j) joins pre one step later.  The arithmetic per state is that of the
// plan kernels, in the same order, so results are identical.

// One step of the walk: load the child value and pair value for element ej, then advance
// pre/suf/ej to the next element (if this is not the last step).  L2ONLY reads the child level
// through L2 only.
template <class M, class PT, class HT, bool B1, bool L2ONLY = false>
__device__ __forceinline__ void walk_step(int x, int c, M &rest, uint32_t &pre, uint32_t &suf, uint32_t &padd, int &ej,
                                          const uint2 *TP, int ld, int pb, const PT *P, const HT *Hprev, int64_t B,
                                          int64_t b, HT &h, PT &p)
{
    const uint32_t child = pre + suf;
    if (L2ONLY) {
        h = ld_l2(Hprev + (B1 ? (int64_t)child : (int64_t)child * B + b));
        p = B1 ? P[pb + ej] : P[(int64_t)(pb + ej) * B + b];
    } else if (B1) {
        h = Hprev[child];
        p = P[pb + ej];
    } else {
        h = Hprev[(int64_t)child * B + b];
        p = P[(int64_t)(pb + ej) * B + b];
    }
    pre += padd;
    if (x < c) {
        const int en = low_bit<M>(rest);
        rest &= rest - 1;
        const uint2 t = TP[(en - 1) * ld + (x - 1)];
        suf -= t.x;
        padd = t.y;
        ej = en;
    }
}

// One state's value (c >= 4): the sum over its transitions, in plan order, of P[pair] * H[child]
// (instance b of B, instance-fastest; B1 when B == 1).  The loads of kBatch transitions are issued
// before any of them is used, so a state waits for one memory round trip per batch rather than one
// per transition; the accumulation order is unchanged.
template <class Op, class M, class PT, class HT, class AT, bool B1, bool L2ONLY = false>
__device__ __forceinline__ AT walk_state(M m, const uint2 *TP, int ld, int c, int K, int m0, const PT *P,
                                         const HT *Hprev, int64_t B, int64_t b)
{
    const int e1 = low_bit<M>(m);
    M rest = m & (m - 1);
    const int e2 = low_bit<M>(rest);
    rest &= rest - 1;  // e3..ec
    uint32_t suf = 0;  // suf_2 = sum_{x=3}^{c} C(e_x - 1, x - 2)
    {
        M r = rest;
        int x = 3;
        for (; x + 3 <= c; x += 4) {
            const int ea = low_bit<M>(r);
            r &= r - 1;
            const int eb = low_bit<M>(r);
            r &= r - 1;
            const int ecc = low_bit<M>(r);
            r &= r - 1;
            const int ed = low_bit<M>(r);
            r &= r - 1;
            suf += TP[(ea - 1) * ld + (x - 2)].x + TP[(eb - 1) * ld + (x - 1)].x + TP[(ecc - 1) * ld + x].x +
                   TP[(ed - 1) * ld + (x + 1)].x;
        }
        for (; x <= c; ++x) {
            const int e = low_bit<M>(r);
            r &= r - 1;
            suf += TP[(e - 1) * ld + (x - 2)].x;
        }
    }
    // 0-based _pair_index(e1 + m0 + 1, ej + m0 + 1, K) - 1 = pb + ej (src/unrolled.jl:60).
    const int ib = e1 + m0 + 1;
    const int pb = (ib - 1) * K - (ib * (ib + 1)) / 2 + m0;
    uint32_t pre = 0;
    uint32_t padd = TP[(e2 - 1) * ld].y;  // C(e2 - 1, 1): joins pre after the first step
    int ej = e2;
    AT acc = zero_of<AT>();
    int x = 2;
    for (; x + kBatch - 1 <= c; x += kBatch) {
        HT hv[kBatch];
        PT pv[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            walk_step<M, PT, HT, B1, L2ONLY>(x + u, c, rest, pre, suf, padd, ej, TP, ld, pb, P, Hprev, B, b, hv[u], pv[u]);
#pragma unroll
        for (int u = 0; u < kBatch; ++u) acc = madd(Op{}, acc, pv[u], hv[u]);
    }
    if (x <= c) {
        HT hv[kBatch];
        PT pv[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (x + u <= c)
                walk_step<M, PT, HT, B1, L2ONLY>(x + u, c, rest, pre, suf, padd, ej, TP, ld, pb, P, Hprev, B, b, hv[u], pv[u]);
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (x + u <= c) acc = madd(Op{}, acc, pv[u], hv[u]);
    }
    return acc;
}

template <class Op, class PT, class HT, class AT>
__global__ void __launch_bounds__(256) dpc_first_kernel(const PT *__restrict__ P, HT *__restrict__ Hcur, int K, int64_t n,
                                                        int64_t B)
{
    const int64_t total = n * B;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = g / B, b = g - s * B;
        Hcur[g] = first_level_value<Op, PT, HT, AT>(s, K, P, B, b);
    }
}

// One level (c >= 4) of a closed-form plan, for levels without a fixed-popcount kernel
// (egg_dp_fixed.cuh): the same two phases with the popcount a runtime value.
template <class Op, class M, class PT, class HT, class AT, bool B1>
__global__ void __launch_bounds__(kLevelThreads) dpc_level_kernel(const uint32_t *__restrict__ binom, const PT *__restrict__ P,
                                                                  const HT *__restrict__ Hprev, HT *__restrict__ Hcur,
                                                                  int K, int c, int64_t n, int64_t B, int run)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int m0 = (K - c) / 2, U = K - m0, ld = c + 1;
    M *masks = reinterpret_cast<M *>(smem_raw);
    uint2 *TP = reinterpret_cast<uint2 *>(smem_raw + (size_t)kRun * kLevelThreads * sizeof(M));
    PT *Ps = reinterpret_cast<PT *>(smem_raw + level_pairs_offset<M>(U, ld));
    fill_pair_table(TP, binom, U, ld, threadIdx.x, kLevelThreads);
    const int npairs = K * (K - 1) / 2;
    if (B1)
        for (int q = threadIdx.x; q < npairs; q += kLevelThreads) Ps[q] = P[q];
    __syncthreads();
    const PT *Pp = B1 ? Ps : P;
    // States per chunk: run * 256 for one instance, fewer for a batch (about that many pairs).
    const int64_t chunk = B1 ? (int64_t)run * kLevelThreads
                             : (B >= (int64_t)run * kLevelThreads ? 1 : ((int64_t)run * kLevelThreads) / B);
    for (int64_t s0 = blockIdx.x * chunk; s0 < n; s0 += (int64_t)gridDim.x * chunk) {
        const int cnt = (int)(n - s0 < chunk ? n - s0 : chunk);
        const int r0 = threadIdx.x * run;
        if (r0 < cnt) {
            M m = colex_unrank<M>(TP, ld, U, c, (uint32_t)(s0 + r0));
            masks[r0] = m;
            for (int r = 1; r < run && r0 + r < cnt; ++r) {
                m = colex_next<M>(m);
                masks[r0 + r] = m;
            }
        }
        __syncthreads();
        const int64_t items = (int64_t)cnt * B;
        for (int64_t i = threadIdx.x; i < items; i += kLevelThreads) {
            int sl;
            int64_t b;
            if (B1) {
                sl = (int)i;
                b = 0;
            } else {
                sl = (int)(i / B);
                b = i - (int64_t)sl * B;
            }
            const AT acc = walk_state<Op, M, PT, HT, AT, B1>(masks[sl], TP, ld, c, K, m0, Pp, Hprev, B, b);
            store(Hcur[(s0 + sl) * B + b], acc);
        }
        __syncthreads();
    }
}

// One state of a deep level evaluated by a whole warp (the levels near the top of a plan hold few
// states with long transition lists, so a state per thread is one long dependent chain).
//   * Unrank by complement: complementing reverses colex order, so state s of the c-subsets of U
//     positions is the complement of the (U-c)-subset of rank C(U,c)-1-s.  Near the top U - c is
//     small, and each of its elements is found by one ballot over candidate positions.
//   * Lane l owns positions l and l+32.  Element x (1-based, x >= 2) at position e contributes
//     a_x = C(e-1, x-1) to the child ranks of later elements and b_x = C(e-1, x-2) to earlier ones,
//     so warp scans give every child rank pre_j + suf_j at once and all loads go out together.
//   * Lane 0 then sums the transitions in plan order from shared memory (the same madd sequence as
//     a thread walking the state, so the same bits).
template <class Op, class PT, class HT, class AT>
__device__ __forceinline__ void wide_state(uint32_t srank, int c, int K, const uint2 *TP, int ld, const PT *Ps, const HT *prev,
                                           HT *cur, PT *pbuf, HT *hbuf, int lane)
{
    const int m0 = (K - c) / 2, U = K - m0, k = U - c;
    // Complement of rank C(U,c)-1-s among k-subsets, element by element from the largest.
    uint32_t R = TP[U * ld + c].x - 1u - srank;
    uint64_t comp = 0;
    int xprev = U;
    for (int i = k; i >= 1; --i) {
        int x = -1;
        for (int base = xprev - 1; x < 0; base -= 32) {
            const int cand = base - lane;
            const bool ok = cand < 0 || TP[cand * ld + i].x <= R;  // C(cand, i) is nondecreasing in cand
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (bal) x = base - (__ffs(bal) - 1);
        }
        x = x < 0 ? 0 : x;
        comp |= (uint64_t)1 << x;
        R -= TP[x * ld + i].x;
        xprev = x;
    }
    const uint64_t all = U >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << U) - 1);
    const uint64_t mask = all & ~comp;
    const int e1 = __ffsll((long long)mask) - 1;
    // Positions p0 = lane, p1 = lane + 32: element index, contributions.
    uint32_t a0 = 0, b0 = 0, a1 = 0, b1 = 0;
    int x0 = 0, x1 = 0;
    const int p0 = lane, p1 = lane + 32;
    if (p0 < U && ((mask >> p0) & 1)) {
        x0 = __popcll(mask & (((uint64_t)1 << p0) - 1)) + 1;
        if (x0 >= 2) {
            const uint2 t = TP[(p0 - 1) * ld + (x0 - 2)];
            b0 = t.x;
            a0 = t.y;
        }
    }
    if (p1 < U && ((mask >> p1) & 1)) {
        x1 = __popcll(mask & (((uint64_t)1 << p1) - 1)) + 1;
        if (x1 >= 2) {
            const uint2 t = TP[(p1 - 1) * ld + (x1 - 2)];
            b1 = t.x;
            a1 = t.y;
        }
    }
    // Inclusive scans over positions 0..63 (low half in lanes, then the high half).
    uint32_t sa0 = a0, sb0 = b0, sa1 = a1, sb1 = b1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t ta0 = __shfl_up_sync(0xffffffffu, sa0, o), tb0 = __shfl_up_sync(0xffffffffu, sb0, o);
        const uint32_t ta1 = __shfl_up_sync(0xffffffffu, sa1, o), tb1 = __shfl_up_sync(0xffffffffu, sb1, o);
        if (lane >= o) {
            sa0 += ta0;
            sb0 += tb0;
            sa1 += ta1;
            sb1 += tb1;
        }
    }
    const uint32_t lowa = __shfl_sync(0xffffffffu, sa0, 31), lowb = __shfl_sync(0xffffffffu, sb0, 31);
    const uint32_t totb = lowb + __shfl_sync(0xffffffffu, sb1, 31);
    sa1 += lowa;
    sb1 += lowb;
    const int ib = e1 + m0 + 1;
    const int pb = (ib - 1) * K - (ib * (ib + 1)) / 2 + m0;
    // pre_j = sum of a over earlier elements (exclusive), suf_j = sum of b over later ones.
    if (x0 >= 2) {
        const uint32_t child = (sa0 - a0) + (totb - sb0);
        pbuf[x0 - 2] = Ps[pb + p0];
        hbuf[x0 - 2] = ld_l2(prev + child);
    }
    if (x1 >= 2) {
        const uint32_t child = (sa1 - a1) + (totb - sb1);
        pbuf[x1 - 2] = Ps[pb + p1];
        hbuf[x1 - 2] = ld_l2(prev + child);
    }
    __syncwarp();
    if (lane == 0) {
        AT acc = zero_of<AT>();
        for (int j = 0; j < c - 1; ++j) acc = madd(Op{}, acc, pbuf[j], hbuf[j]);
        store(cur[srank], acc);
    }
    __syncwarp();
}

// Levels at or above this popcount run a warp per state inside a span launch.
static constexpr int kWideMinC = 14;

// Several consecutive small levels of one instance in one cooperative launch: the levels at either
// end of a plan hold few states each, so a launch per level costs mostly its fixed overhead (the
// table fill, the pairs and the launch itself).  Here the table is filled once, a grid-wide
// barrier separates the levels, and the previous level is read through L2 (the ping-pong buffers
// are rewritten within the launch).  Shallow levels run a thread per state, deep ones a warp per
// state (wide_state); both keep the level kernels' arithmetic and order.
template <class Op, class PT, class HT, class AT>
__global__ void __launch_bounds__(256) dpc_span_kernel(const uint32_t *__restrict__ binom, const PT *__restrict__ P, HT *H0,
                                                       HT *H1, HT *out, int K, int L0, int L1, int out_last)
{
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ld = K + 2;  // columns 0..K+1, so every C(x, k + 1) the walk reads is in the table
    uint2 *TP = reinterpret_cast<uint2 *>(smem_raw);
    PT *Ps = reinterpret_cast<PT *>(smem_raw + (((size_t)(K + 1) * ld * sizeof(uint2) + 15) / 16) * 16);
    const int npairs = K * (K - 1) / 2;
    unsigned char *wbuf = reinterpret_cast<unsigned char *>(Ps) + (((size_t)npairs * sizeof(PT) + 15) / 16) * 16;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    HT *hbuf = reinterpret_cast<HT *>(wbuf) + wid * 64;
    PT *pbuf = reinterpret_cast<PT *>(wbuf + (size_t)(blockDim.x / 32) * 64 * sizeof(HT)) + wid * 64;
    fill_pair_table(TP, binom, K + 1, ld, threadIdx.x, blockDim.x);
    for (int q = threadIdx.x; q < npairs; q += blockDim.x) Ps[q] = P[q];
    __syncthreads();
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nwarps = nth / 32, gwarp = tid / 32;
    for (int L = L0; L <= L1; ++L) {
        const int c = 2 * L, m0 = (K - c) / 2, U = K - m0;
        const int64_t n = TP[U * ld + c].x;
        HT *cur = (L == L1 && out_last) ? out : ((L & 1) ? H1 : H0);
        const HT *prev = (L & 1) ? H0 : H1;
        if (c >= kWideMinC) {
            for (int64_t s = gwarp; s < n; s += nwarps) wide_state<Op, PT, HT, AT>((uint32_t)s, c, K, TP, ld, Ps, prev, cur, pbuf, hbuf, lane);
        } else {
            for (int64_t s = tid; s < n; s += nth) {
                HT v;
                if (c == 2) {
                    v = first_level_value<Op, PT, HT, AT>(s, K, Ps, 1, 0);
                } else {
                    const uint64_t m = colex_unrank<uint64_t>(TP, ld, U, c, (uint32_t)s);
                    store(v, walk_state<Op, uint64_t, PT, HT, AT, true, true>(m, TP, ld, c, K, m0, Ps, prev, 1, 0));
                }
                cur[s] = v;
            }
        }
        if (L < L1) grid.sync();
    }
}

// Whole instances of a closed-form plan in one launch (degrees whose two largest levels fit in
// shared memory): one CTA per instance, the level loop inside the kernel.  Each thread takes a
// run of consecutive states of a level (one unrank, then successors) and walks each in turn.
template <class Op, class PT, class HT, class AT, int MAXT>
__global__ void __launch_bounds__(MAXT) dpc_small_kernel(const uint32_t *__restrict__ binom, const PT *__restrict__ P,
                                                         HT *__restrict__ out, int64_t B, int K, int maxlev)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HT *H0 = reinterpret_cast<HT *>(smem_raw);
    HT *H1 = H0 + maxlev;
    PT *Ps = reinterpret_cast<PT *>(H1 + maxlev);
    const int npairs = K * (K - 1) / 2;
    const int ld = K + 1;
    uint2 *TP = reinterpret_cast<uint2 *>(smem_raw + (((size_t)2 * maxlev * sizeof(HT) + (size_t)npairs * sizeof(PT) + 15) / 16) * 16);
    fill_pair_table(TP, binom, ld, ld, threadIdx.x, blockDim.x);
    for (int64_t b = blockIdx.x; b < B; b += gridDim.x) {
        for (int q = threadIdx.x; q < npairs; q += blockDim.x) Ps[q] = P[(int64_t)q * B + b];
        __syncthreads();
        {
            const int n = (K / 2 + 1) * (K / 2) / 2;  // level c = 2
            for (int s = threadIdx.x; s < n; s += blockDim.x) H1[s] = first_level_value<Op, PT, HT, AT>(s, K, Ps, 1, 0);
        }
        __syncthreads();
        for (int c = 4; c <= K; c += 2) {
            const HT *prev = ((c / 2) & 1) ? H0 : H1;
            HT *cur = ((c / 2) & 1) ? H1 : H0;
            const int m0 = (K - c) / 2, U = K - m0;
            const int n = (int)TP[U * ld + c].x;
            const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
            const int r0 = threadIdx.x * per;
            if (r0 < n) {
                uint32_t m = colex_unrank<uint32_t>(TP, ld, U, c, (uint32_t)r0);
                for (int r = 0; r < per && r0 + r < n; ++r) {
                    if (r) m = colex_next<uint32_t>(m);
                    store(cur[r0 + r], walk_state<Op, uint32_t, PT, HT, AT, true>(m, TP, ld, c, K, m0, Ps, prev, 1, 0));
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) out[b] = ((K / 2) & 1) ? H1[0] : H0[0];
        __syncthreads();
    }
}

// Largest degree and cluster size of the one-instance cluster kernel (a level's states fit in 13
// bits beside an 8-bit pair index up to K = 22).
static constexpr int kClusterMaxK = 22;
static constexpr int kClusterMaxLevels = kClusterMaxK / 2 + 1;
static constexpr int kClusterMaxPairs = kClusterMaxK * (kClusterMaxK - 1) / 2;

// The pairs of a one-instance cluster launch: in device memory (ptr), or, for a call from host
// memory, carried in the launch's own parameters (ptr null), so no copy precedes the launch.  At most
// 231 pairs of 16 bytes, within the 4 KB of kernel parameters.
template <class PT>
struct ClusterPairs {
    const PT *ptr;
    PT v[kClusterMaxPairs];
};

// One state's transitions as (child << 8) | pair, in plan order: walk_state's index arithmetic
// without the loads.
template <class M>
__device__ __forceinline__ void list_state(M m, const uint2 *TP, int ld, int c, int K, int m0, uint32_t *ent)
{
    const int e1 = low_bit<M>(m);
    M rest = m & (m - 1);
    const int e2 = low_bit<M>(rest);
    rest &= rest - 1;
    uint32_t suf = 0;
    {
        M r = rest;
        for (int x = 3; x <= c; ++x) {
            const int e = low_bit<M>(r);
            r &= r - 1;
            suf += TP[(e - 1) * ld + (x - 2)].x;
        }
    }
    const int ib = e1 + m0 + 1;
    const int pb = (ib - 1) * K - (ib * (ib + 1)) / 2 + m0;
    uint32_t pre = 0, padd = TP[(e2 - 1) * ld].y;
    int ej = e2;
    for (int x = 2; x <= c; ++x) {
        ent[x - 2] = ((pre + suf) << 8) | (uint32_t)(pb + ej);
        pre += padd;
        if (x < c) {
            const int en = low_bit<M>(rest);
            rest &= rest - 1;
            const uint2 t = TP[(en - 1) * ld + (x - 1)];
            suf -= t.x;
            padd = t.y;
            ej = en;
        }
    }
}

// CTA `rank`'s share of a closed-form plan in an nr-CTA cluster: its states of level L (c = 2L >= 4)
// are s = rank + nr j, j < cnt(L); unit_lo[L] numbers them level after level and ent_lo[L] their
// transition entries (c - 1 per state).  Entries [2, nlev] are set.
__device__ __forceinline__ void cluster_layout(const uint2 *TP, int ld, int K, int nr, int rank, int *unit_lo, int *ent_lo)
{
    const int nlev = K / 2 + 1;
    int u = 0, e = 0;
    for (int L = 2; L < nlev; ++L) {
        const int c = 2 * L, U = K - (K - c) / 2;
        const int n = (int)TP[U * ld + c].x;
        const int cnt = n > rank ? (n - 1 - rank) / nr + 1 : 0;
        unit_lo[L] = u;
        ent_lo[L] = e;
        u += cnt;
        e += cnt * (c - 1);
    }
    unit_lo[nlev] = u;
    ent_lo[nlev] = e;
}

// The transition lists of dpc_cluster_kernel for one degree and cluster size, built once and kept
// with the plan: CTA r's list is ent[r * stride ...].  blockIdx.x is the CTA, blockIdx.y a slice of
// its states.
__global__ void __launch_bounds__(256) cluster_list_kernel(const uint32_t *__restrict__ binom, uint32_t *ent, int64_t stride,
                                                           int K, int nr)
{
    __shared__ uint2 TP[(kClusterMaxK + 1) * (kClusterMaxK + 1)];
    __shared__ int unit_lo[kClusterMaxLevels + 1], ent_lo[kClusterMaxLevels + 1];
    const int ld = K + 1, rank = blockIdx.x, nlev = K / 2 + 1;
    fill_pair_table(TP, binom, ld, ld, threadIdx.x, blockDim.x);
    __syncthreads();
    if (threadIdx.x == 0) cluster_layout(TP, ld, K, nr, rank, unit_lo, ent_lo);
    __syncthreads();
    uint32_t *mine = ent + (int64_t)rank * stride;
    for (int u = blockIdx.y * blockDim.x + threadIdx.x; u < unit_lo[nlev]; u += gridDim.y * blockDim.x) {
        int L = 2;
        while (u >= unit_lo[L + 1]) ++L;
        const int c = 2 * L, m0 = (K - c) / 2, U = K - m0;
        const int j = u - unit_lo[L];
        const uint32_t m = colex_unrank<uint32_t>(TP, ld, U, c, (uint32_t)(rank + nr * j));
        list_state<uint32_t>(m, TP, ld, c, K, m0, mine + ent_lo[L] + j * (c - 1));
    }
}

// One instance of a small degree on a cluster of nr CTAs (nr a power of two).  State s of a level
// belongs to CTA s mod nr, which keeps its value at s / nr of its own two level buffers in shared
// memory; a state's children are read from their owners through distributed shared memory, and a
// cluster barrier separates the levels.  Each CTA first copies its transition list (built once per
// degree by cluster_list_kernel) into shared memory, so a level is only loads and the ordered sum.
// The walk's order and arithmetic are dpc_small_kernel's: the result is bit for bit the same.
template <class Op, class PT, class HT, class AT, int MAXT>
__global__ void __launch_bounds__(MAXT) dpc_cluster_kernel(const uint32_t *__restrict__ binom, const uint32_t *__restrict__ gent,
                                                           int64_t stride, const __grid_constant__ ClusterPairs<PT> P,
                                                           HT *__restrict__ out, int K, int lmax)
{
    cg::cluster_group cl = cg::this_cluster();
    const int nr = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int lg = __ffs(nr) - 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int unit_lo[kClusterMaxLevels + 1], ent_lo[kClusterMaxLevels + 1];
    HT *H0 = reinterpret_cast<HT *>(smem_raw);
    HT *H1 = H0 + lmax;
    PT *Ps = reinterpret_cast<PT *>(H1 + lmax);
    const int npairs = K * (K - 1) / 2;
    const int ld = K + 1;
    const size_t tp_off = (((size_t)2 * lmax * sizeof(HT) + (size_t)npairs * sizeof(PT) + 15) / 16) * 16;
    uint2 *TP = reinterpret_cast<uint2 *>(smem_raw + tp_off);
    uint32_t *ENT = reinterpret_cast<uint32_t *>(smem_raw + tp_off + (((size_t)ld * ld * sizeof(uint2) + 15) / 16) * 16);
    const int nlev = K / 2 + 1;  // levels L = 0..K/2, popcount c = 2L
    fill_pair_table(TP, binom, ld, ld, threadIdx.x, blockDim.x);
    for (int q = threadIdx.x; q < npairs; q += blockDim.x) Ps[q] = P.ptr ? P.ptr[q] : P.v[q];
    __syncthreads();
    if (threadIdx.x == 0) cluster_layout(TP, ld, K, nr, rank, unit_lo, ent_lo);
    {
        const int n = (K / 2 + 1) * (K / 2) / 2;  // level c = 2, into H1
        for (int j = threadIdx.x; rank + nr * j < n; j += blockDim.x)
            H1[j] = first_level_value<Op, PT, HT, AT>(rank + nr * j, K, Ps, 1, 0);
    }
    __syncthreads();
    {
        // The list, in 16-byte pieces (the stride and this buffer are padded to 4 entries).
        const uint4 *src = reinterpret_cast<const uint4 *>(gent + (int64_t)rank * stride);
        uint4 *dst = reinterpret_cast<uint4 *>(ENT);
        const int n4 = (ent_lo[nlev] + 3) / 4;
        for (int i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    // Every CTA has started, copied its list and written level c = 2.
    cl.sync();
    for (int L = 2; L < nlev; ++L) {
        const int c = 2 * L;
        const HT *prev = (L & 1) ? H0 : H1;
        HT *cur = (L & 1) ? H1 : H0;
        const int cnt = unit_lo[L + 1] - unit_lo[L];
        for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
            const uint32_t *e = ENT + ent_lo[L] + j * (c - 1);
            AT acc = zero_of<AT>();
            // A remote read takes about as long as a level's arithmetic, so as many of the state's
            // children as the registers hold are requested before the first is used.
            constexpr int kCB = sizeof(HT) <= 8 ? kClusterMaxK - 1 : (kClusterMaxK + 1) / 2;
            for (int x0 = 0; x0 < c - 1; x0 += kCB) {
                HT hv[kCB];
                PT pv[kCB];
#pragma unroll
                for (int u = 0; u < kCB; ++u)
                    if (x0 + u < c - 1) {
                        const uint32_t t = e[x0 + u];
                        const uint32_t child = t >> 8;
                        hv[u] = *cl.map_shared_rank(prev + (child >> lg), child & (uint32_t)(nr - 1));
                        pv[u] = Ps[t & 255u];
                    }
#pragma unroll
                for (int u = 0; u < kCB; ++u)
                    if (x0 + u < c - 1) acc = madd(Op{}, acc, pv[u], hv[u]);
            }
            HT v;
            store(v, acc);
            if (L == nlev - 1) out[0] = v;  // the last level has the one state, on CTA 0
            else cur[j] = v;
        }
        // The level is complete everywhere before any CTA reads it, and before any CTA overwrites
        // the buffer this level read; the last barrier also keeps every CTA's shared memory alive
        // until all remote reads are done.
        cl.sync();
    }
}

// Entries per CTA of the cluster lists: the most any CTA of an nr-CTA cluster lists (CTA 0's),
// rounded up to 4 so that lists are copied in 16-byte pieces.
static int64_t cluster_stride(const DevPlan &plan, int nr)
{
    int64_t e = 0;
    for (int L = 2; L < (int)plan.levels.size(); ++L) e += (plan.levels[L].n + nr - 1) / nr * (2 * L - 1);
    return (e + 3) / 4 * 4;
}

template <class HT>
__global__ void fill_one_kernel(HT *H, int64_t B)
{
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x)
        H[b] = one_of<HT>();
}

__global__ void to_f32_kernel(const double *in, float *out, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(in[i]);
}

__global__ void to_f64_kernel(const float *in, double *out, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

template <class HT>
__global__ void copy_out_kernel(const HT *in, HT *out, int64_t B)
{
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x)
        out[b] = in[b];
}

static unsigned grid_for(int64_t work, int threads)
{
    int64_t blocks = (work + threads - 1) / threads;
    int64_t cap = (int64_t)ctx().num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

static int64_t max_level(const DevPlan &plan)
{
    int64_t m = 1;
    for (const Level &lv : plan.levels) m = lv.n > m ? lv.n : m;
    return m;
}

size_t dp_scratch_bytes(const DevPlan &plan, int dtype, int prec, int64_t B)
{
    size_t hs;
    switch (dtype) {
    case EGG_F64: hs = prec == EGG_PREC_MIXED ? 4 : 8; break;
    case EGG_C128: hs = prec == EGG_PREC_MIXED ? 8 : 16; break;
    case EGG_F32: hs = 4; break;
    case EGG_C64: hs = 8; break;
    case EGG_I64: hs = 16; break;
    default: return 0;
    }
    return 2 * (size_t)max_level(plan) * (size_t)B * hs;
}

// Shared memory the whole-instance kernel needs for this plan (0 if it does not fit).
template <class PT, class HT>
static size_t small_smem(const DevPlan &plan)
{
    if (plan.levels.size() > 33 || plan.K - 1 > kSmallMaxDeg) return 0;
    int64_t maxlev = 1;
    for (const Level &lv : plan.levels) maxlev = lv.n > maxlev ? lv.n : maxlev;
    const int64_t npairs = (int64_t)plan.K * (plan.K - 1) / 2;
    size_t bytes = 2 * (size_t)maxlev * sizeof(HT) + (size_t)npairs * sizeof(PT) + 64;
    return bytes <= 160 * 1024 ? bytes : 0;
}

template <class Op, class I, class PT, class HT, class AT>
static int run_small(const DevPlan &plan, const PT *P, HT *out, int64_t B, size_t smem, cudaStream_t st)
{
    SmallLevels lv;
    lv.nlev = (int)plan.levels.size();
    int64_t maxlev = 1;
    for (int L = 0; L < lv.nlev; ++L) {
        lv.toff[L] = plan.levels[L].toff;
        lv.n[L] = (int)plan.levels[L].n;
        lv.deg[L] = plan.levels[L].deg;
        maxlev = plan.levels[L].n > maxlev ? plan.levels[L].n : maxlev;
    }
    auto k = dp_small_kernel<Op, I, PT, HT, AT>;
    int rc0 = smem_limit_at_least((const void *)k, smem);
    if (rc0) return rc0;
    int64_t grid = B;
    const int64_t cap = (int64_t)ctx().num_sms * 8;
    if (grid > cap) grid = cap;
    const int threads = B == 1 ? 512 : (maxlev >= 1024 ? 256 : 128);
    k<<<(unsigned)grid, threads, smem, st>>>((const I *)plan.trans, lv, P, out, B, plan.K * (plan.K - 1) / 2, (int)maxlev,
                                               pair_bits(plan.idx_bytes));
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

// Shared memory dpc_small_kernel needs for a closed-form plan (0 if it does not fit).
template <class PT, class HT>
static size_t closed_small_smem(const DevPlan &plan)
{
    if (plan.K > 24) return 0;
    const int64_t maxlev = max_level(plan);
    const int64_t npairs = (int64_t)plan.K * (plan.K - 1) / 2;
    size_t bytes = (((size_t)2 * maxlev * sizeof(HT) + (size_t)npairs * sizeof(PT) + 15) / 16) * 16 +
                   (size_t)(plan.K + 1) * (plan.K + 1) * sizeof(uint2);
    return bytes <= 160 * 1024 ? bytes : 0;
}

template <class Op, class M, class PT, class HT, class AT>
static int launch_closed_level(const uint32_t *bt, const PT *P, const HT *prev, HT *cur, int K, int c, int64_t n, int64_t B,
                               cudaStream_t st)
{
    auto k = B == 1 ? dpc_level_kernel<Op, M, PT, HT, AT, true> : dpc_level_kernel<Op, M, PT, HT, AT, false>;
    static bool attr_set = false;  // per instantiation; the library's lock serialises callers
    if (!attr_set) {
        EGG_CUDA_TRY(cudaFuncSetAttribute(dpc_level_kernel<Op, M, PT, HT, AT, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
        EGG_CUDA_TRY(cudaFuncSetAttribute(dpc_level_kernel<Op, M, PT, HT, AT, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
        attr_set = true;
    }
    const size_t sm = level_smem<M, PT>(K, c, B);
    // The longest run (fewest unranks) that still gives every SM several blocks.
    const int64_t want = (int64_t)ctx().num_sms * 4;
    int run = kRun;
    while (run > 1) {
        const int64_t ch = B >= (int64_t)run * kLevelThreads ? 1 : ((int64_t)run * kLevelThreads) / B;
        if ((n + ch - 1) / ch >= want) break;
        run /= 2;
    }
    const int64_t chunk = B >= (int64_t)run * kLevelThreads ? 1 : ((int64_t)run * kLevelThreads) / B;
    int64_t blocks = (n + chunk - 1) / chunk;
    const int64_t cap = (int64_t)ctx().num_sms * 8;
    if (blocks > cap) blocks = cap;
    if constexpr (has_fixed<Op, PT>::value) {
        if (B == 1 && fixed_level<Op, PT, HT, AT>(bt, P, prev, cur, K, c, n, run, (int)blocks, 1, 0, 0, 0, st)) return EGG_OK;
    }
    k<<<(unsigned)blocks, kLevelThreads, sm, st>>>(bt, P, prev, cur, K, c, n, B, run);
    count_launch();
    return EGG_OK;
}

// Levels whose states and transitions together stay below this run inside a span launch.
static constexpr int64_t kSpanWork = (int64_t)1 << 18;

static bool span_level(const DevPlan &plan, int L)
{
    const Level &lv = plan.levels[L];
    return lv.n * (lv.deg > 1 ? lv.deg : 1) <= kSpanWork;
}

// Levels L0..L1 (L0 >= 1) of one instance in one cooperative launch (dpc_span_kernel).
template <class Op, class PT, class HT, class AT>
static int launch_span(const uint32_t *bt, const DevPlan &plan, const PT *P, HT *h0, HT *h1, HT *out, bool out_last, int L0,
                       int L1, cudaStream_t st)
{
    const int K = plan.K;
    auto k = dpc_span_kernel<Op, PT, HT, AT>;
    const size_t smem = (((size_t)(K + 1) * (K + 2) * sizeof(uint2) + 15) / 16) * 16 +
                        (((size_t)K * (K - 1) / 2 * sizeof(PT) + 15) / 16) * 16 + (size_t)8 * 64 * (sizeof(HT) + sizeof(PT));
    static bool attr_set = false;  // per instantiation; callers hold the library's lock
    if (!attr_set) {
        EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
        attr_set = true;
    }
    int per_sm = 0;
    int rc0 = blocks_per_sm((const void *)k, 256, smem, &per_sm);
    if (rc0) return rc0;
    if (per_sm < 1) return fail(EGG_ERR_CUDA, "span kernel cannot be resident");
    int64_t need = 1;  // threads the widest level can use (a warp per state for deep levels)
    for (int L = L0; L <= L1; ++L) {
        const int64_t t = plan.levels[L].n * (2 * L >= kWideMinC ? 32 : 1);
        need = t > need ? t : need;
    }
    int64_t blocks = (need + 255) / 256;
    const int64_t cap = (int64_t)per_sm * ctx().num_sms;
    if (blocks > cap) blocks = cap;
    int oln = out_last ? 1 : 0;
    void *args[] = {(void *)&bt, (void *)&P, (void *)&h0, (void *)&h1, (void *)&out, (void *)&K, (void *)&L0, (void *)&L1,
                    (void *)&oln};
    EGG_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k, dim3((unsigned)blocks), dim3(256), args, smem, st));
    count_launch();
    return EGG_OK;
}

// One instance of a small degree on one cluster (dpc_cluster_kernel) of 16 CTAs, or of 8 where 16
// cannot be placed.  Returns kNoCluster, with nothing launched, when the degree is out of its range
// or the device cannot place such a cluster.
static constexpr int kNoCluster = -1;
static constexpr size_t kClusterSmemMax = 200 * 1024;

template <class Op, class PT, class HT, class AT>
static int launch_cluster(const uint32_t *bt, const DevPlan &plan, const PT *P, HT *out, cudaStream_t st,
                          bool host_pairs = false)
{
    const int K = plan.K;
    if (K < 4 || K > kClusterMaxK || (int)plan.levels.size() != K / 2 + 1 || !plan.closed_form()) return kNoCluster;
    constexpr int kMaxT = 512;  // a level holds at most 8008 / 16 states per CTA at N = 22
    auto k = dpc_cluster_kernel<Op, PT, HT, AT, kMaxT>;
    const int64_t maxlev = max_level(plan);
    const int64_t npairs = (int64_t)K * (K - 1) / 2;
    auto smem_for = [&](int nr) {
        const int64_t lmax = (maxlev + nr - 1) / nr;
        return (((size_t)2 * lmax * sizeof(HT) + (size_t)npairs * sizeof(PT) + 15) / 16) * 16 +
               (((size_t)(K + 1) * (K + 1) * sizeof(uint2) + 15) / 16) * 16 +
               (size_t)cluster_stride(plan, nr) * sizeof(uint32_t);
    };
    // Whether a cluster of this shape can be placed, per (cluster size, shared memory); callers hold
    // the library's lock.
    static std::map<std::pair<int, size_t>, bool> placeable;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kMaxT);
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    // 16 CTAs where they can be placed (each level's remote reads spread over twice the SMs), else 8.
    int nr = 0;
    size_t smem = 0;
    for (int cand : {16, 8}) {
        const size_t sm = smem_for(cand);
        if (sm > kClusterSmemMax) continue;
        at[0].val.clusterDim.x = (unsigned)cand;
        cfg.gridDim = dim3((unsigned)cand);
        cfg.dynamicSmemBytes = sm;
        const auto key = std::make_pair(cand, sm);
        auto it = placeable.find(key);
        if (it == placeable.end()) {
            int rc = smem_limit_at_least((const void *)k, sm);
            if (rc) return rc;
            if (cand > 8) EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, k, &cfg) != cudaSuccess) {
                cudaGetLastError();
                nclusters = 0;
            }
            it = placeable.emplace(key, nclusters > 0).first;
        }
        if (it->second) {
            nr = cand;
            smem = sm;
            break;
        }
    }
    if (!nr) return kNoCluster;
    const int lmax = (int)((maxlev + nr - 1) / nr);
    const int slot = nr == 8 ? 0 : 1;
    const int64_t stride = cluster_stride(plan, nr);
    if (!plan.cluster_lists[slot]) {
        const size_t bytes = (size_t)nr * stride * sizeof(uint32_t);
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return kNoCluster;
        }
        cluster_list_kernel<<<dim3((unsigned)nr, 8), 256, 0, st>>>(bt, (uint32_t *)p, stride, K, nr);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            cudaFree(p);
            return fail(EGG_ERR_CUDA, std::string("cluster lists: ") + cudaGetErrorString(e));
        }
        plan.cluster_lists[slot] = p;
        plan.cluster_list_bytes[slot] = (int64_t)bytes;
    }
    const uint32_t *gent = (const uint32_t *)plan.cluster_lists[slot];
    ClusterPairs<PT> pa;
    pa.ptr = host_pairs ? nullptr : P;
    if (host_pairs) std::memcpy(pa.v, P, (size_t)npairs * sizeof(PT));
    EGG_CUDA_TRY(cudaLaunchKernelEx(&cfg, k, bt, gent, stride, pa, out, K, lmax));
    count_launch();
    return EGG_OK;
}

// A closed-form plan: one launch for small degrees, else one launch per level with the last level
// written straight into `out` when the state type is the output type.  For one instance of a larger
// degree, the runs of small levels at either end of the plan each take one span launch.
template <class Op, class PT, class HT, class AT>
static int run_closed(const DevPlan &plan, const PT *P, HT *h0, HT *h1, HT *out, bool out_direct, int64_t B,
                      cudaStream_t st)
{
    int rc = EGG_OK;
    const uint32_t *bt = binom32_device(&rc);
    if (!bt) return rc;
    const int K = plan.K;
    // A single instance of a small degree: one cluster of CTAs.  A batch of small degrees, whose two
    // largest levels fit in shared memory: one CTA per instance with the whole plan inside it.
    const size_t small = out_direct ? closed_small_smem<PT, HT>(plan) : 0;
    if (out_direct && B == 1) {
        rc = launch_cluster<Op, PT, HT, AT>(bt, plan, P, out, st);
        if (rc != kNoCluster) return rc;
    }
    if (small && B > 1) {
        constexpr int kMaxT = sizeof(HT) <= 8 ? 1024 : 512;
        auto k = dpc_small_kernel<Op, PT, HT, AT, kMaxT>;
        rc = smem_limit_at_least((const void *)k, small);
        if (rc) return rc;
        int64_t grid = B;
        const int64_t cap = (int64_t)ctx().num_sms * 8;
        if (grid > cap) grid = cap;
        const int threads = max_level(plan) >= 1024 ? 256 : 128;
        k<<<(unsigned)grid, threads, small, st>>>(bt, P, out, B, K, (int)max_level(plan));
        count_launch();
        EGG_CUDA_TRY(cudaGetLastError());
        return EGG_OK;
    }
    for (int64_t L = 0; L < (int64_t)plan.levels.size(); ++L)
        if (plan.levels[L].n >= ((int64_t)1 << 31))
            return fail(EGG_ERR_TOO_LARGE, "a level of the degree-" + std::to_string(K) + " plan has 2^31 states or more");
    const int nlev = (int)plan.levels.size();
    int Lh = 0, Lt = nlev;  // levels 1..Lh and Lt..nlev-1 run as spans
    if (B == 1 && K <= 62) {
        while (Lh + 1 < nlev && span_level(plan, Lh + 1)) ++Lh;
        while (Lt - 1 > Lh + 1 && span_level(plan, Lt - 1)) --Lt;
        if (Lh < 2) Lh = 0;            // a span of one level gains nothing
        if (nlev - Lt < 2) Lt = nlev;
    }
    HT *prev;
    int Lnext;
    if (Lh) {
        rc = launch_span<Op, PT, HT, AT>(bt, plan, P, h0, h1, out, out_direct && Lh == nlev - 1, 1, Lh, st);
        if (rc) return rc;
        prev = (Lh == nlev - 1 && out_direct) ? out : ((Lh & 1) ? h1 : h0);
        Lnext = Lh + 1;
    } else {
        prev = (1 == nlev - 1 && out_direct) ? out : h1;  // level c = 2 lands in h1 (odd level)
        const int64_t total = plan.levels[1].n * B;
        dpc_first_kernel<Op, PT, HT, AT><<<grid_for(total, 256), 256, 0, st>>>(P, prev, K, plan.levels[1].n, B);
        count_launch();
        Lnext = 2;
    }
    for (int L = Lnext; L < Lt; ++L) {
        const int c = 2 * L;
        HT *cur = (L == nlev - 1 && out_direct) ? out : ((L & 1) ? h1 : h0);
        const int U = K - (K - c) / 2;
        rc = U <= 32 ? launch_closed_level<Op, uint32_t, PT, HT, AT>(bt, P, prev, cur, K, c, plan.levels[L].n, B, st)
                     : launch_closed_level<Op, uint64_t, PT, HT, AT>(bt, P, prev, cur, K, c, plan.levels[L].n, B, st);
        if (rc) return rc;
        prev = cur;
    }
    if (Lt < nlev) {
        rc = launch_span<Op, PT, HT, AT>(bt, plan, P, h0, h1, out, out_direct, Lt, nlev - 1, st);
        if (rc) return rc;
    }
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <class Op, class I, class PT, class HT, class AT>
static int run_levels(const DevPlan &plan, const PT *P, HT *H0, HT *H1, int64_t B, cudaStream_t st)
{
    fill_one_kernel<HT><<<grid_for(B, 256), 256, 0, st>>>(H0, B);
    count_launch((long long)plan.levels.size());  // the fill and one launch per level below
    const int bits = pair_bits(plan.idx_bytes);
    for (size_t L = 1; L < plan.levels.size(); ++L) {
        const Level &lv = plan.levels[L];
        HT *prev = (L & 1) ? H0 : H1;
        HT *cur = (L & 1) ? H1 : H0;
        int64_t child_lo1 = plan.levels[L - 1].lo + 1;
        unsigned g = grid_for(lv.n * B, 256);
        if (B == 1)
            dp_level_kernel<Op, I, PT, HT, AT, true><<<g, 256, 0, st>>>((const I *)plan.trans, P, prev, cur, lv.n, lv.deg,
                                                                        lv.toff, child_lo1, B, bits);
        else
            dp_level_kernel<Op, I, PT, HT, AT, false><<<g, 256, 0, st>>>((const I *)plan.trans, P, prev, cur, lv.n, lv.deg,
                                                                         lv.toff, child_lo1, B, bits);
    }
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <class I>
static int dp_dispatch(const DevPlan &plan, int dtype, int prec, const void *dP, int64_t B, void *dout, cudaStream_t st)
{
    Context &c = ctx();
    size_t need = dp_scratch_bytes(plan, dtype, prec, B);
    int rc = ensure_buf(c.scratch[0], need);
    if (rc) return rc;
    const size_t half = need / 2;
    char *h0 = (char *)c.scratch[0].ptr, *h1 = h0 + half;
    // The last level holds one state (the full set), so its B values are the results.
    const bool last_in_h0 = ((plan.levels.size() - 1) & 1) == 0;
    char *res = last_in_h0 ? h0 : h1;
    if (prec == EGG_PREC_MIXED && (dtype == EGG_F64 || dtype == EGG_C128)) {
        int64_t npairs = (int64_t)plan.K * (plan.K - 1) / 2;
        int64_t nvals = npairs * B * (dtype == EGG_C128 ? 2 : 1);
        rc = ensure_buf(c.scratch[5], (size_t)nvals * sizeof(float));
        if (rc) return rc;
        float *P32 = (float *)c.scratch[5].ptr;
        to_f32_kernel<<<grid_for(nvals, 256), 256, 0, st>>>((const double *)dP, P32, nvals);
        count_launch();
        if (plan.closed_form()) {
            if (dtype == EGG_F64)
                rc = run_closed<MixedOp, float, float, double>(plan, P32, (float *)h0, (float *)h1, nullptr, false, B, st);
            else
                rc = run_closed<MixedOp, cf, cf, cd>(plan, (const cf *)P32, (cf *)h0, (cf *)h1, nullptr, false, B, st);
        } else if (dtype == EGG_F64) {
            rc = run_levels<MixedOp, I, float, float, double>(plan, P32, (float *)h0, (float *)h1, B, st);
        } else {
            rc = run_levels<MixedOp, I, cf, cf, cd>(plan, (const cf *)P32, (cf *)h0, (cf *)h1, B, st);
        }
        if (rc) return rc;
        to_f64_kernel<<<grid_for(B, 256), 256, 0, st>>>((const float *)res, (double *)dout,
                                                         B * (dtype == EGG_C128 ? 2 : 1));
        count_launch();
        EGG_CUDA_TRY(cudaGetLastError());
        return EGG_OK;
    }
    const bool fma_mode = prec == EGG_PREC_FMA;
    if (prec != EGG_PREC_EXACT && prec != EGG_PREC_FMA && prec != EGG_PREC_MIXED)
        return fail(EGG_ERR_ARGUMENT, "unknown precision mode");
    // Degrees whose levels fit in shared memory run whole instances in one launch.
#define EGG_SMALL_OR_LEVELS(OPX, PT, HT, AT)                                                                   \
    do {                                                                                                      \
        const size_t sm = plan.closed_form() ? 0 : small_smem<PT, HT>(plan);                                  \
        if (plan.closed_form()) {                                                                             \
            rc = run_closed<OPX, PT, HT, AT>(plan, (const PT *)dP, (HT *)h0, (HT *)h1, (HT *)dout, true, B, st); \
        } else if (sm) {                                                                                      \
            rc = run_small<OPX, I, PT, HT, AT>(plan, (const PT *)dP, (HT *)dout, B, sm, st);                  \
        } else {                                                                                              \
            rc = run_levels<OPX, I, PT, HT, AT>(plan, (const PT *)dP, (HT *)h0, (HT *)h1, B, st);             \
            if (!rc) {                                                                                        \
                copy_out_kernel<HT><<<grid_for(B, 256), 256, 0, st>>>((const HT *)res, (HT *)dout, B);        \
                count_launch();                                                                               \
            }                                                                                                 \
        }                                                                                                     \
    } while (0)
    switch (dtype) {
    case EGG_F64:
        if (fma_mode) EGG_SMALL_OR_LEVELS(FmaOp, double, double, double);
        else EGG_SMALL_OR_LEVELS(ExactOp, double, double, double);
        break;
    case EGG_C128:
        if (fma_mode) EGG_SMALL_OR_LEVELS(FmaOp, cd, cd, cd);
        else EGG_SMALL_OR_LEVELS(ExactOp, cd, cd, cd);
        break;
    case EGG_F32:
        if (fma_mode) EGG_SMALL_OR_LEVELS(FmaOp, float, float, float);
        else EGG_SMALL_OR_LEVELS(ExactOp, float, float, float);
        break;
    case EGG_C64:
        if (fma_mode) EGG_SMALL_OR_LEVELS(FmaOp, cf, cf, cf);
        else EGG_SMALL_OR_LEVELS(ExactOp, cf, cf, cf);
        break;
    case EGG_I64:
        EGG_SMALL_OR_LEVELS(IntOp, int64_t, __int128, __int128);
        break;
#undef EGG_SMALL_OR_LEVELS
    default:
        return fail(EGG_ERR_ARGUMENT, "unknown dtype");
    }
    if (rc) return rc;
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

// ---- several single-instance evaluations per launch ------------------------------------------------
//
// For a batch of large degree the instance-fastest level kernel keeps B whole levels live, which
// outgrows L2 (N = 32 complex: 13 MB per instance and level), so every child load reaches HBM.
// Here G instances stored instance-major run the single-instance fixed-popcount kernels side by
// side (blockIdx.y = instance): G levels stay L2-resident and each instance keeps the lean walk.

template <class Op, class PT, class HT, class AT>
__global__ void __launch_bounds__(256) dpc_first_grouped_kernel(const PT *__restrict__ P, HT *__restrict__ Hcur, int K,
                                                                int64_t n, int64_t ldp, int64_t ldh)
{
    const PT *Pi = P + blockIdx.y * ldp;
    HT *Hi = Hcur + blockIdx.y * ldh;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x)
        Hi[s] = first_level_value<Op, PT, HT, AT>(s, K, Pi, 1, 0);
}


template <class HT, class OT>
__global__ void copy_strided_kernel(const HT *__restrict__ in, int64_t ld, OT *__restrict__ out, int64_t G)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < G; g += (int64_t)gridDim.x * blockDim.x)
        store(out[g], in[g * ld]);
}

template <class Op, class PT, class HT, class AT, class OT>
static int run_grouped(const DevPlan &plan, const PT *P, int64_t G, HT *h0, HT *h1, int64_t ldh, OT *out, cudaStream_t st)
{
    int rc = EGG_OK;
    const uint32_t *bt = binom32_device(&rc);
    if (!bt) return rc;
    const int K = plan.K;
    const int64_t ldp = (int64_t)K * (K - 1) / 2;
    const int nlev = (int)plan.levels.size();
    constexpr bool direct = std::is_same<HT, OT>::value;  // the last level can land in `out`
    HT *prev = (nlev == 2 && direct) ? (HT *)out : h1;
    int64_t ldprev = (nlev == 2 && direct) ? 1 : ldh;
    {
        const int64_t n = plan.levels[1].n;
        int64_t bx = (n + 255) / 256;
        if (bx > 4096) bx = 4096;
        dpc_first_grouped_kernel<Op, PT, HT, AT><<<dim3((unsigned)bx, (unsigned)G), 256, 0, st>>>(P, prev, K, n, ldp, ldprev);
        count_launch();
    }
    for (int L = 2; L < nlev; ++L) {
        const int c = 2 * L;
        const int64_t n = plan.levels[L].n;
        const bool last = L == nlev - 1;
        HT *cur = (last && direct) ? (HT *)out : ((L & 1) ? h1 : h0);
        const int64_t ldcur = (last && direct) ? 1 : ldh;
        // Run length as in the single-instance launch, with the G instances sharing the SMs; then
        // one block per chunk of run * 256 states.  Blocks start in index order, x (the chunk)
        // fastest, so the resident blocks work on one or two instances at a time and those
        // instances' previous levels (about 10 MB each at degree 32) stay in L2.  Capping the
        // blocks per instance at 8 * SMs / G, as before, spread the resident blocks over about 16
        // instances, more than L2 holds: the 4096 mix took 42.8 ms against 39.6 ms now.
        const int64_t want = ((int64_t)ctx().num_sms * 4 + G - 1) / G;
        int run = kRun;
        while (run > 1 && (n + (int64_t)run * kLevelThreads - 1) / ((int64_t)run * kLevelThreads) < want) run /= 2;
        const int64_t blocks = (n + (int64_t)run * kLevelThreads - 1) / ((int64_t)run * kLevelThreads);
        if (!fixed_level<Op, PT, HT, AT>(bt, P, prev, cur, K, c, n, run, (int)blocks, (int)G, ldp, ldprev, ldcur, st))
            return fail(EGG_ERR_ARGUMENT, "no fixed-popcount kernel for level " + std::to_string(c) + " of degree " +
                                              std::to_string(K));
        prev = cur;
        ldprev = ldcur;
    }
    if (!direct) {
        copy_strided_kernel<HT, OT><<<grid_for(G, 256), 256, 0, st>>>(prev, ldprev, out, G);
        count_launch();
    }
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

bool dp_grouped_ok(int K, int dtype, int prec)
{
    if (K < 4 || K > 40) return false;  // every level has a fixed-popcount kernel up to K = 40
    if (dtype == EGG_I64) return prec == EGG_PREC_EXACT;
    return dtype == EGG_F64 || dtype == EGG_C128;
}

int dp_run_grouped(const DevPlan &plan, int dtype, int prec, const void *dP, int64_t G, void *dout, cudaStream_t st)
{
    if (!dp_grouped_ok(plan.K, dtype, prec)) return fail(EGG_ERR_ARGUMENT, "no grouped DP for this degree and type");
    if (!plan.closed_form()) return fail(EGG_ERR_ARGUMENT, "grouped DP needs a closed-form plan");
    Context &c = ctx();
    const size_t need = dp_scratch_bytes(plan, dtype, prec, G);
    int rc = ensure_buf(c.scratch[0], need);
    if (rc) return rc;
    const int64_t maxlev = max_level(plan);
    char *h0 = (char *)c.scratch[0].ptr, *h1 = h0 + need / 2;
    const int64_t npairs = (int64_t)plan.K * (plan.K - 1) / 2;
    if (prec == EGG_PREC_MIXED) {
        const int64_t nvals = npairs * G * (dtype == EGG_C128 ? 2 : 1);
        rc = ensure_buf(c.scratch[5], (size_t)nvals * sizeof(float));
        if (rc) return rc;
        float *P32 = (float *)c.scratch[5].ptr;
        to_f32_kernel<<<grid_for(nvals, 256), 256, 0, st>>>((const double *)dP, P32, nvals);
        count_launch();
        if (dtype == EGG_F64)
            return run_grouped<MixedOp, float, float, double, double>(plan, P32, G, (float *)h0, (float *)h1, maxlev,
                                                                      (double *)dout, st);
        return run_grouped<MixedOp, cf, cf, cd, cd>(plan, (const cf *)P32, G, (cf *)h0, (cf *)h1, maxlev, (cd *)dout, st);
    }
    const bool fma_mode = prec == EGG_PREC_FMA;
    switch (dtype) {
    case EGG_F64:
        return fma_mode ? run_grouped<FmaOp, double, double, double, double>(plan, (const double *)dP, G, (double *)h0,
                                                                               (double *)h1, maxlev, (double *)dout, st)
                        : run_grouped<ExactOp, double, double, double, double>(plan, (const double *)dP, G, (double *)h0,
                                                                                 (double *)h1, maxlev, (double *)dout, st);
    case EGG_C128:
        return fma_mode ? run_grouped<FmaOp, cd, cd, cd, cd>(plan, (const cd *)dP, G, (cd *)h0, (cd *)h1, maxlev, (cd *)dout, st)
                        : run_grouped<ExactOp, cd, cd, cd, cd>(plan, (const cd *)dP, G, (cd *)h0, (cd *)h1, maxlev, (cd *)dout, st);
    case EGG_I64:
        return run_grouped<IntOp, int64_t, __int128, __int128, __int128>(plan, (const int64_t *)dP, G, (__int128 *)h0,
                                                                        (__int128 *)h1, maxlev, (__int128 *)dout, st);
    }
    return fail(EGG_ERR_ARGUMENT, "unknown dtype");
}

int dp_run_one_host(const DevPlan &plan, int dtype, int prec, const void *P, void *dout, cudaStream_t st)
{
    if (prec == EGG_PREC_MIXED) return kDpNotHere;
    int rc = EGG_OK;
    const uint32_t *bt = binom32_device(&rc);
    if (!bt) return rc;
    const bool fma_mode = prec == EGG_PREC_FMA;
    switch (dtype) {
    case EGG_F64:
        rc = fma_mode ? launch_cluster<FmaOp, double, double, double>(bt, plan, (const double *)P, (double *)dout, st, true)
                      : launch_cluster<ExactOp, double, double, double>(bt, plan, (const double *)P, (double *)dout, st, true);
        break;
    case EGG_C128:
        rc = fma_mode ? launch_cluster<FmaOp, cd, cd, cd>(bt, plan, (const cd *)P, (cd *)dout, st, true)
                      : launch_cluster<ExactOp, cd, cd, cd>(bt, plan, (const cd *)P, (cd *)dout, st, true);
        break;
    case EGG_F32:
        rc = fma_mode ? launch_cluster<FmaOp, float, float, float>(bt, plan, (const float *)P, (float *)dout, st, true)
                      : launch_cluster<ExactOp, float, float, float>(bt, plan, (const float *)P, (float *)dout, st, true);
        break;
    case EGG_C64:
        rc = fma_mode ? launch_cluster<FmaOp, cf, cf, cf>(bt, plan, (const cf *)P, (cf *)dout, st, true)
                      : launch_cluster<ExactOp, cf, cf, cf>(bt, plan, (const cf *)P, (cf *)dout, st, true);
        break;
    case EGG_I64:
        rc = launch_cluster<IntOp, int64_t, __int128, __int128>(bt, plan, (const int64_t *)P, (__int128 *)dout, st, true);
        break;
    default:
        return kDpNotHere;
    }
    return rc == kNoCluster ? kDpNotHere : rc;
}

int dp_run(const DevPlan &plan, int dtype, int prec, const void *dP, int64_t B, void *dout, cudaStream_t st)
{
    if (prec == EGG_PREC_MIXED && dtype != EGG_F64 && dtype != EGG_C128)
        return fail(EGG_ERR_ARGUMENT, "the mixed form takes Float64 or ComplexF64 inputs");
    return plan.idx_bytes == 4 ? dp_dispatch<int32_t>(plan, dtype, prec, dP, B, dout, st)
                               : dp_dispatch<int64_t>(plan, dtype, prec, dP, B, dout, st);
}

}  // namespace egg
