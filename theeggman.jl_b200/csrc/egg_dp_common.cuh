// egg_dp_common.cuh -- pieces shared by the DP kernels (egg_dp.cu) and the fixed-popcount
// closed-form kernels (egg_dp_fixed.cuh): rounding modes, the colex helpers and the level layout.
#pragma once

#include "egg_internal.cuh"

namespace egg {

struct ExactOp {};
struct FmaOp {};
struct MixedOp {};
struct IntOp {};

template <class A> __device__ __forceinline__ A zero_of();
template <> __device__ __forceinline__ double zero_of<double>() { return 0.0; }
template <> __device__ __forceinline__ float zero_of<float>() { return 0.0f; }
template <> __device__ __forceinline__ cd zero_of<cd>() { return cd{0.0, 0.0}; }
template <> __device__ __forceinline__ cf zero_of<cf>() { return cf{0.0f, 0.0f}; }
template <> __device__ __forceinline__ __int128 zero_of<__int128>() { return 0; }

template <class A> __device__ __forceinline__ A one_of();
template <> __device__ __forceinline__ double one_of<double>() { return 1.0; }
template <> __device__ __forceinline__ float one_of<float>() { return 1.0f; }
template <> __device__ __forceinline__ cd one_of<cd>() { return cd{1.0, 0.0}; }
template <> __device__ __forceinline__ cf one_of<cf>() { return cf{1.0f, 0.0f}; }
template <> __device__ __forceinline__ __int128 one_of<__int128>() { return 1; }

// madd(op, acc, p, h) = acc + p*h in the op's rounding.
__device__ __forceinline__ double madd(ExactOp, double a, double p, double h) { return x_madd(a, p, h); }
__device__ __forceinline__ float madd(ExactOp, float a, float p, float h) { return x_madd(a, p, h); }
__device__ __forceinline__ cd madd(ExactOp, cd a, cd p, cd h) { return x_madd(a, p, h); }
__device__ __forceinline__ cf madd(ExactOp, cf a, cf p, cf h) { return x_madd(a, p, h); }
__device__ __forceinline__ double madd(FmaOp, double a, double p, double h) { return f_madd(a, p, h); }
__device__ __forceinline__ float madd(FmaOp, float a, float p, float h) { return f_madd(a, p, h); }
__device__ __forceinline__ cd madd(FmaOp, cd a, cd p, cd h) { return f_madd(a, p, h); }
__device__ __forceinline__ cf madd(FmaOp, cf a, cf p, cf h) { return f_madd(a, p, h); }
__device__ __forceinline__ double madd(MixedOp, double a, float p, float h) { return __dadd_rn(a, (double)__fmul_rn(p, h)); }
__device__ __forceinline__ cd madd(MixedOp, cd a, cf p, cf h)
{
    cf t = x_cmul(p, h);
    a.re = __dadd_rn(a.re, (double)t.re);
    a.im = __dadd_rn(a.im, (double)t.im);
    return a;
}
__device__ __forceinline__ __int128 madd(IntOp, __int128 a, int64_t p, __int128 h) { return a + (__int128)p * h; }

// Storage conversions from the accumulator.
__device__ __forceinline__ void store(double &d, double a) { d = a; }
__device__ __forceinline__ void store(float &d, float a) { d = a; }
__device__ __forceinline__ void store(float &d, double a) { d = __double2float_rn(a); }
__device__ __forceinline__ void store(cd &d, cd a) { d = a; }
__device__ __forceinline__ void store(cf &d, cf a) { d = a; }
__device__ __forceinline__ void store(cf &d, cd a) { d = cf{__double2float_rn(a.re), __double2float_rn(a.im)}; }
__device__ __forceinline__ void store(__int128 &d, __int128 a) { d = a; }
// Widening stores of the mixed form's results (FP32 storage, FP64 output).
__device__ __forceinline__ void store(double &d, float a) { d = (double)a; }
__device__ __forceinline__ void store(cd &d, cf a) { d = cd{(double)a.re, (double)a.im}; }

// Loads that bypass L1, for a level written earlier in the same kernel by other SMs (their L1
// copies of the buffer, from two levels back, would be stale).
template <class T> __device__ __forceinline__ T ld_l2(const T *p) { return __ldcg(p); }
template <> __device__ __forceinline__ int64_t ld_l2<int64_t>(const int64_t *p)
{
    return (int64_t)__ldcg(reinterpret_cast<const long long *>(p));
}
template <> __device__ __forceinline__ cd ld_l2<cd>(const cd *p)
{
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return cd{v.x, v.y};
}
template <> __device__ __forceinline__ cf ld_l2<cf>(const cf *p)
{
    const float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
    return cf{v.x, v.y};
}
template <> __device__ __forceinline__ __int128 ld_l2<__int128>(const __int128 *p)
{
    const longlong2 v = __ldcg(reinterpret_cast<const longlong2 *>(p));
    return (__int128)(unsigned long long)v.x | ((__int128)v.y << 64);
}

// Weak loads cached in L1 (ld.global.ca), never the read-only path: for a level that other blocks
// of the same launch wrote before a grid-wide barrier.  The barrier's fences order those writes
// before these loads, as for any ordinary load after a cooperative grid synchronisation; the
// read-only path (ld.global.nc), which a const __restrict__ pointer may get, has no such guarantee.
template <class T> __device__ __forceinline__ T ld_ca(const T *p) { return __ldca(p); }
template <> __device__ __forceinline__ int64_t ld_ca<int64_t>(const int64_t *p)
{
    return (int64_t)__ldca(reinterpret_cast<const long long *>(p));
}
template <> __device__ __forceinline__ cd ld_ca<cd>(const cd *p)
{
    const double2 v = __ldca(reinterpret_cast<const double2 *>(p));
    return cd{v.x, v.y};
}
template <> __device__ __forceinline__ cf ld_ca<cf>(const cf *p)
{
    const float2 v = __ldca(reinterpret_cast<const float2 *>(p));
    return cf{v.x, v.y};
}
template <> __device__ __forceinline__ __int128 ld_ca<__int128>(const __int128 *p)
{
    const longlong2 v = __ldca(reinterpret_cast<const longlong2 *>(p));
    return (__int128)(unsigned long long)v.x | ((__int128)v.y << 64);
}

// Level c = 2: state s = {e1 < e2} (colex rank C(e2, 2) + e1) has the single transition to the
// empty set, whose value is 1.
template <class Op, class PT, class HT, class AT>
__device__ __forceinline__ HT first_level_value(int64_t s, int K, const PT *P, int64_t B, int64_t b)
{
    const int m0 = (K - 2) / 2;
    int e2 = (int)((1.0 + sqrt(1.0 + 8.0 * (double)s)) * 0.5);
    while ((int64_t)e2 * (e2 - 1) / 2 > s) --e2;
    while ((int64_t)(e2 + 1) * e2 / 2 <= s) ++e2;
    const int e1 = (int)(s - (int64_t)e2 * (e2 - 1) / 2);
    const int ib = e1 + m0 + 1;
    const int q = (ib - 1) * K - (ib * (ib + 1)) / 2 + m0 + e2;
    HT out;
    store(out, madd(Op{}, zero_of<AT>(), P[(int64_t)q * B + b], one_of<HT>()));
    return out;
}

// Transitions whose loads a thread issues together before accumulating them in order.
static constexpr int kBatch = 8;

template <class M> __device__ __forceinline__ int low_bit(M v);
template <> __device__ __forceinline__ int low_bit<uint32_t>(uint32_t v) { return __ffs((int)v) - 1; }
template <> __device__ __forceinline__ int low_bit<uint64_t>(uint64_t v) { return __ffsll((long long)v) - 1; }

// The colex-successor of a c-subset mask (the next larger integer with the same popcount).
template <class M> __device__ __forceinline__ M colex_next(M v)
{
    const M t = v | (v - 1);
    return (t + 1) | (((~t & (M)(0 - ~t)) - 1) >> (low_bit<M>(v) + 1));
}

// Pair table row x, columns k = 0..ld-1: {C(x, k), C(x, k + 1)}, saturated at 2^32 - 1 (which
// stays above every rank compared against it; saturated entries are never summed).
__device__ __forceinline__ void fill_pair_table(uint2 *TP, const uint32_t *binom, int rows, int ld, int tid, int nthr)
{
    for (int i = tid; i < rows * ld; i += nthr) {
        const int x = i / ld, k = i - (i / ld) * ld;
        TP[i] = make_uint2(binom[x * 65 + k], k + 1 <= 64 ? binom[x * 65 + k + 1] : 0u);
    }
}

// The c-subset of [0, U) with colex rank R.
template <class M>
__device__ __forceinline__ M colex_unrank(const uint2 *TP, int ld, int U, int c, uint32_t R)
{
    M m = 0;
    int x = U - 1;
    for (int i = c; i >= 1; --i) {
        uint32_t v;
        while ((v = TP[x * ld + i].x) > R) --x;
        m |= (M)1 << x;
        R -= v;
        --x;
    }
    return m;
}

// One level (c >= 4) of a closed-form plan.  Each block takes chunks of run * 256 consecutive
// states (run <= kRun, smaller for small levels so that every SM gets blocks): first every thread
// writes the masks of `run` consecutive states into shared memory (one unrank, then colex
// successors), then the threads walk the chunk's (state, instance) pairs with consecutive threads
// on consecutive pairs, so a warp's child loads fall on a few neighbouring sectors.
static constexpr int kRun = 8;
static constexpr int kLevelThreads = 256;

// Byte offset of the staged pairs in dpc_level_kernel's shared memory (16-byte aligned for the
// complex types), after the masks and the pair table.
template <class M>
__host__ __device__ __forceinline__ size_t level_pairs_offset(int U, int ld)
{
    return (((size_t)kRun * kLevelThreads * sizeof(M) + (size_t)U * ld * sizeof(uint2)) + 15) / 16 * 16;
}

template <class M, class PT>
static size_t level_smem(int K, int c, int64_t B)
{
    const int m0 = (K - c) / 2, U = K - m0;
    size_t bytes = level_pairs_offset<M>(U, c + 1);
    if (B == 1) bytes += (size_t)K * (K - 1) / 2 * sizeof(PT);
    return bytes;
}

// Fixed-popcount level kernels exist for these (Op, pair type) combinations
// (egg_dp_fixed_*.cu); other combinations use the runtime-popcount kernel.
template <class Op, class PT> struct has_fixed { static constexpr bool value = false; };
template <> struct has_fixed<ExactOp, double> { static constexpr bool value = true; };
template <> struct has_fixed<FmaOp, double> { static constexpr bool value = true; };
template <> struct has_fixed<ExactOp, cd> { static constexpr bool value = true; };
template <> struct has_fixed<FmaOp, cd> { static constexpr bool value = true; };
template <> struct has_fixed<IntOp, int64_t> { static constexpr bool value = true; };
template <> struct has_fixed<MixedOp, float> { static constexpr bool value = true; };
template <> struct has_fixed<MixedOp, cf> { static constexpr bool value = true; };

// Launches level c of a closed-form plan for G independent instances with a kernel specialised
// for that popcount; instance g's pairs are at P + g * ldp and its level values at prev + g * ldhp
// (read) and cur + g * ldhc (written).  Returns false (and launches nothing) when no
// specialisation covers (c, U).
template <class Op, class PT, class HT, class AT>
bool fixed_level(const uint32_t *binom, const PT *P, const HT *prev, HT *cur, int K, int c, int64_t n, int run,
                 int blocks, int G, int64_t ldp, int64_t ldhp, int64_t ldhc, cudaStream_t st);

}  // namespace egg
