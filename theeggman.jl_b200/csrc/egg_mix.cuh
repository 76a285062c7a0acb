// egg_mix.cuh -- pieces of the mixed-degree batch shared by its two engines: the per-level
// launches (egg_mix.cu) and the single persistent launch (egg_mix_persist.cu).
#pragma once

#include "egg_dp_common.cuh"

namespace egg {

static constexpr int kMaxBins = 32;  // even degrees 2..64

struct MixBin {
    int K, npairs;
    int64_t count;  // instances in the bin
    int64_t first;  // position of the bin's first instance in the sorted order
    int64_t poff;   // element offset of the bin's P
    int64_t ebase;  // gather elements before this bin
    int64_t lay;    // P layout: consecutive groups of `lay` instances, instance-fastest within a group
};

struct MixBins {
    int nb;
    MixBin b[kMaxBins];
};

template <class T> __device__ __forceinline__ T mix_one();
template <> __device__ __forceinline__ double mix_one<double>() { return 1.0; }
template <> __device__ __forceinline__ cd mix_one<cd>() { return cd{1.0, 0.0}; }
template <> __device__ __forceinline__ __int128 mix_one<__int128>() { return 1; }

template <class T> __device__ __forceinline__ T nan_of();
template <> __device__ __forceinline__ double nan_of<double>() { return __longlong_as_double(0x7ff8000000000000LL); }
template <> __device__ __forceinline__ cd nan_of<cd>() { return cd{nan_of<double>(), nan_of<double>()}; }
template <> __device__ __forceinline__ int64_t nan_of<int64_t>() { return 0; }

// A parent entry as a pair value: unchanged, or rounded to FP32 for the mixed form (the rounding
// the per-level engine's FP32 copy of its pairs applies).
__device__ __forceinline__ void pair_from(double &d, double v) { d = v; }
__device__ __forceinline__ void pair_from(cd &d, cd v) { d = v; }
__device__ __forceinline__ void pair_from(int64_t &d, int64_t v) { d = v; }
__device__ __forceinline__ void pair_from(float &d, double v) { d = __double2float_rn(v); }
__device__ __forceinline__ void pair_from(cf &d, cd v) { d = cf{__double2float_rn(v.re), __double2float_rn(v.im)}; }

// Gather element g of a mix (g < the bins' total): the bin's pairs, A[r[qi], r[qj]] for
// q = _pair_index(qi+1, qj+1, K) - 1, in groups of `lay` instances: group j at
// poff + j * npairs * lay, pair q of its instance i at q * glen + i.  (lay = 1 is instance-major;
// lay >= count is the instance-fastest matrix of _gather_pairs_batch.)  Row indices outside
// [0, n) are not read: the pair gets NaN (0 for integers).
template <class T, class PT>
__device__ __forceinline__ void mix_gather_elem(int64_t g, const T *__restrict__ A, int64_t n,
                                                const int64_t *__restrict__ offsets, const int32_t *__restrict__ rows,
                                                const int32_t *__restrict__ order, const MixBins &bins, PT *__restrict__ P)
{
    int k = 0;
    while (k + 1 < bins.nb && bins.b[k + 1].ebase <= g) ++k;
    const MixBin &bn = bins.b[k];
    const int64_t e = g - bn.ebase;
    // e enumerates (group, pair, instance in group); groups hold `lay` instances (the last fewer).
    const int64_t per = (int64_t)bn.npairs * bn.lay;
    const int64_t grp = e / per, g0 = grp * bn.lay;
    const int64_t glen = bn.count - g0 < bn.lay ? bn.count - g0 : bn.lay;
    const int64_t w = e - grp * per;
    const int64_t q = w / glen, i = g0 + (w - q * glen);
    int qi = 0, rem = (int)q, len = bn.K - 1;
    while (rem >= len) {
        rem -= len;
        --len;
        ++qi;
    }
    const int qj = qi + 1 + rem;
    const int32_t *r = rows + offsets[order[bn.first + i]];
    const int64_t a = r[qi], c = r[qj];
    if (a < 0 || a >= n || c < 0 || c >= n) {
        pair_from(P[bn.poff + e], nan_of<T>());
    } else {
        pair_from(P[bn.poff + e], A[a + c * n]);
    }
}

// The persistent engine (egg_mix_persist.cu): whether it takes a mix of these bins (Float64,
// ComplexF64 or Int64 parents, degrees up to 32, closed-form plans), and running it -- the gather,
// every bin's levels and the scatter in one cooperative launch.  dsorted holds the results in
// sorted order (ndp of them) and must not alias out.  Returns kDpNotHere, having launched nothing,
// when the device cannot hold the cooperative grid.
bool mix_persistent_ok(const MixBins &bins, const std::vector<DevPlan *> &plans, int dtype, int prec);
int mix_persistent_run(int dtype, int prec, const void *dA, int64_t n, int64_t B, const MixBins &bins,
                       const std::vector<DevPlan *> &plans, const int64_t *doff, const int32_t *drows,
                       const int32_t *dorder, int64_t total, int64_t ndp, int64_t nzero, char *dsorted, void *dout,
                       cudaStream_t st);
// EGG_ERR_TIMEOUT (once) if a persistent launch that has ended gave up waiting at a barrier.
int mix_persistent_take_timeout();

// The engine a mix runs on: per-level launches (the default; recorded as one CUDA graph on a
// shape's second call and replayed after that), or kMixPersistent, one cooperative launch, where
// mix_persistent_ok.
constexpr int kMixLevels = 0;
constexpr int kMixPersistent = 1;
int mix_engine();
int mix_set_engine(int engine);

// Runs the grid barrier alone: every block of a cooperative grid passes three barriers that expect
// `extra` more blocks than there are (extra = 0: the normal barrier).  EGG_OK when no wait ran out,
// EGG_ERR_TIMEOUT when one did (after wait_ns); *passes = barriers passed over all blocks.
int barrier_selfcheck(int extra, int64_t wait_ns, int64_t *passes);

}  // namespace egg
