// egg_internal.cuh -- shared definitions for libeggman_b200 (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/eggman_b200.h"

namespace egg {

// ---- error plumbing ----------------------------------------------------------------------------

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define EGG_CUDA_TRY(expr)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return ::egg::fail(EGG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ---- complex / double-double value types -------------------------------------------------------

struct __align__(16) cd { double re, im; };
struct __align__(8) cf { float re, im; };

// Exact-order arithmetic: every product and sum rounds separately (no FMA contraction), which is
// how Julia evaluates Float64 and Complex{Float64} on the CPU.  Julia's complex product is
// (ar*br - ai*bi, ar*bi + ai*br).
__device__ __forceinline__ double x_madd(double acc, double p, double h) { return __dadd_rn(acc, __dmul_rn(p, h)); }
__device__ __forceinline__ float x_madd(float acc, float p, float h) { return __fadd_rn(acc, __fmul_rn(p, h)); }
__device__ __forceinline__ cd x_cmul(cd a, cd b)
{
    cd r;
    r.re = __dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im));
    r.im = __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re));
    return r;
}
__device__ __forceinline__ cf x_cmul(cf a, cf b)
{
    cf r;
    r.re = __fsub_rn(__fmul_rn(a.re, b.re), __fmul_rn(a.im, b.im));
    r.im = __fadd_rn(__fmul_rn(a.re, b.im), __fmul_rn(a.im, b.re));
    return r;
}
__device__ __forceinline__ cd x_madd(cd acc, cd p, cd h)
{
    cd t = x_cmul(p, h);
    acc.re = __dadd_rn(acc.re, t.re);
    acc.im = __dadd_rn(acc.im, t.im);
    return acc;
}
__device__ __forceinline__ cf x_madd(cf acc, cf p, cf h)
{
    cf t = x_cmul(p, h);
    acc.re = __fadd_rn(acc.re, t.re);
    acc.im = __fadd_rn(acc.im, t.im);
    return acc;
}

// Fused forms (one rounding per multiply-add).
__device__ __forceinline__ double f_madd(double acc, double p, double h) { return fma(p, h, acc); }
__device__ __forceinline__ float f_madd(float acc, float p, float h) { return fmaf(p, h, acc); }
__device__ __forceinline__ cd f_madd(cd acc, cd p, cd h)
{
    acc.re = fma(p.re, h.re, fma(-p.im, h.im, acc.re));
    acc.im = fma(p.re, h.im, fma(p.im, h.re, acc.im));
    return acc;
}
__device__ __forceinline__ cf f_madd(cf acc, cf p, cf h)
{
    acc.re = fmaf(p.re, h.re, fmaf(-p.im, h.im, acc.re));
    acc.im = fmaf(p.re, h.im, fmaf(p.im, h.re, acc.im));
    return acc;
}

// Double-double accumulation (Knuth's TwoSum, then a fast renormalisation).
struct dd { double hi, lo; };
__device__ __forceinline__ void dd_add(dd &a, double x)
{
    double s = __dadd_rn(a.hi, x);
    double bp = __dsub_rn(s, a.hi);
    double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bp)), __dsub_rn(x, bp));
    double t = __dadd_rn(a.lo, e);
    double h = __dadd_rn(s, t);
    a.lo = __dsub_rn(t, __dsub_rn(h, s));
    a.hi = h;
}
__device__ __forceinline__ void dd_add(dd &a, dd b)
{
    dd_add(a, b.hi);
    dd_add(a, b.lo);
}

// ---- device plans ------------------------------------------------------------------------------

// One subset-size level of a plan: states lo..lo+n-1 (0-based), each with `deg` transitions,
// the first at offset toff (0-based) of trans.  Every state of a level has the same out-degree
// (|S| - 1, src/dp.jl:384-385), so `starts` is implied and never read on the device.
struct Level {
    int64_t lo, n, toff;
    int deg;
};

// A plan is either closed-form (`trans` null: the layout _build_dp_plan produces, evaluated without
// reading any transition array) or explicit (an uploaded `trans` that passed the structure check
// but differs from that layout, evaluated by reading it).
struct DevPlan {
    int K = 0, idx_bytes = 0;
    int64_t nstates = 0, ntrans = 0;
    void *trans = nullptr;        // device, ntrans entries of idx_bytes; null for a closed-form plan
    std::vector<Level> levels;    // levels[0] is the empty set
    std::vector<int64_t> level_starts;  // the reference's 1-based `levels` vector
    // The one-instance cluster kernel's transition lists for clusters of 8 and of 16 CTAs (closed-form
    // plans of small degrees), built on first use and kept with the plan.
    mutable void *cluster_lists[2] = {nullptr, nullptr};
    mutable int64_t cluster_list_bytes[2] = {0, 0};
    bool closed_form() const { return trans == nullptr; }
    int64_t bytes() const
    {
        return (trans ? ntrans * (int64_t)idx_bytes : 0) + cluster_list_bytes[0] + cluster_list_bytes[1];
    }
};

// Frees a plan's device memory (its transition array and its cluster lists).
inline void release_plan_memory(DevPlan &p)
{
    if (p.trans) cudaFree(p.trans);
    p.trans = nullptr;
    for (int i = 0; i < 2; ++i) {
        if (p.cluster_lists[i]) cudaFree(p.cluster_lists[i]);
        p.cluster_lists[i] = nullptr;
        p.cluster_list_bytes[i] = 0;
    }
}

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct Context {
    int device = -1;
    cudaStream_t stream = nullptr;
    // Side streams for launches that leave most of the machine idle (they overlap the main
    // stream's and each other), with the events that fork them from and join them back to the
    // calling stream.
    static constexpr int kSideStreams = 4;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kSideStreams] = {};
    // Page-locked host staging for small transfers: a copy from pageable memory is staged by the
    // driver at a fixed cost of several microseconds, a copy from page-locked memory is not.
    void *pinned = nullptr;      // mapped: pinned_dev is its device address
    void *pinned_dev = nullptr;
    static constexpr size_t kPinnedBytes = 128 * 1024;
    int num_sms = 0;
    std::map<std::pair<int, int>, DevPlan> plans;
    DevBuf scratch[11];  // H, P, out, sieve matrix, sieve out, misc, mixed-degree batch + its staging,
                         // the reference-order sieve's terms, the repeated batches' preparation, the
                         // persistent mix launch's step tables: grown on demand, never shrunk
    std::recursive_mutex mu;
};

Context &ctx();
int ensure_init();
int create_streams(Context &c, int device);

// Kernel launches the library has made since it was loaded (reported by egg_launch_count).
extern std::atomic<long long> g_launches;
inline void count_launch(long long n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int ensure_buf(DevBuf &b, size_t bytes);
// Raises kernel k's dynamic shared-memory limit to at least `bytes`; the runtime is called only
// when the limit last set for k is lower (callers hold the library's lock).
int smem_limit_at_least(const void *k, size_t bytes);
// Resident blocks per SM of kernel k at this block size and dynamic shared memory, cached.
int blocks_per_sm(const void *k, int threads, size_t smem, int *out);
DevPlan *find_plan(int K, int idx_bytes);

// Closed-form plan size (_dp_counts, src/dp.jl:192-208).
void dp_counts(int K, int64_t &nstates, int64_t &ntrans);
inline int pair_bits(int idx_bytes) { return idx_bytes == 4 ? 9 : 12; }

// ---- entry points implemented per file ----------------------------------------------------------

// egg_plan.cu
// Level table of the degree-K plan (no device memory: the plan is closed-form).
int plan_levels(int K, int idx_bytes, DevPlan &out);
// Write the closed-form plan's packed transitions into dst (ntrans entries of idx_bytes).
int plan_materialize(const DevPlan &p, void *dst, cudaStream_t st);
// Whether an explicit plan's transitions equal the closed-form layout, entry for entry.
int plan_is_closed_form(const DevPlan &p, cudaStream_t st, bool *same);
int plan_validate_device(const DevPlan &p, cudaStream_t st);
// Saturated 32-bit binomial table C(n, k), n, k <= 64, row-major with row length 65, in device
// memory (uploaded once; no allocation).
const uint32_t *binom32_device(int *rc);

// egg_dp.cu
// The resident plan for degree K in the layout the reference picks for it (Int32 up to K = 32),
// made resident (closed form) if absent.
DevPlan *dp_plan_for(int K, int *rc);
int dp_run(const DevPlan &plan, int dtype, int prec, const void *dP, int64_t B, void *dout, cudaStream_t st);
// One instance whose pairs are in host memory, carried in the launch's parameters (small degrees on
// one cluster); dout is device-visible.  Returns kDpNotHere, with nothing launched, when that
// kernel does not take the call.
constexpr int kDpNotHere = -1;
int dp_run_one_host(const DevPlan &plan, int dtype, int prec, const void *P, void *dout, cudaStream_t st);
size_t dp_scratch_bytes(const DevPlan &plan, int dtype, int prec, int64_t B);
// G instances of a closed-form plan side by side, each evaluated as a single instance: P is
// instance-major (instance g's pairs at g * npairs), out receives G values.  Degrees 4..40, for
// Float64/ComplexF64 (all modes) and Int64 (exact); dp_grouped_ok says which.
bool dp_grouped_ok(int K, int dtype, int prec);
int dp_run_grouped(const DevPlan &plan, int dtype, int prec, const void *dP, int64_t G, void *dout, cudaStream_t st);

// egg_mix.cu
// Hafnians of the principal submatrices A[r, r], r = rows[offsets[b]..offsets[b+1]), of the n x n
// column-major parent A: A, rows and out in device memory, offsets on the host.
int mix_run(int dtype, int prec, const void *dA, int64_t n, int64_t B, const int64_t *offsets, const int32_t *drows,
            void *dout, cudaStream_t st);
// The evaluation the tuner chose for (K, dtype, prec): batched (1) or grouped single instances (0),
// and the group size.
int mix_tuned(int K, int dtype, int prec, int *batched, int64_t *group);
int mix_set_tuning(int K, int dtype, int prec, int batched, int64_t group);
// Drop the mixed-degree batch's recorded graphs (they hold the library's buffer addresses).
void mix_graphs_clear();

// egg_sieve.cu
// A caller-provided device region for the sieve's tables and partial sums (used instead of the
// library's growable buffer when given), with the SM count to shape the launches.
struct FixedScratch {
    void *ptr;
    size_t bytes;
    int num_sms;
};
// stage (optional, synchronous callers only): page-locked host memory of stage_cap bytes through
// which the launch's small tables are copied, when they fit.
int sieve_run(int dtype, int prec, const void *dAx, int64_t E, const int64_t *edge_reps, int glynn, void *dout,
              cudaStream_t st, void *stage = nullptr, size_t stage_cap = 0);
int sieve_batch_run(int dtype, int prec, int64_t B, int64_t Emax, const void *dAx, const int64_t *E,
                    const int64_t *edge_reps, const int32_t *glynn, void *dout, cudaStream_t st,
                    const FixedScratch *fixed = nullptr, double *terms = nullptr, void *stage = nullptr,
                    size_t stage_cap = 0);
// One sieve summed as the reference sums it (_sieve_sum, src/hafnian.jl:713-738): every term in the
// reference's arithmetic, then plain FP64 sums over `nchunks` equal chunks of the term range, each
// in term order, and the chunk sums left to right.  Host edge_reps, device Ax and out.
int sieve_reference_sum_run(int dtype, const void *dAx, int64_t E, const int64_t *edge_reps, int glynn, int64_t nchunks,
                            void *dout, cudaStream_t st);

inline size_t dtype_size(int dtype)
{
    switch (dtype) {
    case EGG_F64: return 8;
    case EGG_C128: return 16;
    case EGG_F32: return 4;
    case EGG_C64: return 8;
    case EGG_I64: return 8;
    }
    return 0;
}

}  // namespace egg
