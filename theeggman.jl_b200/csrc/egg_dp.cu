// egg_dp.cu -- the subset DP (src/dp.jl:344-363 _dp_states!, :408-442 _haf_dp) on the device.
//
// Layout in HBM.  The plan's packed transitions stay resident (one array per (K, layout)).  State
// values live in two ping-pong buffers, each sized for the largest level: every transition out of a
// level lands in the level immediately below (two subset sizes down, src/dp.jl:146-148), so level L
// only ever reads level L-1 and the full `H` of the reference (1.3 GB at K = 40 in FP64) is never
// materialised.  Within a buffer values are instance-fastest, (state - level_lo) * B + b, the
// reference device layout (ext/TheEggmanKernelAbstractionsExt.jl:13-20, :56-62) restricted to
// one level.
//
// Arithmetic.  Each state is accumulated by one thread in plan order, as the reference does.
// EGG_PREC_EXACT rounds every product and sum separately (__dmul_rn/__dadd_rn), which is how Julia
// evaluates the CPU loop, so results are bit-identical to the reference's _haf_dp.  EGG_PREC_FMA
// contracts each multiply-add as the reference's GPU kernel does.  EGG_PREC_MIXED multiplies in
// FP32 and accumulates each state in FP64.  Integer inputs run exactly in Int128.
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
        for (int k = 0; k < deg; ++k) {
            I t = __ldg(tr + k);
            int64_t pi = (int64_t)(t & mask) - 1;
            int64_t ci = (int64_t)(t >> bits) - child_lo1;
            acc = madd(Op{}, acc, P[pi * B + b], Hprev[ci * B + b]);
        }
        store(Hcur[s * B + b], acc);
    }
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

template <class Op, class I, class PT, class HT, class AT>
static int run_levels(const DevPlan &plan, const PT *P, HT *H0, HT *H1, int64_t B, cudaStream_t st)
{
    fill_one_kernel<HT><<<grid_for(B, 256), 256, 0, st>>>(H0, B);
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
        if (dtype == EGG_F64)
            rc = run_levels<MixedOp, I, float, float, double>(plan, P32, (float *)h0, (float *)h1, B, st);
        else
            rc = run_levels<MixedOp, I, cf, cf, cd>(plan, (const cf *)P32, (cf *)h0, (cf *)h1, B, st);
        if (rc) return rc;
        to_f64_kernel<<<grid_for(B, 256), 256, 0, st>>>((const float *)res, (double *)dout,
                                                         B * (dtype == EGG_C128 ? 2 : 1));
        EGG_CUDA_TRY(cudaGetLastError());
        return EGG_OK;
    }
    const bool fma_mode = prec == EGG_PREC_FMA;
    if (prec != EGG_PREC_EXACT && prec != EGG_PREC_FMA && prec != EGG_PREC_MIXED)
        return fail(EGG_ERR_ARGUMENT, "unknown precision mode");
    switch (dtype) {
    case EGG_F64:
        rc = fma_mode ? run_levels<FmaOp, I, double, double, double>(plan, (const double *)dP, (double *)h0, (double *)h1, B, st)
                      : run_levels<ExactOp, I, double, double, double>(plan, (const double *)dP, (double *)h0, (double *)h1, B, st);
        if (!rc) copy_out_kernel<double><<<grid_for(B, 256), 256, 0, st>>>((const double *)res, (double *)dout, B);
        break;
    case EGG_C128:
        rc = fma_mode ? run_levels<FmaOp, I, cd, cd, cd>(plan, (const cd *)dP, (cd *)h0, (cd *)h1, B, st)
                      : run_levels<ExactOp, I, cd, cd, cd>(plan, (const cd *)dP, (cd *)h0, (cd *)h1, B, st);
        if (!rc) copy_out_kernel<cd><<<grid_for(B, 256), 256, 0, st>>>((const cd *)res, (cd *)dout, B);
        break;
    case EGG_F32:
        rc = fma_mode ? run_levels<FmaOp, I, float, float, float>(plan, (const float *)dP, (float *)h0, (float *)h1, B, st)
                      : run_levels<ExactOp, I, float, float, float>(plan, (const float *)dP, (float *)h0, (float *)h1, B, st);
        if (!rc) copy_out_kernel<float><<<grid_for(B, 256), 256, 0, st>>>((const float *)res, (float *)dout, B);
        break;
    case EGG_C64:
        rc = fma_mode ? run_levels<FmaOp, I, cf, cf, cf>(plan, (const cf *)dP, (cf *)h0, (cf *)h1, B, st)
                      : run_levels<ExactOp, I, cf, cf, cf>(plan, (const cf *)dP, (cf *)h0, (cf *)h1, B, st);
        if (!rc) copy_out_kernel<cf><<<grid_for(B, 256), 256, 0, st>>>((const cf *)res, (cf *)dout, B);
        break;
    case EGG_I64:
        rc = run_levels<IntOp, I, int64_t, __int128, __int128>(plan, (const int64_t *)dP, (__int128 *)h0, (__int128 *)h1, B, st);
        if (!rc) copy_out_kernel<__int128><<<grid_for(B, 256), 256, 0, st>>>((const __int128 *)res, (__int128 *)dout, B);
        break;
    default:
        return fail(EGG_ERR_ARGUMENT, "unknown dtype");
    }
    if (rc) return rc;
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

int dp_run(const DevPlan &plan, int dtype, int prec, const void *dP, int64_t B, void *dout, cudaStream_t st)
{
    if (prec == EGG_PREC_MIXED && dtype != EGG_F64 && dtype != EGG_C128)
        return fail(EGG_ERR_ARGUMENT, "the mixed form takes Float64 or ComplexF64 inputs");
    return plan.idx_bytes == 4 ? dp_dispatch<int32_t>(plan, dtype, prec, dP, B, dout, st)
                               : dp_dispatch<int64_t>(plan, dtype, prec, dP, B, dout, st);
}

}  // namespace egg
