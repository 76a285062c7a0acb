// egg_plan.cu -- subset-DP plans in device memory.
//
// The reference builds a plan on the host (src/dp.jl:223-304): a DFS from the full mask, a sort of
// every reachable mask by (popcount, mask), a Dict from mask to state number, and a CSR walk.
// At K = 40 that is 2.84e9 transitions (22.7 GB as Int64) and needs about twice that in host RAM.
//
// Here that layout is never stored: its closed form is enough to evaluate it (egg_dp.cu), to write
// it out on request and to recognise it in an uploaded array.  The reachable subsets are:
// S is reachable iff, with r = K - |S| removed, its minimum bit (0-based) is >= ceil(r/2)
// (src/dp.jl:16-27: p - 1 <= r <= 2(p - 1)).  So the level of popcount c is exactly the set of all
// c-subsets of the top U = K - ceil((K-c)/2) bit positions, and sorting by mask value within a level
// is colex order.  A state's number is therefore its level's offset plus its colex rank
// sum_i C(e_i, i) (combinatorial number system, e_i the shifted elements in increasing order), and
// each thread can unrank its own state and rank each of its children without any table.
#include "egg_internal.cuh"
#include "egg_perdevice.h"

namespace egg {

static __device__ __forceinline__ int64_t pair_index(int64_t i, int64_t j, int64_t K)
{
    // _pair_index(i, j, K), src/unrolled.jl:60 (1-based, i < j).
    return (i - 1) * K - (i * (i + 1)) / 2 + j;
}

// Binomial table C(n, k) for n, k <= 64 (C(64, 32) < 2^63), staged per block in shared memory.
__constant__ int64_t c_binom_dummy;  // keeps the constant bank initialised on every build

// Writes level c's transitions (CHECK = false) or counts the entries of `trans` that differ from
// them (CHECK = true).
template <class I, bool CHECK>
__global__ void __launch_bounds__(256) plan_level_kernel(I *__restrict__ trans, const int64_t *__restrict__ binom_g,
                                                         int K, int c, int m0, int64_t n, int64_t toff,
                                                         int64_t child_lo1, int bits, unsigned long long *diff)
{
    __shared__ int64_t binom[65 * 65];
    for (int i = threadIdx.x; i < 65 * 65; i += blockDim.x) binom[i] = binom_g[i];
    __syncthreads();
    const int U = K - m0;  // level elements are the shifted positions 0..U-1
    unsigned long long ndiff = 0;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        // Unrank s (colex) into c shifted elements e[1] < ... < e[c].
        int e[65];
        int64_t R = s;
        int x = U - 1;
        for (int i = c; i >= 1; --i) {
            while (binom[x * 65 + i] > R) --x;
            e[i] = x;
            R -= binom[x * 65 + i];
            --x;
        }
        // Child of removing e[1] (the minimum) and e[j]: its elements shift down by one more
        // position (the child level's offset is m0 + 1).  rank = pre[j] + suf[j] with
        // pre[j] = sum_{x=2}^{j-1} C(e_x - 1, x - 1), suf[j] = sum_{x=j+1}^{c} C(e_x - 1, x - 2).
        int64_t suf[66];
        suf[c + 1] = 0;
        suf[c] = 0;
        for (int x2 = c; x2 >= 3; --x2) suf[x2 - 1] = suf[x2] + binom[(e[x2] - 1) * 65 + (x2 - 2)];
        int64_t pre = 0;
        const int64_t ib = (int64_t)e[1] + m0 + 1;  // 1-based index of the minimum
        I *out = trans + toff + s * (int64_t)(c - 1);
        for (int j = 2; j <= c; ++j) {
            int64_t child = child_lo1 + pre + suf[j];
            int64_t jb = (int64_t)e[j] + m0 + 1;
            const I v = (I)((child << bits) | pair_index(ib, jb, K));
            if (CHECK) ndiff += out[j - 2] != v;
            else out[j - 2] = v;
            pre += binom[(e[j] - 1) * 65 + (j - 1)];
        }
    }
    if (CHECK && ndiff) atomicAdd(diff, ndiff);
}

static void host_binom(std::vector<int64_t> &t)
{
    t.assign(65 * 65, 0);
    for (int nn = 0; nn <= 64; ++nn) {
        t[nn * 65 + 0] = 1;
        for (int k = 1; k <= nn; ++k) {
            __int128 v = (__int128)t[(nn - 1) * 65 + (k - 1)] + (k <= nn - 1 ? t[(nn - 1) * 65 + k] : 0);
            t[nn * 65 + k] = v > INT64_MAX ? INT64_MAX : (int64_t)v;
        }
    }
}

int plan_levels(int K, int idx_bytes, DevPlan &p)
{
    int64_t ns, nt;
    dp_counts(K, ns, nt);
    p.K = K;
    p.idx_bytes = idx_bytes;
    p.nstates = ns;
    p.ntrans = nt;
    p.trans = nullptr;
    std::vector<int64_t> binom;
    host_binom(binom);
    // Levels: popcount c = 0, 2, ..., K.
    int64_t lo = 0, toff = 0;
    p.levels.clear();
    p.level_starts.clear();
    for (int c = 0; c <= K; c += 2) {
        int m0 = (K - c + 1) / 2;
        int U = K - m0;
        Level lv;
        lv.lo = lo;
        lv.n = binom[U * 65 + c];
        lv.toff = toff;
        lv.deg = c == 0 ? 0 : c - 1;
        p.levels.push_back(lv);
        p.level_starts.push_back(lo + 1);
        lo += lv.n;
        toff += lv.n * lv.deg;
    }
    p.level_starts.push_back(lo + 1);
    if (lo != ns || toff != nt) return fail(EGG_ERR_PLAN_INVALID, "closed-form level sizes disagree with _dp_counts");
    return EGG_OK;
}

// Runs plan_level_kernel over every level of p into (CHECK = false) or against (CHECK = true) dst.
template <bool CHECK>
static int run_plan_kernels(const DevPlan &p, void *dst, cudaStream_t st, unsigned long long *ddiff)
{
    Context &cx = ctx();
    std::vector<int64_t> binom;
    host_binom(binom);
    int64_t *dbinom = nullptr;
    EGG_CUDA_TRY(cudaMalloc(&dbinom, binom.size() * sizeof(int64_t)));
    cudaError_t e = cudaMemcpyAsync(dbinom, binom.data(), binom.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st);
    const int bits = pair_bits(p.idx_bytes);
    for (size_t L = 1; e == cudaSuccess && L < p.levels.size(); ++L) {
        const Level &lv = p.levels[L];
        const int c = 2 * (int)L;
        const int m0 = (p.K - c + 1) / 2;
        int64_t blocks = (lv.n + 255) / 256;
        const int64_t cap = (int64_t)cx.num_sms * 16;
        if (blocks > cap) blocks = cap;
        const int64_t child_lo1 = p.levels[L - 1].lo + 1;
        if (p.idx_bytes == 4)
            plan_level_kernel<int32_t, CHECK><<<(unsigned)blocks, 256, 0, st>>>((int32_t *)dst, dbinom, p.K, c, m0, lv.n,
                                                                               lv.toff, child_lo1, bits, ddiff);
        else
            plan_level_kernel<int64_t, CHECK><<<(unsigned)blocks, 256, 0, st>>>((int64_t *)dst, dbinom, p.K, c, m0, lv.n,
                                                                               lv.toff, child_lo1, bits, ddiff);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dbinom);
    if (e != cudaSuccess) return fail(EGG_ERR_CUDA, std::string("plan kernels: ") + cudaGetErrorString(e));
    return EGG_OK;
}

int plan_materialize(const DevPlan &p, void *dst, cudaStream_t st) { return run_plan_kernels<false>(p, dst, st, nullptr); }

int plan_is_closed_form(const DevPlan &p, cudaStream_t st, bool *same)
{
    *same = false;
    if (!p.trans) return fail(EGG_ERR_ARGUMENT, "plan has no transition array to compare");
    unsigned long long *ddiff = nullptr;
    EGG_CUDA_TRY(cudaMalloc(&ddiff, sizeof(unsigned long long)));
    cudaError_t e = cudaMemsetAsync(ddiff, 0, sizeof(unsigned long long), st);
    int rc = e == cudaSuccess ? run_plan_kernels<true>(p, p.trans, st, ddiff)
                              : fail(EGG_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    unsigned long long diff = 1;
    if (!rc) {
        e = cudaMemcpy(&diff, ddiff, sizeof(diff), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(EGG_ERR_CUDA, std::string("plan compare: ") + cudaGetErrorString(e));
    }
    cudaFree(ddiff);
    if (!rc) *same = diff == 0;
    return rc;
}

// ---- the binomial table the closed-form DP kernels and the sieve read ---------------------------

// C(n, k) for n, k <= 64, saturated at 2^32 - 1, row-major with row length 65.  Computed at compile
// time and placed in the module image, so every device that loads the library holds its own copy
// from the start: nothing is uploaded and no stream is touched.
struct Binom32Table {
    uint32_t v[65 * 65];
};
static constexpr Binom32Table make_binom32()
{
    Binom32Table t{};
    uint64_t row[65] = {};  // C(nn, k), saturated at 2^32 - 1
    for (int nn = 0; nn <= 64; ++nn) {
        for (int k = nn; k >= 1; --k) {
            const uint64_t v = row[k] + row[k - 1];
            row[k] = v > 0xFFFFFFFFull ? 0xFFFFFFFFull : v;
        }
        row[0] = 1;
        for (int k = 0; k <= 64; ++k) t.v[nn * 65 + k] = (uint32_t)row[k];
    }
    return t;
}
static __device__ const Binom32Table g_binom32 = make_binom32();
static_assert(make_binom32().v[32 * 65 + 16] == 601080390u, "C(32, 16)");
static_assert(make_binom32().v[40 * 65 + 20] == 0xFFFFFFFFu, "C(40, 20) saturates");

static PerDevice<const uint32_t *> g_binom32_addr;

const uint32_t *binom32_device(int *rc)
{
    *rc = EGG_OK;
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *rc = fail(EGG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return nullptr;
    }
    const uint32_t *addr = nullptr;
    *rc = g_binom32_addr.get(
        dev, &addr,
        [](int, const uint32_t **out) {
            void *p = nullptr;
            cudaError_t e2 = cudaGetSymbolAddress(&p, g_binom32);
            if (e2 != cudaSuccess || !p)
                return fail(EGG_ERR_CUDA, std::string("binomial table address: ") + cudaGetErrorString(e2));
            *out = (const uint32_t *)p;
            return (int)EGG_OK;
        });
    if (*rc == PerDevice<const uint32_t *>::kBadDevice)
        *rc = fail(EGG_ERR_NO_DEVICE, "device index " + std::to_string(dev) + " out of range for the binomial table");
    return *rc ? nullptr : addr;
}

// Structure check for a plan that came from the host: every transition of level L must name a
// child in level L-1 and a pair index in 1..K(K-1)/2.  This is what makes the level kernels'
// unchecked loads safe, so a plan that fails is refused before any evaluation runs.
template <class I>
__global__ void plan_check_kernel(const I *__restrict__ trans, int64_t toff, int64_t cnt, int64_t child_lo1,
                                  int64_t child_hi1, int64_t npairs, int bits, unsigned long long *bad)
{
    const I mask = ((I)1 << bits) - 1;
    unsigned long long local = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < cnt; k += (int64_t)gridDim.x * blockDim.x) {
        I t = trans[toff + k];
        int64_t pi = (int64_t)(t & mask), ci = (int64_t)(t >> bits);
        if (t < 0 || pi < 1 || pi > npairs || ci < child_lo1 || ci > child_hi1) ++local;
    }
    if (local) atomicAdd(bad, local);
}

int plan_validate_device(const DevPlan &p, cudaStream_t st)
{
    Context &cx = ctx();
    unsigned long long *dbad = nullptr;
    EGG_CUDA_TRY(cudaMalloc(&dbad, sizeof(unsigned long long)));
    cudaError_t e = cudaMemsetAsync(dbad, 0, sizeof(unsigned long long), st);
    int bits = pair_bits(p.idx_bytes);
    int64_t npairs = (int64_t)p.K * (p.K - 1) / 2;
    for (size_t L = 1; e == cudaSuccess && L < p.levels.size(); ++L) {
        const Level &lv = p.levels[L];
        int64_t cnt = lv.n * lv.deg;
        int64_t blocks = (cnt + 255) / 256;
        int64_t cap = (int64_t)cx.num_sms * 16;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) continue;
        int64_t clo = p.levels[L - 1].lo + 1, chi = p.levels[L - 1].lo + p.levels[L - 1].n;
        if (p.idx_bytes == 4)
            plan_check_kernel<int32_t><<<(unsigned)blocks, 256, 0, st>>>((const int32_t *)p.trans, lv.toff, cnt, clo, chi,
                                                                       npairs, bits, dbad);
        else
            plan_check_kernel<int64_t><<<(unsigned)blocks, 256, 0, st>>>((const int64_t *)p.trans, lv.toff, cnt, clo, chi,
                                                                       npairs, bits, dbad);
        count_launch();
        e = cudaGetLastError();
    }
    unsigned long long bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, dbad, sizeof(bad), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dbad);
    if (e != cudaSuccess) return fail(EGG_ERR_CUDA, std::string("plan check: ") + cudaGetErrorString(e));
    if (bad) return fail(EGG_ERR_PLAN_INVALID, std::to_string(bad) + " transitions name a child outside the previous level "
                                                                     "or a pair index out of range");
    return EGG_OK;
}

}  // namespace egg
