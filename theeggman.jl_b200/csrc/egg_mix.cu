// egg_mix.cu -- hafnians of many principal submatrices of one parent matrix, of uneven degree.
//
// A Gaussian-boson-sampling workload asks for hafnians of A[r, r] for many row sets r of one
// parent A, with |r| varying from instance to instance.  The reference's batch entry takes one
// degree per call (src/hafnian.jl:1263-1301), so a caller loops over degrees and gathers the
// pair vectors on the host (_gather_pairs_batch, src/dp.jl:479-512).  Here one call takes the
// whole mix:
//   1. instances are binned by degree on the host (a stable counting sort of the row-set sizes);
//   2. one gather kernel builds every bin's pair matrix P (npairs x count, instance-fastest)
//      straight from the parent in device memory;
//   3. each bin runs the subset DP of its degree on its resident closed-form plan (dp_run);
//   4. one scatter kernel writes the results back in the caller's order (odd sizes give 0,
//      empty row sets give 1).
// Every result is the value hafnian(A[r, r]; method = :dp) gives for the same precision mode.
#include "egg_internal.cuh"

namespace egg {

static constexpr int kMaxBins = 32;  // even degrees 2..64

struct MixBin {
    int K, npairs;
    int64_t count;  // instances in the bin
    int64_t first;  // position of the bin's first instance in the sorted order
    int64_t poff;   // element offset of the bin's P
    int64_t ebase;  // gather elements before this bin
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

// P_bin[q * count + i] = A[r[qi], r[qj]] for the bin's i-th instance, q = _pair_index(qi+1, qj+1, K) - 1.
// Row indices outside [0, n) are not read: the pair gets NaN (0 for integers).
template <class T>
__global__ void mix_gather_kernel(const T *__restrict__ A, int64_t n, const int64_t *__restrict__ offsets,
                                  const int32_t *__restrict__ rows, const int32_t *__restrict__ order, MixBins bins,
                                  int64_t total, T *__restrict__ P)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        int k = 0;
        while (k + 1 < bins.nb && bins.b[k + 1].ebase <= g) ++k;
        const MixBin &bn = bins.b[k];
        const int64_t e = g - bn.ebase;
        const int64_t q = e / bn.count, i = e - q * bn.count;
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
            P[bn.poff + e] = nan_of<T>();
        } else {
            P[bn.poff + e] = A[a + c * n];
        }
    }
}

// out[order[k]] = sorted[k] for the DP instances; the trailing `nzero` entries of the order get 0
// (odd sizes) and the `none` after them 1 (empty row sets).
template <class OT>
__global__ void mix_scatter_kernel(const OT *__restrict__ sorted, const int32_t *__restrict__ order, int64_t ndp,
                                   int64_t nzero, int64_t none, OT *__restrict__ out)
{
    const int64_t total = ndp + nzero + none;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        OT v;
        if (k < ndp) v = sorted[k];
        else if (k < ndp + nzero) v = OT{};
        else v = mix_one<OT>();
        out[order[k]] = v;
    }
}

static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// The mix with A, the row indices and out in device memory and the row-set boundaries on the host.
int mix_run(int dtype, int prec, const void *dA, int64_t n, int64_t B, const int64_t *offsets, const int32_t *drows,
            void *dout, cudaStream_t st)
{
    if (dtype != EGG_F64 && dtype != EGG_C128 && dtype != EGG_I64)
        return fail(EGG_ERR_ARGUMENT, "the mixed-degree batch takes Float64, ComplexF64 or Int64 parents");
    if (dtype == EGG_I64 && prec != EGG_PREC_EXACT) return fail(EGG_ERR_ARGUMENT, "integer parents run exactly");
    if (B < 0 || n < 0) return fail(EGG_ERR_ARGUMENT, "negative size");
    if (B == 0) return EGG_OK;
    if (B > INT32_MAX) return fail(EGG_ERR_TOO_LARGE, "more than 2^31 - 1 instances");
    // 1. Bin by size: even degrees 2..64 run the DP; odd sizes give 0 and empty sets 1.
    int64_t cnt[65] = {0};
    for (int64_t b = 0; b < B; ++b) {
        const int64_t sz = offsets[b + 1] - offsets[b];
        if (sz < 0) return fail(EGG_ERR_ARGUMENT, "row-set boundaries must not decrease");
        if (sz > 64) return fail(EGG_ERR_TOO_LARGE, "a row set of " + std::to_string(sz) + " exceeds DP_HARD_MAX = 64");
        ++cnt[sz];
    }
    MixBins bins;
    bins.nb = 0;
    int64_t pos[65], ndp = 0, total = 0;
    for (int K = 2; K <= 64; K += 2) {
        if (!cnt[K]) continue;
        MixBin &bn = bins.b[bins.nb++];
        bn.K = K;
        bn.npairs = K * (K - 1) / 2;
        bn.count = cnt[K];
        bn.first = ndp;
        bn.poff = total;
        bn.ebase = total;
        pos[K] = ndp;
        ndp += cnt[K];
        total += bn.npairs * bn.count;
    }
    int64_t nzero = 0;
    for (int K = 1; K <= 63; K += 2) nzero += cnt[K];
    int64_t zpos = ndp, opos = ndp + nzero;
    std::vector<int32_t> order((size_t)B);
    for (int64_t b = 0; b < B; ++b) {
        const int64_t sz = offsets[b + 1] - offsets[b];
        if (sz == 0) order[opos++] = (int32_t)b;
        else if (sz & 1) order[zpos++] = (int32_t)b;
        else order[pos[sz]++] = (int32_t)b;
    }
    // 2. Plans and buffers: every bin's work buffers are sized before anything is enqueued, so no
    // buffer is reallocated while an earlier bin's kernels may still be running.
    const size_t es = dtype_size(dtype), oes = dtype == EGG_I64 ? 16 : es;
    size_t hmax = 0, p32max = 0;
    std::vector<DevPlan *> plans;
    for (int k = 0; k < bins.nb; ++k) {
        int rc = EGG_OK;
        DevPlan *pl = dp_plan_for(bins.b[k].K, &rc);
        if (!pl) return rc;
        plans.push_back(pl);
        const size_t h = dp_scratch_bytes(*pl, dtype, prec, bins.b[k].count);
        hmax = h > hmax ? h : hmax;
        const size_t p32 = (size_t)bins.b[k].npairs * bins.b[k].count * (dtype == EGG_C128 ? 2 : 1) * sizeof(float);
        p32max = p32 > p32max ? p32 : p32max;
    }
    Context &c = ctx();
    const size_t off_o = align256((size_t)(B + 1) * 8), off_p = off_o + align256((size_t)B * 4);
    const size_t off_r = off_p + align256((size_t)total * es), arena = off_r + align256((size_t)(ndp ? ndp : 1) * oes);
    int rc = ensure_buf(c.scratch[6], arena);
    if (!rc && hmax) rc = ensure_buf(c.scratch[0], hmax);
    if (!rc && prec == EGG_PREC_MIXED && p32max) rc = ensure_buf(c.scratch[5], p32max);
    if (rc) return rc;
    char *base = (char *)c.scratch[6].ptr;
    int64_t *doff = (int64_t *)base;
    int32_t *dorder = (int32_t *)(base + off_o);
    char *dP = base + off_p, *dsorted = base + off_r;
    EGG_CUDA_TRY(cudaMemcpyAsync(doff, offsets, (size_t)(B + 1) * 8, cudaMemcpyHostToDevice, st));
    EGG_CUDA_TRY(cudaMemcpyAsync(dorder, order.data(), (size_t)B * 4, cudaMemcpyHostToDevice, st));
    // 3. Gather, 4. DP per bin, 5. scatter.
    if (total > 0) {
        int64_t blocks = (total + 255) / 256, cap = (int64_t)c.num_sms * 16;
        if (blocks > cap) blocks = cap;
        if (dtype == EGG_F64)
            mix_gather_kernel<double><<<(unsigned)blocks, 256, 0, st>>>((const double *)dA, n, doff, drows, dorder, bins, total,
                                                                        (double *)dP);
        else if (dtype == EGG_C128)
            mix_gather_kernel<cd><<<(unsigned)blocks, 256, 0, st>>>((const cd *)dA, n, doff, drows, dorder, bins, total, (cd *)dP);
        else
            mix_gather_kernel<int64_t><<<(unsigned)blocks, 256, 0, st>>>((const int64_t *)dA, n, doff, drows, dorder, bins,
                                                                         total, (int64_t *)dP);
        count_launch();
        EGG_CUDA_TRY(cudaGetLastError());
    }
    for (int k = 0; k < bins.nb; ++k) {
        const MixBin &bn = bins.b[k];
        rc = dp_run(*plans[k], dtype, prec, dP + (size_t)bn.poff * es, bn.count, dsorted + (size_t)bn.first * oes, st);
        if (rc) return rc;
    }
    {
        int64_t blocks = (B + 255) / 256, cap = (int64_t)c.num_sms * 16;
        if (blocks > cap) blocks = cap;
        if (dtype == EGG_F64)
            mix_scatter_kernel<double><<<(unsigned)blocks, 256, 0, st>>>((const double *)dsorted, dorder, ndp, nzero,
                                                                         B - ndp - nzero, (double *)dout);
        else if (dtype == EGG_C128)
            mix_scatter_kernel<cd><<<(unsigned)blocks, 256, 0, st>>>((const cd *)dsorted, dorder, ndp, nzero, B - ndp - nzero,
                                                                     (cd *)dout);
        else
            mix_scatter_kernel<__int128><<<(unsigned)blocks, 256, 0, st>>>((const __int128 *)dsorted, dorder, ndp, nzero,
                                                                           B - ndp - nzero, (__int128 *)dout);
        count_launch();
        EGG_CUDA_TRY(cudaGetLastError());
    }
    return EGG_OK;
}

}  // namespace egg
