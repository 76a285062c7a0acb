// egg_repeated.cu -- batches of hafnian_repeated(A_b, rpt_b) on the sieve, prepared on the device.
//
// For each instance the reference's CPU preparation (src/hafnian.jl:1194-1222) runs here as one
// thread of prepare_kernel:
//   * matched_reps(rpt) (:142-188): repeatedly pair the two most repeated rows (ties broken by the
//     larger row index, as the reference's sort of (count, row) pairs in descending order), or a row
//     with itself when it alone is left or outnumbers the next by more than two to one;
//   * the sieve variant (:855-884, :974-976): the exact multiply-add counts of both variants,
//     computed in the same Float64 operations and order as the reference's cost model, Glynn when
//     its count is not larger (unless the caller forces a variant);
//   * the rows x of the permuted matrix A[x, x] (_permuted, :786-792).
// gather_kernel then builds every instance's permuted matrix in the sieve's slab layout, and the
// sieve (egg_sieve.cu) evaluates the batch.  Only the compact per-instance tables (edge counts,
// multiplicities, variants) come back to the host, where the sieve's launches are planned.
#include <cstring>
#include <vector>

#include "egg_sieve.cuh"

namespace egg {

constexpr int kRepMaxRows = 64;  // rpt length (the matrix dimension d)
constexpr int kRepMaxEdges = 32;

// Per-instance result of the preparation, written by prepare_kernel.
struct RepPrep {
    int E;       // edges after matching (0 when the total is zero or odd)
    int n;       // sum of the multiplicities (half the total)
    int glynn;   // the variant
    int status;  // 0 ok; 1 odd total (the hafnian is 0); 2 more than kRepMaxEdges edges; 3 total over 126
    int reps[kRepMaxEdges];
    int x[2 * kRepMaxEdges];  // 1-based rows of the permuted matrix (x[i] pairs with x[i + E])
};

// round(x) half to even, saturated, as the reference's _clamp_work (src/hafnian.jl:832).
__device__ __forceinline__ long long clamp_work(double x)
{
    return x >= 9.0e18 ? 0x7fffffffffffffffLL : __double2ll_rn(x);
}

// _term_cost(E, n) = (5 (2E)^3) / 3 + 2 E n^2 (src/hafnian.jl:626), exact in Int64 here.
__device__ __forceinline__ long long term_cost(long long E, long long n)
{
    return (5 * (2 * E) * (2 * E) * (2 * E)) / 3 + 2 * E * n * n;
}

// _sieve_variant_cost's work (src/hafnian.jl:855-884): the same Float64 operations in the same
// order (no contraction), so the comparison of the two variants matches the reference's.
__device__ long long variant_work(const int *reps, int E, int n, bool glynn)
{
    double counts[kRepMaxEdges + 1];
    for (int c = 0; c <= E; ++c) counts[c] = 0.0;
    counts[0] = 1.0;
    for (int i = 1; i <= E; ++i) {
        const int r = reps[i - 1];
        const int total = glynn ? (i == 1 ? (r + 2) / 2 : r + 1) : r + 1;
        const int nzero = glynn ? ((r % 2 == 0) ? 1 : 0) : 1;
        const int nkeep = total - nzero;
        for (int c = i - 1; c >= 0; --c) {
            const double v = counts[c];
            if (v == 0.0) continue;
            counts[c] = __dmul_rn(v, (double)nzero);
            counts[c + 1] = __dadd_rn(counts[c + 1], __dmul_rn(v, (double)nkeep));
        }
    }
    double work = 0.0;
    for (int c = 0; c <= E; ++c) {
        if (counts[c] == 0.0) continue;
        work = __dadd_rn(work, __dmul_rn(counts[c], (double)term_cost(c, n)));
    }
    return clamp_work(work);
}

__global__ void prepare_kernel(const int64_t *__restrict__ rpts, int64_t B, int d, int force_glynn, RepPrep *__restrict__ out)
{
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= B) return;
    const int64_t *rp = rpts + b * d;
    RepPrep p;
    p.E = 0;
    p.n = 0;
    p.glynn = 0;
    p.status = 0;
    // The rows with a positive count: (count, row), row 1-based.
    int cnt[kRepMaxRows], row[kRepMaxRows], nv = 0;
    long long total = 0;
    for (int i = 0; i < d; ++i) {
        const long long c = rp[i];
        total += c;
        if (c > 0) {
            cnt[nv] = (int)(c > 0x7fffffff ? 0x7fffffff : c);
            row[nv] = i + 1;
            ++nv;
        }
    }
    if (total > 126) {
        p.status = 3;
    } else if (total & 1) {
        p.status = 1;
    } else {
        int ea[kRepMaxEdges], eb[kRepMaxEdges];
        int E = 0;
        // The greedy pairing of matched_reps: each round, the first two of (count, row) in
        // descending order.
        while (nv > 1 || (nv == 1 && cnt[0] > 1)) {
            int t1 = 0;
            for (int k = 1; k < nv; ++k)
                if (cnt[k] > cnt[t1] || (cnt[k] == cnt[t1] && row[k] > row[t1])) t1 = k;
            int t2 = -1;
            for (int k = 0; k < nv; ++k) {
                if (k == t1) continue;
                if (t2 < 0 || cnt[k] > cnt[t2] || (cnt[k] == cnt[t2] && row[k] > row[t2])) t2 = k;
            }
            if (E >= kRepMaxEdges) {
                p.status = 2;
                break;
            }
            const int reps1 = cnt[t1], x1 = row[t1];
            if (t2 < 0 || reps1 > 2 * cnt[t2]) {
                ea[E] = x1;
                eb[E] = x1;
                p.reps[E] = reps1 / 2;
                ++E;
                if (reps1 % 2 == 0) {
                    cnt[t1] = cnt[nv - 1];
                    row[t1] = row[nv - 1];
                    --nv;
                } else {
                    cnt[t1] = 1;
                }
            } else {
                const int reps2 = cnt[t2], x2 = row[t2];
                ea[E] = x1;
                eb[E] = x2;
                p.reps[E] = reps2;
                ++E;
                if (reps1 > reps2) {
                    cnt[t1] = reps1 - reps2;
                    cnt[t2] = cnt[nv - 1];
                    row[t2] = row[nv - 1];
                    --nv;
                } else {
                    // Remove both (the higher position first, so the lower stays valid).
                    const int hi = t1 > t2 ? t1 : t2, lo = t1 > t2 ? t2 : t1;
                    cnt[hi] = cnt[nv - 1];
                    row[hi] = row[nv - 1];
                    --nv;
                    cnt[lo] = cnt[nv - 1];
                    row[lo] = row[nv - 1];
                    --nv;
                }
            }
        }
        if (p.status == 0) {
            int n = 0;
            for (int e = 0; e < E; ++e) n += p.reps[e];
            for (int e = 0; e < E; ++e) {
                p.x[e] = ea[e];
                p.x[E + e] = eb[e];
            }
            p.E = E;
            p.n = n;
            if (force_glynn >= 0) p.glynn = force_glynn ? 1 : 0;
            else if (E > 0) p.glynn = variant_work(p.reps, E, n, true) <= variant_work(p.reps, E, n, false) ? 1 : 0;
        }
    }
    out[b] = p;
}

// slab[b] (lda x lda, column-major) = A_b[x, x] for each instance's rows x (2E of them).
template <class T>
__global__ void gather_kernel(const T *__restrict__ mats, int64_t mat_stride, int d, const RepPrep *__restrict__ prep,
                              int64_t B, int lda, T *__restrict__ slab)
{
    const int64_t per = (int64_t)lda * lda;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < B * per; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / per;
        const int64_t rem = t - b * per;
        const int col = (int)(rem / lda), rowi = (int)(rem - (int64_t)col * lda);
        const int m = 2 * prep[b].E;
        T v{};
        if (col < m && rowi < m) {
            const int xr = prep[b].x[rowi] - 1, xc = prep[b].x[col] - 1;
            v = mats[b * mat_stride + (int64_t)xc * d + xr];
        }
        slab[t] = v;
    }
}

// Instances whose total is odd have hafnian 0 (their sieve ran on an empty matrix).
template <class T>
__global__ void odd_zero_kernel(const RepPrep *__restrict__ prep, int64_t B, T *__restrict__ out)
{
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b < B && prep[b].status == 1) out[b] = T{};
}

static int repeated_run(int dtype, int prec, int64_t B, int64_t d, const void *dmats, int64_t mat_stride,
                        const int64_t *drpts, int glynn, void *dout, cudaStream_t st)
{
    Context &c = ctx();
    const bool cplx = dtype == EGG_C128;
    const size_t es = cplx ? 16 : 8;
    // 1. Preparation on the device; the compact tables come back for the launch planner.
    int rc = ensure_buf(c.scratch[9], (size_t)B * sizeof(RepPrep) + 256);
    if (rc) return rc;
    RepPrep *dprep = (RepPrep *)c.scratch[9].ptr;
    const unsigned pblocks = (unsigned)((B + 127) / 128);
    prepare_kernel<<<pblocks, 128, 0, st>>>(drpts, B, (int)d, glynn, dprep);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    std::vector<RepPrep> prep((size_t)B);
    EGG_CUDA_TRY(cudaMemcpyAsync(prep.data(), dprep, (size_t)B * sizeof(RepPrep), cudaMemcpyDeviceToHost, st));
    EGG_CUDA_TRY(cudaStreamSynchronize(st));
    int Emax = 0;
    for (int64_t b = 0; b < B; ++b) {
        if (prep[(size_t)b].status == 2)
            return fail(EGG_ERR_TOO_LARGE, "instance " + std::to_string(b) + " matches into more than 32 edges");
        if (prep[(size_t)b].status == 3)
            return fail(EGG_ERR_TOO_LARGE, "instance " + std::to_string(b) + " has a total over 126");
        Emax = prep[(size_t)b].E > Emax ? prep[(size_t)b].E : Emax;
    }
    std::vector<int64_t> E((size_t)B), reps((size_t)B * (Emax > 0 ? Emax : 1), 0);
    std::vector<int32_t> g((size_t)B);
    for (int64_t b = 0; b < B; ++b) {
        const RepPrep &p = prep[(size_t)b];
        E[(size_t)b] = p.E;
        g[(size_t)b] = p.glynn;
        for (int e = 0; e < p.E; ++e) reps[(size_t)b * (Emax > 0 ? Emax : 1) + e] = p.reps[e];
    }
    // 2. The permuted matrices, 3. the sieve, 4. zeros for odd totals.
    const int lda = 2 * Emax > 0 ? 2 * Emax : 1;
    rc = ensure_buf(c.scratch[3], (size_t)B * lda * lda * es + 64);
    if (rc) return rc;
    {
        const int64_t total = B * (int64_t)lda * lda;
        int64_t blocks = (total + 255) / 256, cap = (int64_t)c.num_sms * 16;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        if (cplx)
            gather_kernel<cd><<<(unsigned)blocks, 256, 0, st>>>((const cd *)dmats, mat_stride, (int)d, dprep, B, lda,
                                                                (cd *)c.scratch[3].ptr);
        else
            gather_kernel<double><<<(unsigned)blocks, 256, 0, st>>>((const double *)dmats, mat_stride, (int)d, dprep, B,
                                                                    lda, (double *)c.scratch[3].ptr);
        count_launch();
        EGG_CUDA_TRY(cudaGetLastError());
    }
    rc = sieve_batch_run(dtype, prec, B, Emax, c.scratch[3].ptr, E.data(), reps.data(), g.data(), dout, st);
    if (rc) return rc;
    if (cplx) odd_zero_kernel<cd><<<pblocks, 128, 0, st>>>(dprep, B, (cd *)dout);
    else odd_zero_kernel<double><<<pblocks, 128, 0, st>>>(dprep, B, (double *)dout);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

static int repeated_check(int dtype, int prec, int64_t B, int64_t d, int64_t mat_stride, int glynn)
{
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (prec != EGG_PREC_EXACT && prec != EGG_PREC_FMA) return fail(EGG_ERR_ARGUMENT, "the sieve takes EGG_PREC_EXACT or EGG_PREC_FMA");
    if (B < 0 || d < 0) return fail(EGG_ERR_ARGUMENT, "negative size");
    if (d > kRepMaxRows) return fail(EGG_ERR_TOO_LARGE, "rpt longer than 64 rows");
    if (B > 65535) return fail(EGG_ERR_ARGUMENT, "batch too large for one launch (max 65535)");
    if (mat_stride != 0 && mat_stride < d * d) return fail(EGG_ERR_ARGUMENT, "matrices overlap: stride below d*d");
    if (glynn < -1 || glynn > 1) return fail(EGG_ERR_ARGUMENT, "glynn must be -1 (cost model), 0 or 1");
    return EGG_OK;
}

}  // namespace egg

using namespace egg;

extern "C" int egg_sieve_repeated_batch(int dtype, int prec, int64_t B, int64_t d, const void *mats, int64_t mat_stride,
                                        const int64_t *rpts, int glynn, void *out)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    int rc = ensure_init();
    if (rc) return rc;
    rc = repeated_check(dtype, prec, B, d, mat_stride, glynn);
    if (rc) return rc;
    if (B == 0) return EGG_OK;
    if (!rpts || !out || (d > 0 && !mats)) return fail(EGG_ERR_ARGUMENT, "null argument");
    for (int64_t i = 0; i < B * d; ++i)
        if (rpts[i] < 0) return fail(EGG_ERR_ARGUMENT, "rpt contains a negative entry");
    Context &c = ctx();
    const size_t es = dtype == EGG_C128 ? 16 : 8;
    const int64_t nmats = mat_stride == 0 ? 1 : B;
    const size_t mbytes = (size_t)((nmats - 1) * mat_stride + d * d) * es, rbytes = (size_t)B * d * sizeof(int64_t);
    const size_t off_r = (mbytes + 255) / 256 * 256, off_o = off_r + (rbytes + 255) / 256 * 256;
    rc = ensure_buf(c.scratch[7], off_o + (size_t)B * es + 64);
    if (rc) return rc;
    char *base = (char *)c.scratch[7].ptr;
    if (mbytes) EGG_CUDA_TRY(cudaMemcpyAsync(base, mats, mbytes, cudaMemcpyHostToDevice, c.stream));
    if (rbytes) EGG_CUDA_TRY(cudaMemcpyAsync(base + off_r, rpts, rbytes, cudaMemcpyHostToDevice, c.stream));
    rc = repeated_run(dtype, prec, B, d, base, mat_stride, (const int64_t *)(base + off_r), glynn, base + off_o, c.stream);
    if (rc) return rc;
    EGG_CUDA_TRY(cudaMemcpyAsync(out, base + off_o, (size_t)B * es, cudaMemcpyDeviceToHost, c.stream));
    EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return EGG_OK;
}

extern "C" int egg_sieve_repeated_batch_device(int dtype, int prec, int64_t B, int64_t d, const void *mats,
                                               int64_t mat_stride, const int64_t *rpts, int glynn, void *out, void *stream)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    int rc = ensure_init();
    if (rc) return rc;
    rc = repeated_check(dtype, prec, B, d, mat_stride, glynn);
    if (rc) return rc;
    if (B == 0) return EGG_OK;
    if (!rpts || !out || (d > 0 && !mats)) return fail(EGG_ERR_ARGUMENT, "null argument");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    return repeated_run(dtype, prec, B, d, mats, mat_stride, rpts, glynn, out, st);
}
