// egg_api.cu -- the C ABI of libeggman_b200: context, lock, plan cache, reusable device buffers,
// and the host-pointer entry points that stage data in and out of device memory.
//
// The cache/lock structure mirrors the reference's device caches (src/dp.jl:536-573): plans keyed
// by (degree, layout) and never evicted, work buffers grown on demand and reused, one lock so that
// one call at a time uses the shared buffers (ext/TheEggmanKernelAbstractionsExt.jl:117-119).
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "egg_internal.cuh"
#include "egg_mix.cuh"

namespace egg {

static thread_local std::string t_err;
std::atomic<long long> g_launches{0};

void set_error(const std::string &msg) { t_err = msg; }
int fail(int code, const std::string &msg)
{
    t_err = msg;
    return code;
}

Context &ctx()
{
    static Context c;
    return c;
}

int ensure_init()
{
    Context &c = ctx();
    if (c.device >= 0) return EGG_OK;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(EGG_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    EGG_CUDA_TRY(cudaSetDevice(0));
    int rc = create_streams(c, 0);
    if (rc) return rc;
    c.device = 0;
    return EGG_OK;
}

int create_streams(Context &c, int device)
{
    EGG_CUDA_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    EGG_CUDA_TRY(cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming));
    for (int i = 0; i < Context::kSideStreams; ++i) {
        EGG_CUDA_TRY(cudaStreamCreateWithFlags(&c.side[i], cudaStreamNonBlocking));
        EGG_CUDA_TRY(cudaEventCreateWithFlags(&c.join_ev[i], cudaEventDisableTiming));
    }
    EGG_CUDA_TRY(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, device));
    return EGG_OK;
}

int smem_limit_at_least(const void *k, size_t bytes)
{
    // Own lock: the entry point that allocates nothing reaches this without the library's lock.
    // A kernel's attribute is set per device, so the record is kept per (device, kernel).
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    static std::map<std::pair<int, const void *>, size_t> done;
    int dev = -1;
    EGG_CUDA_TRY(cudaGetDevice(&dev));
    const auto key = std::make_pair(dev, k);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return EGG_OK;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[key] = bytes;
    return EGG_OK;
}

int blocks_per_sm(const void *k, int threads, size_t smem, int *out)
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    static std::map<std::tuple<int, const void *, int, size_t>, int> done;
    int dev = -1;
    EGG_CUDA_TRY(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, k, threads, smem);
    auto it = done.find(key);
    if (it != done.end()) {
        *out = it->second;
        return EGG_OK;
    }
    int nb = 0;
    EGG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, threads, smem));
    done[key] = nb;
    *out = nb;
    return EGG_OK;
}

int ensure_buf(DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes && b.ptr) return EGG_OK;
    if (b.ptr) {
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        cudaGetLastError();
        return fail(EGG_ERR_TOO_LARGE, "device allocation of " + std::to_string(want) + " bytes failed: " +
                                           cudaGetErrorString(e));
    }
    b.bytes = want;
    return EGG_OK;
}

DevPlan *find_plan(int K, int idx_bytes)
{
    auto it = ctx().plans.find({K, idx_bytes});
    return it == ctx().plans.end() ? nullptr : &it->second;
}

static int64_t binom64(int64_t n, int64_t k)
{
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    __int128 r = 1;
    for (int64_t i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return (int64_t)r;
}

void dp_counts(int K, int64_t &nstates, int64_t &ntrans)
{
    // _dp_counts(K), src/dp.jl:192-208.
    int64_t ns = 1, nt = 0;
    for (int p = 1; p <= K; ++p) {
        int lo = p - 1, hi = 2 * (p - 1) < K - 1 ? 2 * (p - 1) : K - 1;
        for (int r = (lo % 2 == 0) ? lo : lo + 1; r <= hi; r += 2) {
            int64_t k = K - r - 1, c = binom64(K - p, k);
            ns += c;
            nt += c * k;
        }
    }
    nstates = ns;
    ntrans = nt;
}

}  // namespace egg

using namespace egg;

#define EGG_GUARD()                                         \
    std::lock_guard<std::recursive_mutex> lk_(ctx().mu);    \
    do {                                                    \
        int rc_ = ensure_init();                            \
        if (!rc_) rc_ = check_current_device();             \
        if (rc_) return rc_;                                \
    } while (0)

// The library's context (streams, plans, work buffers) belongs to one device, the one egg_init
// bound (device 0 if egg_init was not called).  A call from a thread whose current device is
// another one is refused instead of handing that device's kernels this device's memory.
static int check_current_device()
{
    int dev = -1;
    EGG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != ctx().device)
        return fail(EGG_ERR_ARGUMENT, "the library is bound to device " + std::to_string(ctx().device) +
                                          " but the calling thread's current device is " + std::to_string(dev));
    return EGG_OK;
}

static int check_layout(int K, int idx_bytes);

DevPlan *egg::dp_plan_for(int K, int *rc)
{
    const int ib = K <= 32 ? 4 : 8;  // _dp_index_type: Int32 through DP_MAX = 32 (src/dp.jl:180)
    DevPlan *p = find_plan(K, ib);
    if (p) return p;
    *rc = check_layout(K, ib);
    if (*rc) return nullptr;
    DevPlan np;
    *rc = plan_levels(K, ib, np);
    if (*rc) return nullptr;
    ctx().plans[{K, ib}] = std::move(np);
    return find_plan(K, ib);
}

static int check_layout(int K, int idx_bytes)
{
    // The reference's refusals, src/dp.jl:224-234.
    if (K < 0 || K > 64) return fail(EGG_ERR_TOO_LARGE, "degree " + std::to_string(K) + " exceeds DP_HARD_MAX = 64");
    if (idx_bytes != 4 && idx_bytes != 8) return fail(EGG_ERR_ARGUMENT, "idx_bytes must be 4 or 8");
    int64_t ns, nt;
    dp_counts(K, ns, nt);
    int bits = pair_bits(idx_bytes);
    int64_t npairs = (int64_t)K * (K - 1) / 2;
    int64_t imax = idx_bytes == 4 ? INT32_MAX : INT64_MAX;
    if (npairs > ((int64_t)1 << bits) - 1)
        return fail(EGG_ERR_TOO_LARGE, "degree " + std::to_string(K) + " needs more than " + std::to_string(bits) +
                                           " bits per pair index");
    if (ns > (imax >> bits))
        return fail(EGG_ERR_TOO_LARGE, "degree " + std::to_string(K) + " has too many states to pack");
    if (nt > imax) return fail(EGG_ERR_TOO_LARGE, "degree " + std::to_string(K) + " has too many transitions");
    return EGG_OK;
}

extern "C" {

const char *egg_version(void) { return "eggman_b200 0.1.0 (sm_100a)"; }

const char *egg_last_error(void) { return t_err.c_str(); }

int64_t egg_launch_count(void) { return (int64_t)g_launches.load(std::memory_order_relaxed); }

int egg_init(int device)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    Context &c = ctx();
    if (c.device >= 0) {
        if (device != c.device) return fail(EGG_ERR_ARGUMENT, "the library is bound to device " + std::to_string(c.device));
        return EGG_OK;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(EGG_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= n) return fail(EGG_ERR_ARGUMENT, "device index out of range");
    EGG_CUDA_TRY(cudaSetDevice(device));
    int rc = create_streams(c, device);
    if (rc) return rc;
    c.device = device;
    return EGG_OK;
}

int64_t egg_cache_bytes(void)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    int64_t total = 0;
    for (auto &kv : ctx().plans) total += kv.second.bytes();
    for (auto &b : ctx().scratch) total += (int64_t)b.bytes;
    return total;
}

int egg_cache_clear(void)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    Context &c = ctx();
    if (c.device >= 0) cudaStreamSynchronize(c.stream);
    mix_graphs_clear();
    for (auto &kv : c.plans) release_plan_memory(kv.second);
    c.plans.clear();
    for (auto &b : c.scratch) {
        if (b.ptr) cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    return EGG_OK;
}

int64_t egg_dp_batch_bytes(int N, int dtype, int64_t B)
{
    // dp_batch_bytes(N, T, B), src/dp.jl:584-587: B x (nstates + npairs) x sizeof(T).  The
    // engine keeps only two levels of states live, so this is an upper bound on what it uses.
    if (N < 0 || N > 64 || B < 0) return -1;
    size_t es = dtype_size(dtype);
    if (!es) return -1;
    int64_t ns, nt;
    dp_counts(N, ns, nt);
    return B * (ns + (int64_t)N * (N - 1) / 2) * (int64_t)es;
}

int egg_dp_counts(int K, int64_t *nstates, int64_t *ntrans)
{
    if (K < 0 || K > 64 || !nstates || !ntrans) return fail(EGG_ERR_ARGUMENT, "bad arguments to egg_dp_counts");
    dp_counts(K, *nstates, *ntrans);
    return EGG_OK;
}

int egg_plan_upload(int K, int idx_bytes, const void *starts, const void *trans, const void *levels,
                    int64_t nlevels, int64_t nstates, int64_t ntrans)
{
    EGG_GUARD();
    int rc = check_layout(K, idx_bytes);
    if (rc) return rc;
    if (find_plan(K, idx_bytes)) return EGG_OK;  // idempotent, as _device_plan's get!
    if (!starts || !levels || (ntrans > 0 && !trans)) return fail(EGG_ERR_ARGUMENT, "null plan array");
    int64_t ns_expect, nt_expect;
    dp_counts(K, ns_expect, nt_expect);
    if (K % 2 != 0 || K < 2) return fail(EGG_ERR_ARGUMENT, "device plans are built for even degrees >= 2");
    if (nstates != ns_expect || ntrans != nt_expect || nlevels != K / 2 + 2)
        return fail(EGG_ERR_DIMENSION, "plan sizes do not match _dp_counts(" + std::to_string(K) + ")");
    auto ld = [&](const void *a, int64_t i) -> int64_t {
        return idx_bytes == 4 ? (int64_t)((const int32_t *)a)[i] : ((const int64_t *)a)[i];
    };
    DevPlan p;
    p.K = K;
    p.idx_bytes = idx_bytes;
    p.nstates = nstates;
    p.ntrans = ntrans;
    // Levels and the uniform out-degree of each (the structure the kernels rely on).
    if (ld(levels, 0) != 1 || ld(levels, nlevels - 1) != nstates + 1 || ld(starts, 0) != 1 ||
        ld(starts, nstates) != ntrans + 1)
        return fail(EGG_ERR_PLAN_INVALID, "plan bounds are inconsistent");
    for (int64_t L = 0; L + 1 < nlevels; ++L) {
        int64_t lo = ld(levels, L) - 1, hi = ld(levels, L + 1) - 1;  // 0-based [lo, hi)
        if (hi <= lo) return fail(EGG_ERR_PLAN_INVALID, "empty plan level");
        Level lv;
        lv.lo = lo;
        lv.n = hi - lo;
        lv.toff = ld(starts, lo) - 1;
        lv.deg = (int)(ld(starts, lo + 1) - ld(starts, lo));
        if (lv.deg != (L == 0 ? 0 : 2 * (int)L - 1))
            return fail(EGG_ERR_PLAN_INVALID, "level " + std::to_string(L) + " has the wrong out-degree");
        for (int64_t s = lo; s < hi; ++s)
            if (ld(starts, s + 1) - ld(starts, s) != lv.deg)
                return fail(EGG_ERR_PLAN_INVALID, "out-degree varies within level " + std::to_string(L));
        p.levels.push_back(lv);
        p.level_starts.push_back(ld(levels, L));
    }
    p.level_starts.push_back(ld(levels, nlevels - 1));
    size_t bytes = (size_t)ntrans * idx_bytes;
    cudaError_t e = cudaMalloc(&p.trans, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(EGG_ERR_TOO_LARGE, "device allocation of the plan failed: " + std::string(cudaGetErrorString(e)));
    }
    if (bytes) {
        e = cudaMemcpyAsync(p.trans, trans, bytes, cudaMemcpyHostToDevice, ctx().stream);
        if (e != cudaSuccess) {
            cudaFree(p.trans);
            return fail(EGG_ERR_CUDA, std::string("plan upload: ") + cudaGetErrorString(e));
        }
    }
    rc = plan_validate_device(p, ctx().stream);
    bool same = false;
    if (!rc) rc = plan_is_closed_form(p, ctx().stream, &same);
    if (rc) {
        cudaStreamSynchronize(ctx().stream);
        cudaFree(p.trans);
        return rc;
    }
    if (same) {
        // The uploaded plan is _build_dp_plan's layout: evaluate it in closed form and drop the
        // array (the results are the same entry for entry; only the memory traffic differs).
        cudaFree(p.trans);
        p.trans = nullptr;
    }
    ctx().plans[{K, idx_bytes}] = std::move(p);
    return EGG_OK;
}

int egg_plan_build(int K, int idx_bytes)
{
    EGG_GUARD();
    int rc = check_layout(K, idx_bytes);
    if (rc) return rc;
    if (K % 2 != 0 || K < 2) return fail(EGG_ERR_ARGUMENT, "device plans are built for even degrees >= 2");
    if (find_plan(K, idx_bytes)) return EGG_OK;
    DevPlan p;
    rc = plan_levels(K, idx_bytes, p);
    if (rc) return rc;
    ctx().plans[{K, idx_bytes}] = std::move(p);
    return EGG_OK;
}

int egg_plan_info(int K, int idx_bytes, int64_t *nstates, int64_t *ntrans, int64_t *nlevels, int64_t *device_bytes)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    DevPlan *p = find_plan(K, idx_bytes);
    if (!p) return fail(EGG_ERR_NO_PLAN, "no resident plan for degree " + std::to_string(K));
    if (nstates) *nstates = p->nstates;
    if (ntrans) *ntrans = p->ntrans;
    if (nlevels) *nlevels = (int64_t)p->level_starts.size();
    if (device_bytes) *device_bytes = p->bytes();
    return EGG_OK;
}

int egg_plan_download(int K, int idx_bytes, void *starts, void *trans, void *levels)
{
    EGG_GUARD();
    DevPlan *p = find_plan(K, idx_bytes);
    if (!p) return fail(EGG_ERR_NO_PLAN, "no resident plan for degree " + std::to_string(K));
    auto st = [&](void *a, int64_t i, int64_t v) {
        if (idx_bytes == 4) ((int32_t *)a)[i] = (int32_t)v;
        else ((int64_t *)a)[i] = v;
    };
    if (levels)
        for (size_t i = 0; i < p->level_starts.size(); ++i) st(levels, (int64_t)i, p->level_starts[i]);
    if (starts) {
        st(starts, 0, 1);
        for (const Level &lv : p->levels)
            for (int64_t s = 0; s < lv.n; ++s) st(starts, lv.lo + s + 1, lv.toff + (s + 1) * lv.deg + 1);
    }
    if (trans && p->ntrans) {
        const size_t bytes = (size_t)p->ntrans * idx_bytes;
        if (p->closed_form()) {
            // Written out on request into a temporary device array.
            void *tmp = nullptr;
            cudaError_t e = cudaMalloc(&tmp, bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(EGG_ERR_TOO_LARGE, "writing out the plan needs " + std::to_string(bytes) + " device bytes: " +
                                                   cudaGetErrorString(e));
            }
            int rc = plan_materialize(*p, tmp, ctx().stream);
            if (!rc) {
                e = cudaMemcpy(trans, tmp, bytes, cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) rc = fail(EGG_ERR_CUDA, std::string("plan download: ") + cudaGetErrorString(e));
            }
            cudaFree(tmp);
            return rc;
        }
        EGG_CUDA_TRY(cudaMemcpyAsync(trans, p->trans, bytes, cudaMemcpyDeviceToHost, ctx().stream));
        EGG_CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    }
    return EGG_OK;
}

int egg_plan_release(int K, int idx_bytes)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    auto it = ctx().plans.find({K, idx_bytes});
    if (it == ctx().plans.end()) return fail(EGG_ERR_NO_PLAN, "no resident plan for degree " + std::to_string(K));
    cudaStreamSynchronize(ctx().stream);
    mix_graphs_clear();  // recorded mixed-degree batches may read this plan's arrays
    release_plan_memory(it->second);
    ctx().plans.erase(it);
    return EGG_OK;
}

static size_t state_out_size(int dtype) { return dtype == EGG_I64 ? 16 : dtype_size(dtype); }

// The page-locked staging buffer of small synchronous calls, mapped into the device's address
// space (pinned_dev), allocated on first use.
static int ensure_pinned()
{
    Context &c = ctx();
    if (c.pinned) return EGG_OK;
    EGG_CUDA_TRY(cudaHostAlloc(&c.pinned, Context::kPinnedBytes, cudaHostAllocMapped));
    cudaError_t e = cudaHostGetDevicePointer(&c.pinned_dev, c.pinned, 0);
    if (e != cudaSuccess) {
        cudaFreeHost(c.pinned);
        c.pinned = nullptr;
        return fail(EGG_ERR_CUDA, std::string("mapping the staging buffer: ") + cudaGetErrorString(e));
    }
    return EGG_OK;
}

int egg_dp_batch(int K, int idx_bytes, int dtype, int prec, const void *P, int64_t B, int64_t max_batch, void *out)
{
    EGG_GUARD();
    if (B < 0) return fail(EGG_ERR_ARGUMENT, "negative batch size");
    if (B == 0) return EGG_OK;
    if (!P || !out) return fail(EGG_ERR_ARGUMENT, "null P or out");
    size_t es = dtype_size(dtype);
    if (!es) return fail(EGG_ERR_ARGUMENT, "unknown dtype");
    DevPlan *plan = find_plan(K, idx_bytes);
    if (!plan) return fail(EGG_ERR_NO_PLAN, "no resident plan for degree " + std::to_string(K) + "; upload or build it first");
    Context &c = ctx();
    int64_t chunk = (max_batch > 0 && max_batch < B) ? max_batch : B;
    int64_t npairs = (int64_t)K * (K - 1) / 2;
    size_t oes = state_out_size(dtype);
    const size_t per = dp_scratch_bytes(*plan, dtype, prec, 1) + (size_t)npairs * es * 2 + oes;
    const size_t held = c.scratch[0].bytes + c.scratch[1].bytes + c.scratch[2].bytes;
    if (max_batch <= 0 && per * (size_t)B > held && per * (size_t)B > ((size_t)1 << 30)) {
        // The reference leaves chunking to the caller (src/dp.jl:581-582).  Here the free device
        // memory is known, so an unchunked batch of more than 1 GiB is split to fit half of it.
        size_t free_b = 0, total_b = 0;
        EGG_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        int64_t fit = (int64_t)((free_b + held) / 2 / (per ? per : 1));
        if (fit < 1) return fail(EGG_ERR_TOO_LARGE, "one instance's work buffers do not fit in device memory");
        if (chunk > fit) chunk = fit;
    }
    int rc = ensure_buf(c.scratch[1], (size_t)chunk * npairs * es);
    if (rc) return rc;
    rc = ensure_buf(c.scratch[2], (size_t)chunk * oes);
    if (rc) return rc;
    const size_t in_bytes = (size_t)B * npairs * es, out_bytes = (size_t)B * oes;
    if (chunk == B && in_bytes + out_bytes + 256 <= Context::kPinnedBytes) {
        // A small call: both transfers through the page-locked staging buffer.
        rc = ensure_pinned();
        if (rc) return rc;
        char *pin_in = (char *)c.pinned, *pin_out = pin_in + ((in_bytes + 255) / 256) * 256;
        if (B == 1) {
            // One instance of a small degree: its pairs travel in the launch and its value is
            // written straight into the mapped staging buffer, so neither copy is needed.
            rc = dp_run_one_host(*plan, dtype, prec, P, (char *)c.pinned_dev + (pin_out - pin_in), c.stream);
            if (rc == EGG_OK) {
                EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
                std::memcpy(out, pin_out, out_bytes);
                return EGG_OK;
            }
            if (rc != kDpNotHere) return rc;
        }
        if (in_bytes) {
            std::memcpy(pin_in, P, in_bytes);
            EGG_CUDA_TRY(cudaMemcpyAsync(c.scratch[1].ptr, pin_in, in_bytes, cudaMemcpyHostToDevice, c.stream));
        }
        rc = dp_run(*plan, dtype, prec, c.scratch[1].ptr, B, c.scratch[2].ptr, c.stream);
        if (rc) return rc;
        EGG_CUDA_TRY(cudaMemcpyAsync(pin_out, c.scratch[2].ptr, out_bytes, cudaMemcpyDeviceToHost, c.stream));
        EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
        std::memcpy(out, pin_out, out_bytes);
        return EGG_OK;
    }
    for (int64_t b0 = 0; b0 < B; b0 += chunk) {
        int64_t nb = B - b0 < chunk ? B - b0 : chunk;
        // This chunk's pairs, re-laid with the chunk's own instance count as leading dimension
        // (the host transpose of ext/TheEggmanKernelAbstractionsExt.jl:127-130, done as one
        // strided copy).
        // An unchunked batch is already in that layout and goes as one contiguous copy: a 2-D
        // copy of short rows from pageable memory costs one staged transfer per row.
        if (npairs > 0 && nb == B)
            EGG_CUDA_TRY(cudaMemcpyAsync(c.scratch[1].ptr, P, (size_t)B * npairs * es, cudaMemcpyHostToDevice, c.stream));
        else if (npairs > 0)
            EGG_CUDA_TRY(cudaMemcpy2DAsync(c.scratch[1].ptr, nb * es, (const char *)P + b0 * es, B * es, nb * es, npairs,
                                           cudaMemcpyHostToDevice, c.stream));
        rc = dp_run(*plan, dtype, prec, c.scratch[1].ptr, nb, c.scratch[2].ptr, c.stream);
        if (rc) return rc;
        EGG_CUDA_TRY(cudaMemcpyAsync((char *)out + b0 * oes, c.scratch[2].ptr, nb * oes, cudaMemcpyDeviceToHost, c.stream));
    }
    EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return EGG_OK;
}

int egg_dp_batch_device(int K, int idx_bytes, int dtype, int prec, const void *P, int64_t B, void *out, void *stream)
{
    EGG_GUARD();
    if (B < 0) return fail(EGG_ERR_ARGUMENT, "negative batch size");
    if (B == 0) return EGG_OK;
    if (!dtype_size(dtype)) return fail(EGG_ERR_ARGUMENT, "unknown dtype");
    DevPlan *plan = find_plan(K, idx_bytes);
    if (!plan) return fail(EGG_ERR_NO_PLAN, "no resident plan for degree " + std::to_string(K));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    return dp_run(*plan, dtype, prec, P, B, out, st);
}

int egg_sieve(int dtype, int prec, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn, void *out)
{
    EGG_GUARD();
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (E < 0 || E > 32) return fail(EGG_ERR_TOO_LARGE, "the device sieve supports up to 32 edges (N <= 64)");
    if (!out || (E > 0 && (!Ax || !edge_reps))) return fail(EGG_ERR_ARGUMENT, "null argument");
    Context &c = ctx();
    size_t es = dtype_size(dtype);
    size_t abytes = (size_t)(2 * E) * (2 * E) * es;
    int rc = ensure_buf(c.scratch[3], abytes + 64);
    if (rc) return rc;
    rc = ensure_buf(c.scratch[4], 64);
    if (rc) return rc;
    if (abytes + 512 <= Context::kPinnedBytes / 2) {
        // A small call: the matrix and the launch's tables go through the page-locked staging
        // buffer, and the result is written straight into it (it is mapped), so no copy follows.
        rc = ensure_pinned();
        if (rc) return rc;
        char *pin = (char *)c.pinned;
        const size_t out_off = Context::kPinnedBytes - 256, stage_off = ((abytes + 255) / 256) * 256;
        if (abytes) {
            std::memcpy(pin, Ax, abytes);
            EGG_CUDA_TRY(cudaMemcpyAsync(c.scratch[3].ptr, pin, abytes, cudaMemcpyHostToDevice, c.stream));
        }
        rc = sieve_run(dtype, prec, c.scratch[3].ptr, E, edge_reps, glynn, (char *)c.pinned_dev + out_off, c.stream,
                       pin + stage_off, out_off - stage_off);
        if (rc) return rc;
        EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
        std::memcpy(out, pin + out_off, es);
        return EGG_OK;
    }
    if (abytes) EGG_CUDA_TRY(cudaMemcpyAsync(c.scratch[3].ptr, Ax, abytes, cudaMemcpyHostToDevice, c.stream));
    rc = sieve_run(dtype, prec, c.scratch[3].ptr, E, edge_reps, glynn, c.scratch[4].ptr, c.stream);
    if (rc) return rc;
    EGG_CUDA_TRY(cudaMemcpyAsync(out, c.scratch[4].ptr, es, cudaMemcpyDeviceToHost, c.stream));
    EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return EGG_OK;
}

int egg_sieve_device(int dtype, int prec, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn, void *out,
                     void *stream)
{
    EGG_GUARD();
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (E < 0 || E > 32) return fail(EGG_ERR_TOO_LARGE, "the device sieve supports up to 32 edges (N <= 64)");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    return sieve_run(dtype, prec, Ax, E, edge_reps, glynn, out, st);
}

int egg_sieve_batch(int dtype, int prec, int64_t B, int64_t Emax, const void *Ax, const int64_t *E,
                    const int64_t *edge_reps, const int32_t *glynn, void *out)
{
    EGG_GUARD();
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (B < 0 || Emax < 0 || Emax > 32) return fail(EGG_ERR_ARGUMENT, "bad batch shape");
    if (B == 0) return EGG_OK;
    if (!Ax || !E || !edge_reps || !glynn || !out) return fail(EGG_ERR_ARGUMENT, "null argument");
    for (int64_t b = 0; b < B; ++b)
        if (E[b] < 0 || E[b] > Emax) return fail(EGG_ERR_DIMENSION, "instance edge count exceeds Emax");
    Context &c = ctx();
    size_t es = dtype_size(dtype);
    size_t abytes = (size_t)B * (2 * Emax) * (2 * Emax) * es;
    int rc = ensure_buf(c.scratch[3], abytes + 64);
    if (rc) return rc;
    rc = ensure_buf(c.scratch[4], (size_t)B * es + 64);
    if (rc) return rc;
    if (abytes) EGG_CUDA_TRY(cudaMemcpyAsync(c.scratch[3].ptr, Ax, abytes, cudaMemcpyHostToDevice, c.stream));
    rc = sieve_batch_run(dtype, prec, B, Emax, c.scratch[3].ptr, E, edge_reps, glynn, c.scratch[4].ptr, c.stream);
    if (rc) return rc;
    EGG_CUDA_TRY(cudaMemcpyAsync(out, c.scratch[4].ptr, (size_t)B * es, cudaMemcpyDeviceToHost, c.stream));
    EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return EGG_OK;
}

int egg_sieve_batch_device(int dtype, int prec, int64_t B, int64_t Emax, const void *Ax, const int64_t *E,
                           const int64_t *edge_reps, const int32_t *glynn, void *out, void *stream)
{
    EGG_GUARD();
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (B < 0 || Emax < 0 || Emax > 32) return fail(EGG_ERR_ARGUMENT, "bad batch shape");
    if (B == 0) return EGG_OK;
    if (!Ax || !E || !edge_reps || !glynn || !out) return fail(EGG_ERR_ARGUMENT, "null argument");
    for (int64_t b = 0; b < B; ++b)
        if (E[b] < 0 || E[b] > Emax) return fail(EGG_ERR_DIMENSION, "instance edge count exceeds Emax");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    return sieve_batch_run(dtype, prec, B, Emax, Ax, E, edge_reps, glynn, out, st);
}

int egg_dp_mix(int dtype, int prec, const void *A, int64_t n, int64_t B, const int64_t *offsets, const int32_t *rows,
               void *out)
{
    EGG_GUARD();
    if (B < 0 || n < 0) return fail(EGG_ERR_ARGUMENT, "negative size");
    if (B == 0) return EGG_OK;
    if (!offsets || !out || (n > 0 && !A)) return fail(EGG_ERR_ARGUMENT, "null argument");
    if (offsets[0] != 0) return fail(EGG_ERR_ARGUMENT, "offsets[0] must be 0");
    const int64_t nrows = offsets[B];
    if (nrows < 0) return fail(EGG_ERR_ARGUMENT, "row-set boundaries must not decrease");
    if (nrows > 0 && !rows) return fail(EGG_ERR_ARGUMENT, "null rows");
    for (int64_t i = 0; i < nrows; ++i)
        if (rows[i] < 0 || rows[i] >= n)
            return fail(EGG_ERR_ARGUMENT, "row index " + std::to_string(rows[i]) + " outside the " + std::to_string(n) +
                                              " x " + std::to_string(n) + " parent");
    const size_t es = dtype_size(dtype);
    if (!es) return fail(EGG_ERR_ARGUMENT, "unknown dtype");
    const size_t oes = dtype == EGG_I64 ? 16 : es;
    Context &c = ctx();
    const size_t abytes = (size_t)n * n * es, offr = (abytes + 255) / 256 * 256;
    const size_t offo = offr + ((size_t)nrows * 4 + 255) / 256 * 256;
    int rc = ensure_buf(c.scratch[7], offo + (size_t)B * oes);
    if (rc) return rc;
    char *base = (char *)c.scratch[7].ptr;
    if (abytes) EGG_CUDA_TRY(cudaMemcpyAsync(base, A, abytes, cudaMemcpyHostToDevice, c.stream));
    if (nrows) EGG_CUDA_TRY(cudaMemcpyAsync(base + offr, rows, (size_t)nrows * 4, cudaMemcpyHostToDevice, c.stream));
    rc = mix_persistent_take_timeout();  // an earlier asynchronous mix that gave up at a barrier
    if (rc) return rc;
    rc = mix_run(dtype, prec, base, n, B, offsets, (const int32_t *)(base + offr), base + offo, c.stream);
    if (rc) return rc;
    EGG_CUDA_TRY(cudaMemcpyAsync(out, base + offo, (size_t)B * oes, cudaMemcpyDeviceToHost, c.stream));
    EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return mix_persistent_take_timeout();
}

int egg_dp_mix_device(int dtype, int prec, const void *A, int64_t n, int64_t B, const int64_t *offsets, const int32_t *rows,
                      void *out, void *stream)
{
    EGG_GUARD();
    if (B < 0 || n < 0) return fail(EGG_ERR_ARGUMENT, "negative size");
    if (B == 0) return EGG_OK;
    if (!offsets || !out || (n > 0 && !A) || (offsets[B] > 0 && !rows)) return fail(EGG_ERR_ARGUMENT, "null argument");
    if (offsets[0] != 0) return fail(EGG_ERR_ARGUMENT, "offsets[0] must be 0");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    const int rc = mix_persistent_take_timeout();  // an earlier asynchronous mix that gave up at a barrier
    if (rc) return rc;
    return mix_run(dtype, prec, A, n, B, offsets, rows, out, st);
}

int egg_dp_mix_set_engine(int engine)
{
    std::lock_guard<std::recursive_mutex> lk(ctx().mu);
    return mix_set_engine(engine);
}

int egg_dp_mix_engine(void) { return mix_engine(); }

int egg_selfcheck_barrier(int extra, int64_t wait_ns, int64_t *passes)
{
    EGG_GUARD();
    return barrier_selfcheck(extra, wait_ns, passes);
}

int egg_dp_mix_set_tuning(int K, int dtype, int prec, int batched, int64_t group)
{
    return mix_set_tuning(K, dtype, prec, batched, group);
}

int egg_dp_mix_tuning(int K, int dtype, int prec, int *batched, int64_t *group)
{
    if (!batched || !group) return fail(EGG_ERR_ARGUMENT, "null argument");
    return mix_tuned(K, dtype, prec, batched, group);
}

int egg_sieve_reference_sum(int dtype, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn, int64_t nchunks,
                            void *out)
{
    EGG_GUARD();
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (E < 0 || E > 32) return fail(EGG_ERR_TOO_LARGE, "the device sieve supports up to 32 edges (N <= 64)");
    if (!out || (E > 0 && (!Ax || !edge_reps))) return fail(EGG_ERR_ARGUMENT, "null argument");
    Context &c = ctx();
    const size_t es = dtype_size(dtype);
    const size_t abytes = (size_t)(2 * E) * (2 * E) * es;
    int rc = ensure_buf(c.scratch[3], abytes + 64);
    if (!rc) rc = ensure_buf(c.scratch[4], 64);
    if (rc) return rc;
    if (abytes) EGG_CUDA_TRY(cudaMemcpyAsync(c.scratch[3].ptr, Ax, abytes, cudaMemcpyHostToDevice, c.stream));
    rc = sieve_reference_sum_run(dtype, c.scratch[3].ptr, E, edge_reps, glynn, nchunks, c.scratch[4].ptr, c.stream);
    if (rc) return rc;
    EGG_CUDA_TRY(cudaMemcpyAsync(out, c.scratch[4].ptr, es, cudaMemcpyDeviceToHost, c.stream));
    EGG_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return EGG_OK;
}

}  // extern "C"
