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
// Those are the per-level engine's launches, the default.  On request (egg_dp_mix_set_engine),
// mixes of degrees up to 32 run steps 2-4 as one cooperative launch instead (egg_mix_persist.cu);
// both give the same results, bit for bit.
// Every result is the value hafnian(A[r, r]; method = :dp) gives for the same precision mode.
#include <map>
#include <tuple>

#include "egg_internal.cuh"
#include "egg_mix.cuh"
#include "egg_tunecache.h"

namespace egg {

template <class T>
__global__ void mix_gather_kernel(const T *__restrict__ A, int64_t n, const int64_t *__restrict__ offsets,
                                  const int32_t *__restrict__ rows, const int32_t *__restrict__ order, MixBins bins,
                                  int64_t total, T *__restrict__ P)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x)
        mix_gather_elem<T, T>(g, A, n, offsets, rows, order, bins, P);
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

// How a degree bin is evaluated: `batched` runs groups of `group` instances through dp_run
// (instance-fastest, one thread per (state, instance)); otherwise groups of `group` instances go
// through dp_run_grouped (instance-major, each instance walked as a single instance).
struct BinExec {
    bool batched;
    int64_t group;
};

// Chosen per (degree, dtype, precision, size class of the bin) by timing on first use, kept for the
// process and in the tuning file (egg_tunecache.h), from which the next process on the same GPU
// model starts.  The size class keeps a choice timed on a handful of instances (where small groups
// can win) from deciding a batch of hundreds (where they lose by 2x).  Choices pinned with
// mix_set_tuning apply to every size; g_last is what egg_dp_mix_tuning reports.
static std::map<std::tuple<int, int, int, int>, BinExec> g_tuned;
static std::map<std::tuple<int, int, int>, BinExec> g_pinned, g_last;
static std::mutex g_tuned_mu;
static bool g_tuned_loaded = false;

// Size class of a bin of `count` instances: fewer than 4, 16, 64, 256, or more.
static int size_class(int64_t count)
{
    int cls = 0;
    for (int64_t lim = 4; cls < 4 && count >= lim; lim *= 4) ++cls;
    return cls;
}

// This device's identity in the tuning file: its model name and SM count.
static TuneRecord tune_identity()
{
    TuneRecord r;
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
        r.device = prop.name;
        r.sms = prop.multiProcessorCount;
    }
    return r;
}

// Reads the tuning file's records of this device into g_tuned, once (callers hold g_tuned_mu).
// Choices pinned or tuned in this process before the first read take precedence.
static void tuned_load_once()
{
    if (g_tuned_loaded) return;
    g_tuned_loaded = true;
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    std::vector<TuneRecord> rs;
    if (!tune_read_file(path, rs)) return;
    const TuneRecord me = tune_identity();
    // Per (degree, type, mode) the file's choice for the largest size class is the one reported.
    std::map<std::tuple<int, int, int>, std::pair<long long, BinExec>> largest;
    for (const TuneRecord &r : rs) {
        if (r.device != me.device || r.sms != me.sms || r.group < 1 || r.K < 2 || r.K > 64 || r.size < 0 || r.size > 4)
            continue;
        const BinExec ex{r.batched != 0, r.group};
        g_tuned.emplace(std::make_tuple((int)r.K, (int)r.dtype, (int)r.prec, (int)r.size), ex);
        const auto k3 = std::make_tuple((int)r.K, (int)r.dtype, (int)r.prec);
        auto it = largest.find(k3);
        if (it == largest.end() || r.size > it->second.first) largest[k3] = std::make_pair(r.size, ex);
    }
    for (const auto &kv : largest) g_last.emplace(kv.first, kv.second.second);
}

// Adds one tuned choice to the tuning file (a failure to write only costs a re-tune later).
static void tuned_save(int K, int dtype, int prec, int cls, const BinExec &ex)
{
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    TuneRecord r = tune_identity();
    r.K = K;
    r.dtype = dtype;
    r.prec = prec;
    r.batched = ex.batched ? 1 : 0;
    r.group = ex.group;
    r.size = cls;
    tune_merge_file(path, r);
}

static int launch_gather(int dtype, const void *dA, int64_t n, const int64_t *doff, const int32_t *drows,
                         const int32_t *dorder, const MixBins &bins, int64_t total, void *dP, cudaStream_t st)
{
    if (total <= 0) return EGG_OK;
    int64_t blocks = (total + 255) / 256, cap = (int64_t)ctx().num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (dtype == EGG_F64)
        mix_gather_kernel<double><<<(unsigned)blocks, 256, 0, st>>>((const double *)dA, n, doff, drows, dorder, bins, total,
                                                                    (double *)dP);
    else if (dtype == EGG_C128)
        mix_gather_kernel<cd><<<(unsigned)blocks, 256, 0, st>>>((const cd *)dA, n, doff, drows, dorder, bins, total, (cd *)dP);
    else
        mix_gather_kernel<int64_t><<<(unsigned)blocks, 256, 0, st>>>((const int64_t *)dA, n, doff, drows, dorder, bins, total,
                                                                     (int64_t *)dP);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

// Evaluate one bin (already gathered in the layout of `ex`) into its slice of the sorted results.
static int run_bin(const DevPlan &plan, int dtype, int prec, const MixBin &bn, const BinExec &ex, const char *dP,
                   char *dout, size_t es, size_t oes, cudaStream_t st)
{
    for (int64_t g0 = 0; g0 < bn.count; g0 += ex.group) {
        const int64_t len = bn.count - g0 < ex.group ? bn.count - g0 : ex.group;
        const char *P = dP + (size_t)g0 * bn.npairs * es;
        char *o = dout + (size_t)g0 * oes;
        const int rc = ex.batched ? dp_run(plan, dtype, prec, P, len, o, st) : dp_run_grouped(plan, dtype, prec, P, len, o, st);
        if (rc) return rc;
    }
    return EGG_OK;
}

// Instances a degree is tuned on: the whole bin up to this many, so that the timing sees the
// groups the batch will run (a small sample favoured small groups that the full batch runs slower).
static constexpr int64_t kTuneSample = 512;

// Time each candidate on the bin's first instances (at most kTuneSample) and keep the fastest.
// Each candidate is timed in three rounds, the candidates taking turns within a round, and its best
// round counts: one timing alone can be thrown off (a clock change, the host falling behind a run
// of many small launches) and pick a grouping that is slower in the batch.
static int tune_bin(const DevPlan &plan, int dtype, int prec, const MixBin &bn, const void *dA, int64_t n,
                    const int64_t *doff, const int32_t *drows, const int32_t *dorder, char *tmpP, char *tmpO, size_t es,
                    size_t oes, cudaStream_t st, BinExec *best)
{
    const int64_t S = bn.count < kTuneSample ? bn.count : kTuneSample;
    std::vector<BinExec> cands;
    for (int64_t L : {(int64_t)64, (int64_t)16})
        if (L <= S || L == 64) cands.push_back({true, L < S ? L : S});
    if (dp_grouped_ok(bn.K, dtype, prec) && plan.closed_form())
        for (int64_t G : {(int64_t)1, (int64_t)2, (int64_t)4, (int64_t)8, (int64_t)16, (int64_t)32, (int64_t)64})
            if (G <= S) cands.push_back({false, G});
    cudaEvent_t e0, e1;
    EGG_CUDA_TRY(cudaEventCreate(&e0));
    EGG_CUDA_TRY(cudaEventCreate(&e1));
    std::vector<float> bestms(cands.size(), 0.0f);
    bool have = false;
    int rc = EGG_OK;
    constexpr int kRounds = 3;
    for (int round = 0; round < kRounds && !rc; ++round) {
        for (size_t ci = 0; ci < cands.size() && !rc; ++ci) {
            const BinExec &cand = cands[ci];
            MixBins one;
            one.nb = 1;
            one.b[0] = bn;
            one.b[0].count = S;
            one.b[0].poff = 0;
            one.b[0].ebase = 0;
            one.b[0].lay = cand.batched ? cand.group : 1;
            rc = launch_gather(dtype, dA, n, doff, drows, dorder, one, (int64_t)bn.npairs * S, tmpP, st);
            if (!rc && round == 0) rc = run_bin(plan, dtype, prec, one.b[0], cand, tmpP, tmpO, es, oes, st);  // warm-up
            if (rc) break;
            cudaEventRecord(e0, st);
            rc = run_bin(plan, dtype, prec, one.b[0], cand, tmpP, tmpO, es, oes, st);
            cudaEventRecord(e1, st);
            if (rc) break;
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = fail(EGG_ERR_CUDA, "tuning run failed");
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (round == 0 || ms < bestms[ci]) bestms[ci] = ms;
        }
    }
    if (!rc) {
        float bestv = 0;
        for (size_t ci = 0; ci < cands.size(); ++ci)
            if (!have || bestms[ci] < bestv) {
                bestv = bestms[ci];
                *best = cands[ci];
                have = true;
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!rc && !have) rc = fail(EGG_ERR_CUDA, "no candidate to tune");
    if (!rc && best->batched) best->group = best->group >= S ? bn.count : best->group;  // the sample stood for "all"
    return rc;
}

// ---- graph replay -------------------------------------------------------------------------------
//
// The kernels of one mix (gather, every bin's levels, scatter) depend only on the bin sizes, the
// chosen evaluations and the buffers; the row sets themselves are read from device memory.  So the
// second call of the same shape captures them into one CUDA graph and later calls replay it: one
// launch instead of hundreds.  The offsets and the sorted order are copied in before the replay.
struct GraphKey {
    int dtype, prec;
    int64_t n, B;
    std::vector<int64_t> shape;  // per bin: K, count, batched, group
    std::vector<const void *> ptrs;
    bool operator==(const GraphKey &o) const
    {
        return dtype == o.dtype && prec == o.prec && n == o.n && B == o.B && shape == o.shape && ptrs == o.ptrs;
    }
};

struct GraphEntry {
    GraphKey key;
    int seen = 0;
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;  // kernel launches one replay makes
};

static std::vector<GraphEntry> g_graphs;  // a few recent shapes; callers hold the library's lock
static constexpr size_t kMaxGraphs = 8;

static GraphEntry &graph_entry(const GraphKey &key)
{
    for (GraphEntry &e : g_graphs)
        if (e.key == key) return e;
    if (g_graphs.size() >= kMaxGraphs) {
        if (g_graphs.front().exec) cudaGraphExecDestroy(g_graphs.front().exec);
        g_graphs.erase(g_graphs.begin());
    }
    g_graphs.push_back(GraphEntry{key});
    return g_graphs.back();
}

void mix_graphs_clear()
{
    for (GraphEntry &e : g_graphs)
        if (e.exec) cudaGraphExecDestroy(e.exec);
    g_graphs.clear();
}

static int mix_kernels(int dtype, int prec, const void *dA, int64_t n, int64_t B, const MixBins &bins,
                       const std::vector<BinExec> &exs, const std::vector<DevPlan *> &plans, const int64_t *doff,
                       const int32_t *drows, const int32_t *dorder, int64_t total, int64_t ndp, int64_t nzero, char *dP,
                       char *dsorted, void *dout, cudaStream_t st);

// The mix with A, the row indices and out in device memory and the row-set boundaries on the host.
int mix_run(int dtype, int prec, const void *dA, int64_t n, int64_t B, const int64_t *offsets, const int32_t *drows,
            void *dout, cudaStream_t st)
{
    if (dtype != EGG_F64 && dtype != EGG_C128 && dtype != EGG_I64)
        return fail(EGG_ERR_ARGUMENT, "the mixed-degree batch takes Float64, ComplexF64 or Int64 parents");
    if (dtype == EGG_I64 && prec != EGG_PREC_EXACT) return fail(EGG_ERR_ARGUMENT, "integer parents run exactly");
    if (prec != EGG_PREC_EXACT && prec != EGG_PREC_FMA && prec != EGG_PREC_MIXED)
        return fail(EGG_ERR_ARGUMENT, "unknown precision mode");
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
        bn.lay = bn.count;
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
    // 2. Plans; buffers for the largest group of every bin (sized before anything is enqueued, so
    // no buffer is reallocated while an earlier bin's kernels may still be running).
    const size_t es = dtype_size(dtype), oes = dtype == EGG_I64 ? 16 : es;
    std::vector<DevPlan *> plans;
    for (int k = 0; k < bins.nb; ++k) {
        int rc = EGG_OK;
        DevPlan *pl = dp_plan_for(bins.b[k].K, &rc);
        if (!pl) return rc;
        plans.push_back(pl);
    }
    Context &c = ctx();
    int npmax = 0;
    for (int k = 0; k < bins.nb; ++k) npmax = bins.b[k].npairs > npmax ? bins.b[k].npairs : npmax;
    const size_t off_o = align256((size_t)(B + 1) * 8), off_p = off_o + align256((size_t)B * 4);
    const size_t off_r = off_p + align256((size_t)total * es), off_t = off_r + align256((size_t)(ndp ? ndp : 1) * oes);
    const size_t off_to = off_t + align256((size_t)kTuneSample * npmax * es), arena = off_to + align256((size_t)kTuneSample * oes);
    int rc = ensure_buf(c.scratch[6], arena);
    if (rc) return rc;
    char *base = (char *)c.scratch[6].ptr;
    int64_t *doff = (int64_t *)base;
    int32_t *dorder = (int32_t *)(base + off_o);
    char *dP = base + off_p, *dsorted = base + off_r, *tmpP = base + off_t, *tmpO = base + off_to;
    EGG_CUDA_TRY(cudaMemcpyAsync(doff, offsets, (size_t)(B + 1) * 8, cudaMemcpyHostToDevice, st));
    EGG_CUDA_TRY(cudaMemcpyAsync(dorder, order.data(), (size_t)B * 4, cudaMemcpyHostToDevice, st));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    EGG_CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    // The whole mix in one cooperative launch where that engine takes it (a stream being captured
    // records the per-level launches instead).
    if (mix_engine() == kMixPersistent && cap == cudaStreamCaptureStatusNone && mix_persistent_ok(bins, plans, dtype, prec)) {
        rc = mix_persistent_run(dtype, prec, dA, n, B, bins, plans, doff, drows, dorder, total, ndp, nzero, dsorted, dout, st);
        if (rc != kDpNotHere) return rc;
        rc = EGG_OK;
    }
    // 3. How each bin runs: one launch for degrees the whole-instance kernel covers, else the tuned
    // choice (timed on first use, unless the stream is being captured).
    std::vector<BinExec> exs(bins.nb);
    size_t hmax = 0, p32max = 0;
    for (int k = 0; k < bins.nb; ++k) {
        MixBin &bn = bins.b[k];
        BinExec ex{true, bn.count};
        if (bn.K > 22 && bn.count > 1) {
            const int cls = size_class(bn.count);
            const auto key3 = std::make_tuple(bn.K, dtype, prec);
            const auto key = std::make_tuple(bn.K, dtype, prec, cls);
            bool found = false;
            {
                std::lock_guard<std::mutex> lk(g_tuned_mu);
                tuned_load_once();
                auto ip = g_pinned.find(key3);
                auto it = g_tuned.find(key);
                if (ip != g_pinned.end()) {
                    ex = ip->second;
                    found = true;
                } else if (it != g_tuned.end()) {
                    ex = it->second;
                    found = true;
                }
            }
            if (!found && cap == cudaStreamCaptureStatusNone) {
                // Tuning needs the largest candidate's buffers.
                size_t h = dp_scratch_bytes(*plans[k], dtype, prec, 64);
                rc = ensure_buf(c.scratch[0], h);
                if (!rc && prec == EGG_PREC_MIXED)
                    rc = ensure_buf(c.scratch[5], (size_t)64 * bn.npairs * (dtype == EGG_C128 ? 2 : 1) * sizeof(float));
                if (!rc) rc = tune_bin(*plans[k], dtype, prec, bn, dA, n, doff, drows, dorder, tmpP, tmpO, es, oes, st, &ex);
                if (rc) return rc;
                std::lock_guard<std::mutex> lk(g_tuned_mu);
                g_tuned[key] = ex;
                g_last[key3] = ex;
                tuned_save(bn.K, dtype, prec, cls, ex);
            } else if (!found) {
                ex = dp_grouped_ok(bn.K, dtype, prec) && plans[k]->closed_form() ? BinExec{false, 4} : BinExec{true, bn.count};
            }
            if (!ex.batched && !plans[k]->closed_form()) ex = BinExec{true, bn.count};  // an explicit plan is now resident
            if (ex.group > bn.count) ex.group = bn.count;
        }
        exs[k] = ex;
        bn.lay = ex.batched ? ex.group : 1;
        const size_t h = dp_scratch_bytes(*plans[k], dtype, prec, ex.group);
        hmax = h > hmax ? h : hmax;
        const size_t p32 = (size_t)bn.npairs * ex.group * (dtype == EGG_C128 ? 2 : 1) * sizeof(float);
        p32max = p32 > p32max ? p32 : p32max;
    }
    if (hmax) rc = ensure_buf(c.scratch[0], hmax);
    if (!rc && prec == EGG_PREC_MIXED && p32max) rc = ensure_buf(c.scratch[5], p32max);
    if (rc) return rc;
    // 4. Gather, 5. DP per bin, 6. scatter: eagerly the first time a shape is seen, captured into a
    // graph the second time, replayed after that (not when the caller is capturing the stream).
    if (!binom32_device(&rc)) return rc;
    GraphKey key{dtype, prec, n, B, {}, {dA, drows, dout}};
    for (int k = 0; k < bins.nb; ++k) {
        key.shape.insert(key.shape.end(), {(int64_t)bins.b[k].K, bins.b[k].count, exs[k].batched ? 1 : 0, exs[k].group});
    }
    for (const DevBuf &b : c.scratch) key.ptrs.push_back(b.ptr);
    // Every device array a recorded kernel may read: the plans' transition arrays (explicit plans)
    // and their cluster lists, which exist only once built.  A graph keyed on them is never
    // replayed against a plan that was released and rebuilt elsewhere.
    for (const DevPlan *pl : plans) {
        key.ptrs.push_back(pl->trans);
        key.ptrs.push_back(pl->cluster_lists[0]);
        key.ptrs.push_back(pl->cluster_lists[1]);
    }
    GraphEntry *ge = cap == cudaStreamCaptureStatusNone ? &graph_entry(key) : nullptr;
    if (ge && ge->exec) {
        EGG_CUDA_TRY(cudaGraphLaunch(ge->exec, st));
        count_launch(ge->nodes);
        return EGG_OK;
    }
    const bool capture = ge && ge->seen >= 1;
    if (ge) ++ge->seen;
    const long long launches0 = g_launches.load();
    if (capture) EGG_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = mix_kernels(dtype, prec, dA, n, B, bins, exs, plans, doff, drows, dorder, total, ndp, nzero, dP, dsorted, dout, st);
    if (capture) {
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (rc || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return rc ? rc : fail(EGG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) return fail(EGG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        ge->exec = exec;
        ge->nodes = g_launches.load() - launches0;
        g_launches.fetch_sub(ge->nodes);  // counted when the graph runs, not when it is recorded
        EGG_CUDA_TRY(cudaGraphLaunch(exec, st));
        count_launch(ge->nodes);
    }
    return rc;
}

// Steps 4-6 of mix_run: the gather, each bin's DP, and the scatter, enqueued on `st`.
static int mix_kernels(int dtype, int prec, const void *dA, int64_t n, int64_t B, const MixBins &bins,
                       const std::vector<BinExec> &exs, const std::vector<DevPlan *> &plans, const int64_t *doff,
                       const int32_t *drows, const int32_t *dorder, int64_t total, int64_t ndp, int64_t nzero, char *dP,
                       char *dsorted, void *dout, cudaStream_t st)
{
    Context &c = ctx();
    const size_t es = dtype_size(dtype), oes = dtype == EGG_I64 ? 16 : es;
    int rc = launch_gather(dtype, dA, n, doff, drows, dorder, bins, total, dP, st);
    if (rc) return rc;
    for (int k = 0; k < bins.nb; ++k) {
        const MixBin &bn = bins.b[k];
        rc = run_bin(*plans[k], dtype, prec, bn, exs[k], dP + (size_t)bn.poff * es, dsorted + (size_t)bn.first * oes, es, oes,
                     st);
        if (rc) return rc;
    }
    {
        int64_t blocks = (B + 255) / 256, capb = (int64_t)c.num_sms * 16;
        if (blocks > capb) blocks = capb;
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

int mix_set_tuning(int K, int dtype, int prec, int batched, int64_t group)
{
    if (K < 2 || K > 64 || K % 2) return fail(EGG_ERR_ARGUMENT, "degree must be even, 2..64");
    if (group < 1) return fail(EGG_ERR_ARGUMENT, "group must be >= 1");
    if (!batched && !dp_grouped_ok(K, dtype, prec))
        return fail(EGG_ERR_ARGUMENT, "no grouped single-instance evaluation for this degree and type");
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    g_pinned[std::make_tuple(K, dtype, prec)] = BinExec{batched != 0, group};
    g_last[std::make_tuple(K, dtype, prec)] = BinExec{batched != 0, group};
    return EGG_OK;
}

int mix_tuned(int K, int dtype, int prec, int *batched, int64_t *group)
{
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    tuned_load_once();
    auto it = g_last.find(std::make_tuple(K, dtype, prec));
    if (it == g_last.end()) return fail(EGG_ERR_NO_PLAN, "degree " + std::to_string(K) + " has not been tuned");
    *batched = it->second.batched ? 1 : 0;
    *group = it->second.group;
    return EGG_OK;
}

}  // namespace egg
