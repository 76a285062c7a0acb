// egg_mix_persist.cu -- a whole mixed-degree batch in one cooperative launch.
//
// The per-level engine (egg_mix.cu) runs a mix as a gather launch, a launch per level of every
// group of every degree bin, and a scatter launch.  Here one launch does all of it, in phases
// separated by grid-wide barriers (egg_gridbar.cuh):
//   1. the gather: every bin's pairs, instance-major, straight from the parent;
//   2. the levels, in lockstep over the bins: step t evaluates level c = 2t of every bin whose
//      degree K >= c, for a wave of at most W instances per bin (W chosen on the host so that
//      two level buffers per instance of every bin fit a fixed device-memory budget; larger
//      mixes run several waves);
//   3. the scatter of the results into the caller's order.
// Within a step the work is a list of units -- (bin, instance, chunk of 2048 consecutive states of
// the level) -- that blocks claim in short runs from a counter, so bins of every size share the
// SMs and small levels fill the gaps of large ones.  A unit is evaluated exactly as the per-level
// engine's fixed-popcount kernel evaluates a chunk (egg_dp_fixed.cuh: colex unrank and successors,
// then walk_fixed in plan order), so every result is bit-identical to that engine's and to
// hafnian(A[r, r]; method = :dp) in the same precision mode.  Values other blocks wrote earlier in
// the launch are read after a grid barrier: the previous level with weak loads cached in L1
// (ld_ca), the pairs and the results through L2 only; never through the read-only path.
//
// Measured on the 4096-instance configuration-4 mix (ComplexF64, degrees 8..32, one B200): this
// engine 50.4 ms a batch, the per-level engine (tuned groups, graph replay) 45.3 ms at the time and
// 39.1 ms since its level kernels got per-popcount block counts and one block per chunk, so the
// per-level engine is the default.  The level kernels there are compiled per popcount, each with
// the registers its walk needs; one kernel serving every popcount carries the largest walk's
// registers (or spills them at three blocks per SM), and that is most of the difference.
// Measured variants: two blocks per SM 53.1 ms, four 53.6 ms; a claim of one unit at a time
// 61.7 ms; the previous level read through L2 only instead of L1, no change; waves of 1 GiB,
// 8 GiB and 16 GiB of level buffers 54.7, 49.8 and 50.6 ms.
#include "egg_gridbar.cuh"
#include "egg_internal.cuh"
#include "egg_dp_fixed.cuh"
#include "egg_mix.cuh"

namespace egg {

static constexpr int kChunk = kRun * kLevelThreads;                                 // states per unit
static constexpr int kMaxU = 32;                                                    // mask positions
static constexpr size_t kTableBytes = (size_t)kMaxU * (kMaxU + 1) * sizeof(uint2);  // pair table, c <= 32
static constexpr unsigned long long kBarrierWaitNs = 2000000000ull;                  // 2 s per barrier
// Blocks per SM the kernel is compiled for (at most 85 registers a thread at three).
static constexpr int kPersistMinBlocks = 3;
// A block claims about 1/kClaimsPerBlock of its share of a step's units at a time: consecutive
// chunks of one instance stay on one SM (its pairs and pair table stay in shared memory, and
// neighbouring chunks share children in L1), while late claims still even out the blocks.
static constexpr int64_t kClaimsPerBlock = 64;

// One (bin, level) of a step: the level's states for `ninst` consecutive instances of the bin.
struct PSeg {
    const void *P;     // pairs of the segment's first instance; instance i at + i * npairs elements
    const void *prev;  // level c - 2 of the first instance; instance i at + i * ldh elements
    void *cur;         // level c (c < K): instance i at + i * ldh elements
    void *out;         // the results (c == K): instance i at + i elements
    int64_t n;         // states of level c
    int64_t nchunk;    // units per instance
    int64_t ubegin;    // the segment's first unit within its step
    int64_t ldh;       // level-buffer stride between instances
    int K, c;
};

struct PStep {
    int seg0, nseg;
    int64_t units;
    int64_t grab;  // units per claim
};

struct PersistArgs {
    // phase 1: the gather
    const void *A;
    int64_t n;
    const int64_t *offsets;
    const int32_t *rows;
    const int32_t *order;
    MixBins bins;
    int64_t gtotal;
    void *P;
    // phase 2: the levels
    const PStep *steps;
    const PSeg *segs;
    int nsteps;
    const uint32_t *binom;
    // phase 3: the scatter
    const void *sorted;
    int64_t ndp, nzero, none;
    void *out;
    // synchronisation: nsteps unit counters, then the barrier's two words (all zero at launch)
    unsigned *ctr;
    int *flag;       // device word: a barrier wait gave up
    int *host_flag;  // mapped host word the launch raises when it ends after a timeout
    unsigned nblocks;
    unsigned long long wait_ns;
};

// walk_fixed for a popcount known only at run time (uniform across the block): one case per level.
template <class Op, class PT, class HT, class AT>
__device__ __forceinline__ AT walk_level(int c, uint32_t m, const uint2 *TP, int K, int m0, const PT *Ps, const HT *Hp)
{
#define EGG_WALK_CASE(CC) \
    case CC: return walk_fixed<CC, Op, uint32_t, PT, HT, AT, kLoadCA>(m, TP, K, m0, Ps, Hp);
    switch (c) {
        EGG_WALK_CASE(4) EGG_WALK_CASE(6) EGG_WALK_CASE(8) EGG_WALK_CASE(10) EGG_WALK_CASE(12) EGG_WALK_CASE(14)
        EGG_WALK_CASE(16) EGG_WALK_CASE(18) EGG_WALK_CASE(20) EGG_WALK_CASE(22) EGG_WALK_CASE(24) EGG_WALK_CASE(26)
        EGG_WALK_CASE(28) EGG_WALK_CASE(30) EGG_WALK_CASE(32)
    }
#undef EGG_WALK_CASE
    return zero_of<AT>();
}

template <class Op, class T, class PT, class HT, class AT, class OT>
__global__ void __launch_bounds__(kLevelThreads, kPersistMinBlocks) mix_persistent_kernel(PersistArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t *masks = reinterpret_cast<uint32_t *>(smem_raw);
    uint2 *TP = reinterpret_cast<uint2 *>(smem_raw + (size_t)kChunk * sizeof(uint32_t));
    PT *Ps = reinterpret_cast<PT *>(smem_raw + (size_t)kChunk * sizeof(uint32_t) + kTableBytes);
    __shared__ PSeg sseg[kMaxBins];
    __shared__ int64_t s_unit;
    const int tid = threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x, gtid = blockIdx.x * (int64_t)blockDim.x + tid;
    unsigned *bar = a.ctr + a.nsteps;
    unsigned epoch = 0;

    // 1. The gather, instance-major within each bin (lay = 1).
    for (int64_t g = gtid; g < a.gtotal; g += nth)
        mix_gather_elem<T, PT>(g, (const T *)a.A, a.n, a.offsets, a.rows, a.order, a.bins, (PT *)a.P);
    grid_barrier(bar, a.nblocks, epoch, a.flag, a.wait_ns);

    // 2. The levels.
    int tkey = -1;             // (K, c) of the pair table in shared memory
    const PT *pkey = nullptr;  // instance whose pairs are in shared memory
    for (int st = 0; st < a.nsteps; ++st) {
        const PStep sd = a.steps[st];
        for (int i = tid; i < sd.nseg; i += blockDim.x) sseg[i] = a.segs[sd.seg0 + i];
        for (;;) {
            __syncthreads();  // the previous claim is done with s_unit, the masks, the table and the pairs
            if (tid == 0) s_unit = (int64_t)atomicAdd(&a.ctr[st], (unsigned)sd.grab);
            __syncthreads();
            const int64_t u0 = s_unit;
            if (u0 >= sd.units) break;
            const int64_t u1 = u0 + sd.grab < sd.units ? u0 + sd.grab : sd.units;
            for (int64_t u = u0; u < u1; ++u) {
                if (u > u0) __syncthreads();  // the previous unit is done with the masks, the table and the pairs
                int j = 0;
                while (j + 1 < sd.nseg && sseg[j + 1].ubegin <= u) ++j;
                const PSeg &sg = sseg[j];
                const int64_t w = u - sg.ubegin, inst = w / sg.nchunk;
                const int64_t s0 = (w - inst * sg.nchunk) * (int64_t)kChunk;
                const int K = sg.K, c = sg.c, npairs = K * (K - 1) / 2;
                const int cnt = (int)(sg.n - s0 < kChunk ? sg.n - s0 : kChunk);
                const PT *Pi = (const PT *)sg.P + inst * npairs;
                if (c > 2 && tkey != K * 64 + c) {
                    fill_pair_table(TP, a.binom, (K + c) / 2, c + 1, tid, blockDim.x);
                    tkey = K * 64 + c;
                }
                if (pkey != Pi) {
                    for (int q = tid; q < npairs; q += blockDim.x) Ps[q] = ld_l2(Pi + q);
                    pkey = Pi;
                }
                __syncthreads();
                if (c == 2) {
                    for (int i = tid; i < cnt; i += blockDim.x) {
                        const HT v = first_level_value<Op, PT, HT, AT>(s0 + i, K, Ps, 1, 0);
                        if (c == K) store(((OT *)sg.out)[inst], v);
                        else ((HT *)sg.cur)[inst * sg.ldh + s0 + i] = v;
                    }
                } else {
                    const int m0 = (K - c) / 2, U = K - m0;
                    const int r0 = tid * kRun;
                    if (r0 < cnt) {
                        uint32_t m = colex_unrank<uint32_t>(TP, c + 1, U, c, (uint32_t)(s0 + r0));
                        masks[r0] = m;
                        for (int r = 1; r < kRun && r0 + r < cnt; ++r) {
                            m = colex_next<uint32_t>(m);
                            masks[r0 + r] = m;
                        }
                    }
                    __syncthreads();
                    const HT *Hp = (const HT *)sg.prev + inst * sg.ldh;
                    for (int i = tid; i < cnt; i += blockDim.x) {
                        const AT acc = walk_level<Op, PT, HT, AT>(c, masks[i], TP, K, m0, Ps, Hp);
                        if (c == K) {
                            HT h;
                            store(h, acc);
                            store(((OT *)sg.out)[inst], h);
                        } else {
                            store(((HT *)sg.cur)[inst * sg.ldh + s0 + i], acc);
                        }
                    }
                }
            }
        }
        grid_barrier(bar, a.nblocks, epoch, a.flag, a.wait_ns);
    }

    // 3. The scatter: sorted results to the caller's order, 0 for odd sizes, 1 for empty sets.
    const int64_t total = a.ndp + a.nzero + a.none;
    for (int64_t k = gtid; k < total; k += nth) {
        OT v;
        if (k < a.ndp) v = ld_l2((const OT *)a.sorted + k);
        else if (k < a.ndp + a.nzero) v = OT{};
        else v = mix_one<OT>();
        ((OT *)a.out)[a.order[k]] = v;
    }
    if (tid == 0 && *(volatile int *)a.flag) {
        *(volatile int *)a.host_flag = 1;
        __threadfence_system();
    }
}

// ---- host ----------------------------------------------------------------------------------------

// The mapped host word the launches raise after a barrier timeout (allocated on first use).
static int *g_host_flag = nullptr, *g_host_flag_dev = nullptr;

static int host_flag(int **host, int **dev)
{
    if (!g_host_flag) {
        void *p = nullptr;
        EGG_CUDA_TRY(cudaHostAlloc(&p, sizeof(int), cudaHostAllocMapped));
        *(volatile int *)p = 0;
        void *d = nullptr;
        const cudaError_t e = cudaHostGetDevicePointer(&d, p, 0);
        if (e != cudaSuccess) {
            cudaFreeHost(p);
            return fail(EGG_ERR_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
        }
        g_host_flag = (int *)p;
        g_host_flag_dev = (int *)d;
    }
    *host = g_host_flag;
    *dev = g_host_flag_dev;
    return EGG_OK;
}

int mix_persistent_take_timeout()
{
    if (g_host_flag && *(volatile int *)g_host_flag) {
        *(volatile int *)g_host_flag = 0;
        return fail(EGG_ERR_TIMEOUT, "a grid barrier of the persistent mixed-degree launch gave up waiting; "
                                     "its results are invalid");
    }
    return EGG_OK;
}

static int g_engine = kMixLevels;

int mix_engine() { return g_engine; }

int mix_set_engine(int engine)
{
    if (engine != kMixLevels && engine != kMixPersistent) return fail(EGG_ERR_ARGUMENT, "engine must be 0 or 1");
    g_engine = engine;
    return EGG_OK;
}

bool mix_persistent_ok(const MixBins &bins, const std::vector<DevPlan *> &plans, int dtype, int prec)
{
    if (dtype == EGG_I64) {
        if (prec != EGG_PREC_EXACT) return false;
    } else if (dtype != EGG_F64 && dtype != EGG_C128) {
        return false;
    }
    if (prec != EGG_PREC_EXACT && prec != EGG_PREC_FMA && prec != EGG_PREC_MIXED) return false;
    for (int k = 0; k < bins.nb; ++k)
        if (bins.b[k].K > kMaxU || !plans[k]->closed_form()) return false;  // 32-bit masks; the closed-form order
    return true;
}

// Level buffers of every bin for a wave of at most this many bytes (W = 1 is always allowed).
static constexpr size_t kWaveBudget = (size_t)4 << 30;

template <class Op, class T, class PT, class HT, class AT, class OT>
static int persistent_launch(const void *dA, int64_t n, const MixBins &bins, const std::vector<DevPlan *> &plans,
                             const int64_t *doff, const int32_t *drows, const int32_t *dorder, int64_t total,
                             int64_t ndp, int64_t nzero, int64_t B, char *dsorted, void *dout, cudaStream_t st)
{
    Context &cx = ctx();
    int rc = EGG_OK;
    const uint32_t *bt = binom32_device(&rc);
    if (!bt) return rc;
    // Wave size: halve W until two level buffers per instance of every bin fit the budget.
    int64_t cmax = 0;
    std::vector<int64_t> maxlev(bins.nb);
    for (int k = 0; k < bins.nb; ++k) {
        int64_t mx = 1;
        for (const Level &L : plans[k]->levels) mx = L.n > mx ? L.n : mx;
        maxlev[k] = mx;
        cmax = bins.b[k].count > cmax ? bins.b[k].count : cmax;
    }
    auto wave_bytes = [&](int64_t w) {
        size_t s = 0;
        for (int k = 0; k < bins.nb; ++k)
            s += (size_t)2 * maxlev[k] * (size_t)(bins.b[k].count < w ? bins.b[k].count : w) * sizeof(HT);
        return s;
    };
    int64_t W = cmax > 1 ? cmax : 1;  // no bins (only odd and empty row sets): no waves, W unused
    while (W > 1 && wave_bytes(W) > kWaveBudget) W = (W + 1) / 2;
    // Buffers: the pairs (instance-major), then per bin two level buffers of W instances.
    const size_t pbytes = ((size_t)total * sizeof(PT) + 255) / 256 * 256;
    std::vector<size_t> hoff(bins.nb);
    size_t hb = pbytes;
    for (int k = 0; k < bins.nb; ++k) {
        hoff[k] = hb;
        const int64_t wk = bins.b[k].count < W ? bins.b[k].count : W;
        hb += ((size_t)2 * maxlev[k] * wk * sizeof(HT) + 255) / 256 * 256;
    }
    rc = ensure_buf(cx.scratch[0], hb > 256 ? hb : 256);
    if (rc) return rc;
    char *base = (char *)cx.scratch[0].ptr;
    PT *dP = (PT *)base;
    auto kfn = mix_persistent_kernel<Op, T, PT, HT, AT, OT>;
    const size_t smem = (size_t)kChunk * sizeof(uint32_t) + kTableBytes + (size_t)kMaxU * (kMaxU - 1) / 2 * sizeof(PT);
    rc = smem_limit_at_least((const void *)kfn, smem);
    if (rc) return rc;
    int bps = 0;
    rc = blocks_per_sm((const void *)kfn, kLevelThreads, smem, &bps);
    if (rc) return rc;
    if (bps < 1) return fail(EGG_ERR_CUDA, "the persistent mixed-degree kernel does not fit on an SM");
    const int64_t nblocks = (int64_t)bps * cx.num_sms;
    // Steps and segments: for each wave, steps t = 1 .. Kmax/2 (level c = 2t of every bin with K >= c).
    MixBins gb = bins;
    for (int k = 0; k < gb.nb; ++k) gb.b[k].lay = 1;  // instance-major pairs
    std::vector<PStep> steps;
    std::vector<PSeg> segs;
    int Kmax = 0;
    for (int k = 0; k < bins.nb; ++k) Kmax = bins.b[k].K > Kmax ? bins.b[k].K : Kmax;
    const int64_t nwaves = (cmax + W - 1) / W;
    for (int64_t wv = 0; wv < nwaves; ++wv) {
        for (int t = 1; 2 * t <= Kmax; ++t) {
            const int c = 2 * t;
            PStep sp{(int)segs.size(), 0, 0, 1};
            for (int k = 0; k < bins.nb; ++k) {
                const MixBin &bn = bins.b[k];
                const int64_t inst0 = wv * W;
                if (bn.K < c || bn.count <= inst0) continue;
                const int64_t ninst = bn.count - inst0 < W ? bn.count - inst0 : W;
                const int64_t lev = plans[k]->levels[t].n;
                const int64_t wk = bn.count < W ? bn.count : W;
                HT *H0 = (HT *)(base + hoff[k]), *H1 = H0 + (size_t)maxlev[k] * wk;
                PSeg sg{};
                sg.P = dP + bn.poff + inst0 * bn.npairs;
                sg.prev = (t - 1) & 1 ? H1 : H0;
                sg.cur = t & 1 ? H1 : H0;
                sg.out = dsorted + (size_t)(bn.first + inst0) * sizeof(OT);
                sg.n = lev;
                sg.nchunk = (lev + kChunk - 1) / kChunk;
                sg.ubegin = sp.units;
                sg.ldh = maxlev[k];
                sg.K = bn.K;
                sg.c = c;
                sp.units += ninst * sg.nchunk;
                segs.push_back(sg);
                ++sp.nseg;
            }
            if (sp.units) {
                sp.grab = sp.units / (nblocks * kClaimsPerBlock);
                if (sp.grab < 1) sp.grab = 1;
                steps.push_back(sp);
            }
        }
    }
    if (steps.size() > (size_t)INT32_MAX / 2) return fail(EGG_ERR_TOO_LARGE, "too many steps for one launch");
    // Tables, counters and the barrier words.
    const int nsteps = (int)steps.size();
    const size_t off_seg = ((size_t)nsteps * sizeof(PStep) + 255) / 256 * 256;
    const size_t off_ctr = off_seg + (segs.size() * sizeof(PSeg) + 255) / 256 * 256;
    const size_t ctr_bytes = ((size_t)nsteps + 2) * sizeof(unsigned), off_flag = off_ctr + (ctr_bytes + 15) / 16 * 16;
    rc = ensure_buf(cx.scratch[10], off_flag + 16);
    if (rc) return rc;
    char *tb = (char *)cx.scratch[10].ptr;
    if (nsteps) EGG_CUDA_TRY(cudaMemcpyAsync(tb, steps.data(), (size_t)nsteps * sizeof(PStep), cudaMemcpyHostToDevice, st));
    if (!segs.empty())
        EGG_CUDA_TRY(cudaMemcpyAsync(tb + off_seg, segs.data(), segs.size() * sizeof(PSeg), cudaMemcpyHostToDevice, st));
    EGG_CUDA_TRY(cudaMemsetAsync(tb + off_ctr, 0, off_flag + 16 - off_ctr, st));
    int *hflag = nullptr, *hflag_dev = nullptr;
    rc = host_flag(&hflag, &hflag_dev);
    if (rc) return rc;
    // One cooperative launch of as many blocks as fit on the device at once.
    PersistArgs a{};
    a.A = dA;
    a.n = n;
    a.offsets = doff;
    a.rows = drows;
    a.order = dorder;
    a.bins = gb;
    a.gtotal = total;
    a.P = dP;
    a.steps = (const PStep *)tb;
    a.segs = (const PSeg *)(tb + off_seg);
    a.nsteps = nsteps;
    a.binom = bt;
    a.sorted = dsorted;
    a.ndp = ndp;
    a.nzero = nzero;
    a.none = B - ndp - nzero;
    a.out = dout;
    a.ctr = (unsigned *)(tb + off_ctr);
    a.flag = (int *)(tb + off_flag);
    a.host_flag = hflag_dev;
    a.nblocks = (unsigned)nblocks;
    a.wait_ns = kBarrierWaitNs;
    void *params[] = {&a};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void *)kfn, dim3(a.nblocks), dim3(kLevelThreads), params, smem, st);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
        cudaGetLastError();  // another context holds part of the device: the per-level engine runs instead
        return kDpNotHere;
    }
    if (e != cudaSuccess) return fail(EGG_ERR_CUDA, std::string("cudaLaunchCooperativeKernel: ") + cudaGetErrorString(e));
    count_launch();
    return EGG_OK;
}

int mix_persistent_run(int dtype, int prec, const void *dA, int64_t n, int64_t B, const MixBins &bins,
                       const std::vector<DevPlan *> &plans, const int64_t *doff, const int32_t *drows,
                       const int32_t *dorder, int64_t total, int64_t ndp, int64_t nzero, char *dsorted, void *dout,
                       cudaStream_t st)
{
    const bool fma_mode = prec == EGG_PREC_FMA, mixed = prec == EGG_PREC_MIXED;
    switch (dtype) {
    case EGG_F64:
        if (mixed)
            return persistent_launch<MixedOp, double, float, float, double, double>(dA, n, bins, plans, doff, drows, dorder, total,
                                                                                   ndp, nzero, B, dsorted, dout, st);
        return fma_mode ? persistent_launch<FmaOp, double, double, double, double, double>(dA, n, bins, plans, doff, drows, dorder,
                                                                                          total, ndp, nzero, B, dsorted, dout, st)
                        : persistent_launch<ExactOp, double, double, double, double, double>(
                              dA, n, bins, plans, doff, drows, dorder, total, ndp, nzero, B, dsorted, dout, st);
    case EGG_C128:
        if (mixed)
            return persistent_launch<MixedOp, cd, cf, cf, cd, cd>(dA, n, bins, plans, doff, drows, dorder, total, ndp, nzero, B,
                                                                 dsorted, dout, st);
        return fma_mode ? persistent_launch<FmaOp, cd, cd, cd, cd, cd>(dA, n, bins, plans, doff, drows, dorder, total, ndp, nzero,
                                                                      B, dsorted, dout, st)
                        : persistent_launch<ExactOp, cd, cd, cd, cd, cd>(dA, n, bins, plans, doff, drows, dorder, total, ndp,
                                                                        nzero, B, dsorted, dout, st);
    case EGG_I64:
        return persistent_launch<IntOp, int64_t, int64_t, __int128, __int128, __int128>(
            dA, n, bins, plans, doff, drows, dorder, total, ndp, nzero, B, dsorted, dout, st);
    }
    return fail(EGG_ERR_ARGUMENT, "unknown dtype");
}

// ---- the barrier's bounded wait, exercised on its own ---------------------------------------------

// Every block passes `rounds` barriers that expect `nexpect` blocks (more than the grid has, to make
// the waits run out).  With nexpect > the grid the first wait ends after wait_ns and the rest
// return at once.
static __global__ void barrier_check_kernel(unsigned *bar, int *flag, unsigned nexpect, int rounds,
                                            unsigned long long wait_ns, unsigned *passes)
{
    unsigned epoch = 0;
    for (int r = 0; r < rounds; ++r) {
        grid_barrier(bar, nexpect, epoch, flag, wait_ns);
        if (threadIdx.x == 0) atomicAdd(passes, 1u);
    }
}

int barrier_selfcheck(int extra, int64_t wait_ns, int64_t *passes_out)
{
    Context &cx = ctx();
    if (extra < 0 || extra > 1024) return fail(EGG_ERR_ARGUMENT, "extra must be in [0, 1024]");
    if (wait_ns < 1000000 || wait_ns > 2000000000LL) return fail(EGG_ERR_ARGUMENT, "wait_ns must be in [1 ms, 2 s]");
    int rc = ensure_buf(cx.scratch[10], 64);
    if (rc) return rc;
    unsigned *w = (unsigned *)cx.scratch[10].ptr;  // bar[2], flag, passes
    EGG_CUDA_TRY(cudaMemsetAsync(w, 0, 16, cx.stream));
    int bps = 0;
    rc = blocks_per_sm((const void *)barrier_check_kernel, 128, 0, &bps);
    if (rc) return rc;
    if (bps < 1) return fail(EGG_ERR_CUDA, "the barrier check kernel does not fit on an SM");
    const unsigned nblocks = (unsigned)((bps < 2 ? bps : 2) * cx.num_sms);
    unsigned *bar = w;
    int *flag = (int *)(w + 2);
    unsigned *passes = w + 3;
    unsigned nexpect = nblocks + (unsigned)extra;
    int rounds = 3;
    unsigned long long wns = (unsigned long long)wait_ns;
    void *params[] = {&bar, &flag, &nexpect, &rounds, &wns, &passes};
    EGG_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)barrier_check_kernel, dim3(nblocks), dim3(128), params, 0, cx.stream));
    count_launch();
    unsigned hv[4] = {0, 0, 0, 0};
    EGG_CUDA_TRY(cudaMemcpyAsync(hv, w, 16, cudaMemcpyDeviceToHost, cx.stream));
    EGG_CUDA_TRY(cudaStreamSynchronize(cx.stream));
    if (passes_out) *passes_out = (int64_t)hv[3];
    if (hv[3] != (unsigned)rounds * nblocks) return fail(EGG_ERR_CUDA, "barrier check: not every block passed every barrier");
    if (hv[2]) return fail(EGG_ERR_TIMEOUT, "barrier check: the bounded wait ran out");
    return EGG_OK;
}

}  // namespace egg
