/*
 * eggman_oracle.c -- CPU restatement of TheEggman.jl's subset DP and Bjorklund/Glynn sieve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the smoke check and
 * the CPU-baseline leg of the benchmark call it.  Nothing in the product library links it,
 * and the product never falls back to it.
 *
 * It follows the reference line by line, with the same loop orders and the same arithmetic:
 *   - plan build        src/dp.jl:192-208 (_dp_counts), :223-304 (_build_dp_plan)
 *   - DP evaluation     src/dp.jl:344-363 (_dp_states!), :408-442 (_haf_dp, level chunking
 *                       :370-388), :452-462 (_gather_pairs!), src/unrolled.jl:60 (_pair_index)
 *   - sieve             src/hafnian.jl:142-188 (matched_reps), :210-258 (_hessenberg!),
 *                       :271-335 (_hessenberg_split!), :346-365 (_reduce_hessenberg!),
 *                       :454-492 (_charpoly_hessenberg!), :502-514 (_inv_sqrt_det_coeff!),
 *                       :528-602 (_glynn_term!), :608-623 (_haf_range), :626 (_term_cost),
 *                       :646-647 (_sieve_chunks), :684-738 (_calc_hafnian/_sieve_sum),
 *                       :855-884 (_sieve_variant_cost)
 *   - brute force       test/runtests.jl:11-25 (brute_hafnian)
 *   - Householder       src/hafnian.jl:377-437 (test-only cross-check of the Gaussian reduction)
 *
 * Julia evaluates Float64/Float32 arithmetic without contracting a*b+c into an FMA, and its
 * Complex{T} product is (ar*br - ai*bi, ar*bi + ai*br).  This file is compiled with
 * -ffp-contract=off so that every expression rounds exactly as the reference's does.
 *
 * Beyond the reference it provides gold values: an __int128 DP for integer adjacency matrices,
 * and a __float128 DP (113-bit significand) whose no-cancellation sums are far more accurate
 * than any FP64 result they are compared with.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <quadmath.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } c128;
typedef struct { float re, im; } c64;
typedef struct { __float128 re, im; } cq;

static inline c128 c128_mul(c128 a, c128 b) { c128 r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline c128 c128_add(c128 a, c128 b) { c128 r = {a.re + b.re, a.im + b.im}; return r; }
static inline c128 c128_sub(c128 a, c128 b) { c128 r = {a.re - b.re, a.im - b.im}; return r; }
static inline c64 c64_mul(c64 a, c64 b) { c64 r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline c64 c64_add(c64 a, c64 b) { c64 r = {a.re + b.re, a.im + b.im}; return r; }
static inline cq cq_mul(cq a, cq b) { cq r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cq cq_add(cq a, cq b) { cq r = {a.re + b.re, a.im + b.im}; return r; }

enum { ORC_F64 = 0, ORC_C128 = 1, ORC_F32 = 2, ORC_C64 = 3, ORC_I64 = 4, ORC_Q_F64 = 5, ORC_Q_C128 = 6 };

/* ------------------------------------------------------------------------------------------ */
/* DP plan                                                                                     */
/* ------------------------------------------------------------------------------------------ */

static int64_t binom_i64(int64_t n, int64_t k)
{
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    __int128 r = 1;
    for (int64_t i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return (int64_t)r;
}

/* _pair_index(i, j, K), src/unrolled.jl:60 (1-based i < j). */
int64_t orc_pair_index(int64_t i, int64_t j, int64_t K) { return (i - 1) * K - (i * (i + 1)) / 2 + j; }

/* _dp_counts(K), src/dp.jl:192-208. */
void orc_dp_counts(int K, int64_t *nstates, int64_t *ntrans)
{
    int64_t ns = 1, nt = 0;
    for (int p = 1; p <= K; ++p) {
        int lo = p - 1;
        int hi = 2 * (p - 1) < K - 1 ? 2 * (p - 1) : K - 1;
        int r = (lo % 2 == 0) ? lo : lo + 1;
        while (r <= hi) {
            int64_t k = K - r - 1;
            int64_t c = binom_i64(K - p, k);
            ns += c;
            nt += c * k;
            r += 2;
        }
    }
    *nstates = ns;
    *ntrans = nt;
}

/* _pair_bits, src/dp.jl:170-171. */
static int pair_bits(int idx_bytes) { return idx_bytes == 4 ? 9 : 12; }

/* Open-addressed set/map from mask to 1-based state number (the reference uses Set/Dict). */
typedef struct { uint64_t *keys; int64_t *vals; uint64_t cap; } mask_map;

static uint64_t mix64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}
static int mm_init(mask_map *m, uint64_t n)
{
    uint64_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    m->cap = cap;
    m->keys = (uint64_t *)malloc(cap * sizeof(uint64_t));
    m->vals = (int64_t *)malloc(cap * sizeof(int64_t));
    if (!m->keys || !m->vals) return -1;
    memset(m->vals, 0xff, cap * sizeof(int64_t)); /* -1 marks an empty slot */
    return 0;
}
static void mm_free(mask_map *m) { free(m->keys); free(m->vals); }
static int64_t *mm_slot(mask_map *m, uint64_t key, int *found)
{
    uint64_t h = mix64(key) & (m->cap - 1);
    for (;;) {
        if (m->vals[h] == -1) { *found = 0; m->keys[h] = key; return &m->vals[h]; }
        if (m->keys[h] == key) { *found = 1; return &m->vals[h]; }
        h = (h + 1) & (m->cap - 1);
    }
}

static int cmp_mask(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    int cx = __builtin_popcountll(x), cy = __builtin_popcountll(y);
    if (cx != cy) return cx < cy ? -1 : 1;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/*
 * _build_dp_plan(K, I), src/dp.jl:223-304: DFS from the full mask, sort by (popcount, mask),
 * number the states, emit CSR with the partner j ascending, record level starts.
 * starts has nstates+1 entries, trans ntrans, levels K/2+2 (all 1-based, as the reference).
 * Returns 0, or -1 when the reference would refuse the layout (:224-234), -2 on allocation failure.
 */
int orc_build_plan(int K, int idx_bytes, void *starts_out, void *trans_out, void *levels_out, int64_t *nlevels_out)
{
    if (K < 0 || K > 64 || (idx_bytes != 4 && idx_bytes != 8)) return -1;
    int64_t nstates, ntrans;
    orc_dp_counts(K, &nstates, &ntrans);
    int bits = pair_bits(idx_bytes);
    int64_t npairs = (int64_t)K * (K - 1) / 2;
    int64_t pmask = ((int64_t)1 << bits) - 1;
    int64_t imax = idx_bytes == 4 ? INT32_MAX : INT64_MAX;
    if (npairs > pmask) return -1;
    if (nstates > (imax >> bits)) return -1;
    if (ntrans > imax) return -1;

    uint64_t full = K == 0 ? 0 : (~(uint64_t)0) >> (64 - K);
    mask_map seen;
    if (mm_init(&seen, (uint64_t)nstates)) return -2;
    uint64_t *masks = (uint64_t *)malloc((size_t)nstates * sizeof(uint64_t));
    uint64_t *stack = (uint64_t *)malloc((size_t)nstates * sizeof(uint64_t));
    if (!masks || !stack) { mm_free(&seen); free(masks); free(stack); return -2; }
    int64_t nm = 0, sp = 0;
    int found;
    *mm_slot(&seen, full, &found) = 0;
    masks[nm++] = full;
    stack[sp++] = full;
    while (sp > 0) {
        uint64_t m = stack[--sp];
        if (m == 0) continue;
        int i = __builtin_ctzll(m) + 1;
        uint64_t rest = m & ~((uint64_t)1 << (i - 1));
        uint64_t r = rest;
        while (r != 0) {
            int j = __builtin_ctzll(r) + 1;
            r &= ~((uint64_t)1 << (j - 1));
            uint64_t sub = rest & ~((uint64_t)1 << (j - 1));
            int64_t *slot = mm_slot(&seen, sub, &found);
            if (!found) {
                *slot = 0;
                masks[nm++] = sub;
                stack[sp++] = sub;
            }
        }
    }
    free(stack);
    if (nm != nstates) { mm_free(&seen); free(masks); return -3; }
    qsort(masks, (size_t)nstates, sizeof(uint64_t), cmp_mask);
    for (int64_t s = 0; s < nstates; ++s) *mm_slot(&seen, masks[s], &found) = s + 1;

    int64_t n = 0;
    int64_t *st64 = (int64_t *)starts_out, *tr64 = (int64_t *)trans_out, *lv64 = (int64_t *)levels_out;
    int32_t *st32 = (int32_t *)starts_out, *tr32 = (int32_t *)trans_out, *lv32 = (int32_t *)levels_out;
#define PUT(arr32, arr64, idx, v) do { if (idx_bytes == 4) arr32[idx] = (int32_t)(v); else arr64[idx] = (int64_t)(v); } while (0)
    PUT(st32, st64, 0, 1);
    for (int64_t s = 0; s < nstates; ++s) {
        uint64_t m = masks[s];
        if (m != 0) {
            int i = __builtin_ctzll(m) + 1;
            uint64_t rest = m & ~((uint64_t)1 << (i - 1));
            uint64_t r = rest;
            while (r != 0) {
                int j = __builtin_ctzll(r) + 1;
                r &= ~((uint64_t)1 << (j - 1));
                int64_t c = *mm_slot(&seen, rest & ~((uint64_t)1 << (j - 1)), &found);
                int64_t t = (c << bits) | orc_pair_index(i, j, K);
                PUT(tr32, tr64, n, t);
                n += 1;
            }
        }
        PUT(st32, st64, s + 1, n + 1);
    }
    int64_t nl = 0;
    PUT(lv32, lv64, nl, 1); nl++;
    for (int64_t s = 1; s < nstates; ++s)
        if (__builtin_popcountll(masks[s]) != __builtin_popcountll(masks[s - 1])) { PUT(lv32, lv64, nl, s + 1); nl++; }
    PUT(lv32, lv64, nl, nstates + 1); nl++;
#undef PUT
    *nlevels_out = nl;
    mm_free(&seen);
    free(masks);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* DP evaluation                                                                               */
/* ------------------------------------------------------------------------------------------ */

static inline int64_t ld_idx(const void *a, int idx_bytes, int64_t i)
{
    return idx_bytes == 4 ? (int64_t)((const int32_t *)a)[i] : ((const int64_t *)a)[i];
}

/*
 * _dp_states!(H, P, starts, trans, lo, hi), src/dp.jl:344-363, for each element type.
 * lo, hi are 1-based inclusive; H and P are 1-based through the -1 offsets.
 */
#define DP_STATES_BODY(T, ZERO, MULADD)                                                        \
    for (int64_t s = lo; s <= hi; ++s) {                                                       \
        T acc = ZERO;                                                                          \
        int64_t k0 = ld_idx(starts, ib, s - 1), k1 = ld_idx(starts, ib, s);                    \
        for (int64_t k = k0; k < k1; ++k) {                                                    \
            int64_t t = ld_idx(trans, ib, k - 1);                                              \
            int64_t pi = t & pmask, ci = t >> bits;                                            \
            MULADD(acc, P[pi - 1], H[ci - 1]);                                                 \
        }                                                                                      \
        H[s - 1] = acc;                                                                        \
    }

#define MA_REAL(acc, p, h) acc += (p) * (h)
#define MA_C128(acc, p, h) acc = c128_add(acc, c128_mul(p, h))
#define MA_C64(acc, p, h) acc = c64_add(acc, c64_mul(p, h))
#define MA_I128(acc, p, h) acc += (__int128)(p) * (h)
#define MA_QR(acc, p, h) acc += (__float128)(p) * (h)
#define MA_QC(acc, p, h) do { cq pq = {(__float128)(p).re, (__float128)(p).im}; acc = cq_add(acc, cq_mul(pq, h)); } while (0)

static void dp_states(int dtype, void *Hv, const void *Pv, const void *starts, const void *trans, int ib,
                      int64_t lo, int64_t hi)
{
    int bits = pair_bits(ib);
    int64_t pmask = ((int64_t)1 << bits) - 1;
    switch (dtype) {
    case ORC_F64: { double *H = Hv; const double *P = Pv; DP_STATES_BODY(double, 0.0, MA_REAL) break; }
    case ORC_F32: { float *H = Hv; const float *P = Pv; DP_STATES_BODY(float, 0.0f, MA_REAL) break; }
    case ORC_C128: { c128 *H = Hv; const c128 *P = Pv; c128 z = {0, 0}; DP_STATES_BODY(c128, z, MA_C128) break; }
    case ORC_C64: { c64 *H = Hv; const c64 *P = Pv; c64 z = {0, 0}; DP_STATES_BODY(c64, z, MA_C64) break; }
    case ORC_I64: { __int128 *H = Hv; const int64_t *P = Pv; DP_STATES_BODY(__int128, 0, MA_I128) break; }
    case ORC_Q_F64: { __float128 *H = Hv; const double *P = Pv; DP_STATES_BODY(__float128, 0, MA_QR) break; }
    case ORC_Q_C128: { cq *H = Hv; const c128 *P = Pv; cq z = {0, 0}; DP_STATES_BODY(cq, z, MA_QC) break; }
    }
}

static size_t dp_elsize(int dtype)
{
    switch (dtype) {
    case ORC_F64: return 8;
    case ORC_F32: return 4;
    case ORC_C128: return 16;
    case ORC_C64: return 8;
    case ORC_I64: return 16;   /* state values are __int128 */
    case ORC_Q_F64: return 16; /* __float128 */
    case ORC_Q_C128: return 32;
    }
    return 0;
}

static void set_one(int dtype, void *H)
{
    switch (dtype) {
    case ORC_F64: ((double *)H)[0] = 1.0; break;
    case ORC_F32: ((float *)H)[0] = 1.0f; break;
    case ORC_C128: ((c128 *)H)[0].re = 1.0; ((c128 *)H)[0].im = 0.0; break;
    case ORC_C64: ((c64 *)H)[0].re = 1.0f; ((c64 *)H)[0].im = 0.0f; break;
    case ORC_I64: ((__int128 *)H)[0] = 1; break;
    case ORC_Q_F64: ((__float128 *)H)[0] = 1; break;
    case ORC_Q_C128: ((cq *)H)[0].re = 1; ((cq *)H)[0].im = 0; break;
    }
}

/* _DP_CHUNK_WORK, _DP_PARALLEL_MIN, _dp_level_chunks: src/dp.jl:370, :377, :387-388. */
#define DP_CHUNK_WORK 2000
#define DP_PARALLEL_MIN 60000
static int64_t dp_level_chunks(int64_t ntrans, int64_t nst, int64_t nthreads)
{
    int64_t c = ntrans / DP_CHUNK_WORK;
    int64_t hi = nthreads < nst ? nthreads : nst;
    if (c > hi) c = hi;
    if (c < 1) c = 1;
    return c;
}

/*
 * _haf_dp's forward pass over a plan, src/dp.jl:420-441, given the gathered pairs P (length
 * K(K-1)/2).  `out` receives H[nstates] (for ORC_I64 an __int128, for the quad types the
 * __float128 value(s)).  nthreads > 1 reproduces the reference's per-level chunking; the result
 * is bit-identical either way because each state is accumulated by one task in plan order.
 */
int orc_haf_dp(int dtype, int idx_bytes, const void *starts, const void *trans, const void *levels,
               int64_t nlevels, int64_t nstates, const void *P, int nthreads, void *out)
{
    size_t es = dp_elsize(dtype);
    if (!es || nstates < 1) return -1;
    void *H = malloc((size_t)nstates * es);
    if (!H) return -2;
    set_one(dtype, H);
    int64_t ntr_total = ld_idx(starts, idx_bytes, nstates) - 1;
    int parallel = nthreads > 1 && ntr_total >= DP_PARALLEL_MIN;
    for (int64_t L = 2; L <= nlevels - 1; ++L) {
        int64_t lo = ld_idx(levels, idx_bytes, L - 1);
        int64_t hi = ld_idx(levels, idx_bytes, L) - 1;
        int64_t n = hi - lo + 1;
        int64_t ntr = ld_idx(starts, idx_bytes, hi) - ld_idx(starts, idx_bytes, lo - 1);
        int64_t nchunks = parallel ? dp_level_chunks(ntr, n, nthreads) : 1;
        if (nchunks == 1) {
            dp_states(dtype, H, P, starts, trans, idx_bytes, lo, hi);
        } else {
#pragma omp parallel for schedule(static, 1) num_threads(nthreads)
            for (int64_t c = 1; c <= nchunks; ++c) {
                int64_t clo = lo + ((c - 1) * n) / nchunks;
                int64_t chi = lo + (c * n) / nchunks - 1;
                if (clo <= chi) dp_states(dtype, H, P, starts, trans, idx_bytes, clo, chi);
            }
        }
    }
    memcpy(out, (char *)H + (size_t)(nstates - 1) * es, es);
    free(H);
    return 0;
}

/*
 * Batched CPU loop, src/hafnian.jl:1226-1242 (_batch_cpu!): B instances, each evaluated serially,
 * spread over min(nthreads, B) contiguous chunks.  P is B x npairs, instance index fastest
 * (src/dp.jl:468-469).
 */
int orc_haf_dp_batch(int dtype, int idx_bytes, const void *starts, const void *trans, const void *levels,
                     int64_t nlevels, int64_t nstates, const void *P, int64_t B, int64_t npairs,
                     int nthreads, void *out)
{
    size_t es = dp_elsize(dtype);
    size_t pes = dtype == ORC_I64 ? 8 : (dtype == ORC_Q_F64 ? 8 : (dtype == ORC_Q_C128 ? 16 : es));
    int64_t nchunks = nthreads < B ? nthreads : B;
    if (nchunks < 1) nchunks = 1;
    int err = 0;
#pragma omp parallel for schedule(static, 1) num_threads(nchunks) reduction(| : err)
    for (int64_t c = 1; c <= nchunks; ++c) {
        int64_t lo = ((c - 1) * B) / nchunks, hi = (c * B) / nchunks;
        char *Pb = (char *)malloc((size_t)npairs * pes);
        if (!Pb) { err |= 1; continue; }
        for (int64_t b = lo; b < hi; ++b) {
            for (int64_t q = 0; q < npairs; ++q)
                memcpy(Pb + q * pes, (const char *)P + ((size_t)q * B + b) * pes, pes);
            err |= orc_haf_dp(dtype, idx_bytes, starts, trans, levels, nlevels, nstates, Pb, 1,
                              (char *)out + (size_t)b * es) != 0;
        }
        free(Pb);
    }
    return err ? -1 : 0;
}

/*
 * The same forward pass without a stored plan, for degrees whose plan would not fit in host memory
 * (N = 36: 3.2 GB of transitions, N = 40: 24 GB).  It walks exactly the states and transitions
 * _build_dp_plan (src/dp.jl:223-304) would list, in its order, and sums each state as _dp_states!
 * (:344-363) does:
 *   - A non-empty mask S with r = K - |S| bits removed is reachable iff r <= 2(min(S) - 1)
 *     (src/dp.jl:16-27, 1-based min), so the reachable masks of popcount c are exactly the
 *     c-subsets of the bits m0..K-1 (0-based) with m0 = (K - c)/2, and sorting by
 *     (popcount, mask) lists each level in colex order of the element sets shifted down by m0.
 *     A state is identified by (c, colex rank); only two levels are kept.
 *   - State S (lowest bit i) has one transition per other bit j, ascending (:283-292), to the
 *     child S \ {i, j} of level c - 2 with pair index _pair_index(i, j, K) (src/unrolled.jl:60).
 *     The child's colex rank is found from its elements with the binomial table.
 * Each state is accumulated by one thread in plan order, so the value is bit-identical to
 * orc_haf_dp on the stored plan for any thread count; the tests pin this against orc_build_plan
 * (transition by transition, and value by value) for K <= 28.  Supports ORC_F64, ORC_C128,
 * ORC_I64 (Int128 states) and ORC_Q_F64.
 */
static int64_t g_cbinom[65][65];
static void cbinom_init(void)
{
    if (g_cbinom[0][0] == 1) return;
    for (int n = 0; n <= 64; ++n)
        for (int k = 0; k <= 64; ++k) g_cbinom[n][k] = binom_i64(n, k);
}

/* The colex unrank of r among the c-subsets of {0..U-1}: elements e[1] < ... < e[c]. */
static void colex_unrank(int64_t r, int c, int U, int *e)
{
    int x = U - 1;
    for (int i = c; i >= 1; --i) {
        while (g_cbinom[x][i] > r) --x;
        e[i] = x;
        r -= g_cbinom[x][i];
        --x;
    }
}

/* The closed-form plan's transitions of degree K, in the stored layout (the test compares them
 * with orc_build_plan's, entry for entry).  trans_out has ntrans entries of idx_bytes. */
int orc_closed_trans(int K, int idx_bytes, void *trans_out)
{
    if (K < 2 || K > 64 || (K & 1) || (idx_bytes != 4 && idx_bytes != 8)) return -1;
    cbinom_init();
    const int bits = pair_bits(idx_bytes);
    int64_t n = 0, child_lo1 = 1; /* 1-based number of the child level's first state */
    int64_t level_lo1 = 2;        /* level c = 2 starts after the empty set */
    for (int c = 2; c <= K; c += 2) {
        const int m0 = (K - c) / 2, U = K - m0;
        const int64_t cnt = g_cbinom[U][c];
        for (int64_t r = 0; r < cnt; ++r) {
            int e[66];
            colex_unrank(r, c, U, e);
            const int64_t i1 = e[1] + m0 + 1;
            for (int j = 2; j <= c; ++j) {
                int64_t rank = 0;
                for (int x = 2; x <= c; ++x) {
                    if (x == j) continue;
                    const int pos = x < j ? x - 1 : x - 2; /* position in the child's set */
                    rank += g_cbinom[e[x] - 1][pos];
                }
                const int64_t t = ((child_lo1 + rank) << bits) | orc_pair_index(i1, e[j] + m0 + 1, K);
                if (idx_bytes == 4) ((int32_t *)trans_out)[n] = (int32_t)t;
                else ((int64_t *)trans_out)[n] = t;
                ++n;
            }
        }
        child_lo1 = level_lo1;
        level_lo1 += cnt;
    }
    return 0;
}

#define CLOSED_LEVEL_BODY(T, ZERO, MULADD)                                                      \
    _Pragma("omp parallel num_threads(nthreads)")                                              \
    {                                                                                          \
        int nt_ = 1, id_ = 0;                                                                  \
        CLOSED_OMP_IDS(nt_, id_);                                                              \
        const int64_t r0 = cnt * id_ / nt_, r1 = cnt * (id_ + 1) / nt_;                        \
        int e[66];                                                                             \
        int64_t suf[67];                                                                       \
        if (r0 < r1) colex_unrank(r0, c, U, e);                                                \
        for (int64_t r = r0; r < r1; ++r) {                                                    \
            if (r > r0) { /* colex successor: raise the lowest element that can move */        \
                int x = 1;                                                                     \
                while (x < c && e[x] + 1 == e[x + 1]) ++x;                                     \
                e[x] += 1;                                                                     \
                for (int y = 1; y < x; ++y) e[y] = y - 1;                                      \
            }                                                                                  \
            suf[c + 1] = 0;                                                                    \
            suf[c] = 0;                                                                        \
            for (int x = c; x >= 3; --x) suf[x - 1] = suf[x] + g_cbinom[e[x] - 1][x - 2];      \
            int64_t pre = 0;                                                                   \
            const int64_t i1 = e[1] + m0 + 1;                                                  \
            T acc = ZERO;                                                                      \
            for (int j = 2; j <= c; ++j) {                                                     \
                const int64_t q = orc_pair_index(i1, e[j] + m0 + 1, K);                        \
                MULADD(acc, P[q - 1], prev[pre + suf[j]]);                                     \
                pre += g_cbinom[e[j] - 1][j - 1];                                              \
            }                                                                                  \
            cur[r] = acc;                                                                      \
        }                                                                                      \
    }

#ifdef _OPENMP
#define CLOSED_OMP_IDS(nt, id) do { nt = omp_get_num_threads(); id = omp_get_thread_num(); } while (0)
#else
#define CLOSED_OMP_IDS(nt, id) do { } while (0)
#endif

int orc_haf_dp_closed(int dtype, int K, const void *Pv, int nthreads, void *out)
{
    if (K < 0 || K > 64 || (K & 1)) return -1;
    if (dtype != ORC_F64 && dtype != ORC_C128 && dtype != ORC_I64 && dtype != ORC_Q_F64) return -1;
    cbinom_init();
    const size_t es = dp_elsize(dtype);
    if (nthreads < 1) nthreads = 1;
    if (K == 0) { set_one(dtype, out); return 0; }
    int64_t maxlev = 1;
    for (int c = 2; c <= K; c += 2) {
        const int U = K - (K - c) / 2;
        if (g_cbinom[U][c] > maxlev) maxlev = g_cbinom[U][c];
    }
    char *buf0 = (char *)malloc((size_t)maxlev * es), *buf1 = (char *)malloc((size_t)maxlev * es);
    if (!buf0 || !buf1) { free(buf0); free(buf1); return -2; }
    set_one(dtype, buf0); /* the empty set */
    char *pv = buf0, *cv = buf1;
    for (int c = 2; c <= K; c += 2) {
        const int m0 = (K - c) / 2, U = K - m0;
        const int64_t cnt = g_cbinom[U][c];
        switch (dtype) {
        case ORC_F64: { const double *P = Pv, *prev = (const double *)pv; double *cur = (double *)cv;
                        CLOSED_LEVEL_BODY(double, 0.0, MA_REAL) break; }
        case ORC_C128: { const c128 *P = Pv, *prev = (const c128 *)pv; c128 *cur = (c128 *)cv; const c128 z = {0, 0};
                         CLOSED_LEVEL_BODY(c128, z, MA_C128) break; }
        case ORC_I64: { const int64_t *P = Pv; const __int128 *prev = (const __int128 *)pv; __int128 *cur = (__int128 *)cv;
                        CLOSED_LEVEL_BODY(__int128, 0, MA_I128) break; }
        case ORC_Q_F64: { const double *P = Pv; const __float128 *prev = (const __float128 *)pv; __float128 *cur = (__float128 *)cv;
                          CLOSED_LEVEL_BODY(__float128, 0, MA_QR) break; }
        }
        char *t = pv; pv = cv; cv = t;
    }
    memcpy(out, pv, es); /* the last level holds one state, the full mask */
    free(buf0);
    free(buf1);
    return 0;
}

/* _gather_pairs!(P, A, idx, K), src/dp.jl:452-462.  A is column-major N x N, idx 1-based. */
void orc_gather_pairs(int dtype, const void *A, int64_t N, const int64_t *idx, int64_t K, void *P)
{
    size_t es = dtype == ORC_C128 ? 16 : (dtype == ORC_F32 ? 4 : 8);
    for (int64_t i = 1; i <= K - 1; ++i)
        for (int64_t j = i + 1; j <= K; ++j) {
            int64_t q = orc_pair_index(i, j, K);
            memcpy((char *)P + (q - 1) * es, (const char *)A + ((idx[j - 1] - 1) * N + (idx[i - 1] - 1)) * es, es);
        }
}

/* ------------------------------------------------------------------------------------------ */
/* Brute force, test/runtests.jl:11-25                                                         */
/* ------------------------------------------------------------------------------------------ */

static void brute_rec_r(const double *A, int64_t N, int *rem, int nrem, double *out)
{
    if (nrem == 0) { *out = 1.0; return; }
    int i = rem[0];
    double s = 0.0;
    int sub[64];
    for (int t = 1; t < nrem; ++t) {
        int ns = 0;
        for (int k = 1; k < nrem; ++k) if (k != t) sub[ns++] = rem[k];
        double v;
        brute_rec_r(A, N, sub, ns, &v);
        s += A[(int64_t)rem[t] * N + i] * v;
    }
    *out = s;
}
static void brute_rec_c(const c128 *A, int64_t N, int *rem, int nrem, c128 *out)
{
    if (nrem == 0) { out->re = 1.0; out->im = 0.0; return; }
    int i = rem[0];
    c128 s = {0, 0};
    int sub[64];
    for (int t = 1; t < nrem; ++t) {
        int ns = 0;
        for (int k = 1; k < nrem; ++k) if (k != t) sub[ns++] = rem[k];
        c128 v;
        brute_rec_c(A, N, sub, ns, &v);
        s = c128_add(s, c128_mul(A[(int64_t)rem[t] * N + i], v));
    }
    *out = s;
}
/* A column-major; A[i, rem[t]] is at rem[t]*N + i (0-based). */
int orc_brute_hafnian(int dtype, const void *A, int64_t N, void *out)
{
    if (N > 20) return -1;
    int rem[64];
    for (int k = 0; k < N; ++k) rem[k] = k;
    if (N % 2) {
        if (dtype == ORC_F64) *(double *)out = 0.0; else { ((c128 *)out)->re = 0; ((c128 *)out)->im = 0; }
        return 0;
    }
    if (dtype == ORC_F64) brute_rec_r((const double *)A, N, rem, (int)N, (double *)out);
    else brute_rec_c((const c128 *)A, N, rem, (int)N, (c128 *)out);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* matched_reps, src/hafnian.jl:142-188                                                        */
/* ------------------------------------------------------------------------------------------ */

/* Insertion sort, descending by (count, row) -- tuple order, as sort!(v; rev=true). */
static void sort_desc(int64_t *cnt, int64_t *row, int64_t n)
{
    for (int64_t a = 1; a < n; ++a) {
        int64_t c = cnt[a], r = row[a], b = a - 1;
        while (b >= 0 && (cnt[b] < c || (cnt[b] == c && row[b] < r))) {
            cnt[b + 1] = cnt[b];
            row[b + 1] = row[b];
            --b;
        }
        cnt[b + 1] = c;
        row[b + 1] = r;
    }
}

/* x has room for 2*len(rpt) entries, edge_reps for len(rpt); *E receives the edge count. */
int orc_matched_reps(const int64_t *rpt, int64_t N, int64_t *x, int64_t *edge_reps, int64_t *E_out)
{
    int64_t *cnt = malloc((size_t)(N + 1) * sizeof(int64_t)), *row = malloc((size_t)(N + 1) * sizeof(int64_t));
    int64_t *eA = malloc((size_t)(2 * N + 2) * sizeof(int64_t)), *eB = malloc((size_t)(2 * N + 2) * sizeof(int64_t));
    int64_t n = 0, E = 0;
    for (int64_t i = 0; i < N; ++i)
        if (rpt[i] > 0) { cnt[n] = rpt[i]; row[n] = i + 1; ++n; }
    if (n > 0) {
        sort_desc(cnt, row, n);
        while (n > 1 || (n == 1 && cnt[0] > 1)) {
            sort_desc(cnt, row, n);
            int64_t reps1 = cnt[0], x1 = row[0];
            if (n == 1 || reps1 > 2 * cnt[1]) {
                eA[E] = x1; eB[E] = x1; edge_reps[E] = reps1 / 2; ++E;
                if (reps1 % 2 == 0) {
                    memmove(cnt, cnt + 1, (size_t)(n - 1) * sizeof(int64_t));
                    memmove(row, row + 1, (size_t)(n - 1) * sizeof(int64_t));
                    --n;
                } else {
                    cnt[0] = 1;
                }
            } else {
                int64_t reps2 = cnt[1], x2 = row[1];
                eA[E] = x1; eB[E] = x2; edge_reps[E] = reps2; ++E;
                if (reps1 > reps2) {
                    cnt[0] = reps1 - reps2;
                    memmove(cnt + 1, cnt + 2, (size_t)(n - 2) * sizeof(int64_t));
                    memmove(row + 1, row + 2, (size_t)(n - 2) * sizeof(int64_t));
                    --n;
                } else {
                    memmove(cnt, cnt + 2, (size_t)(n - 2) * sizeof(int64_t));
                    memmove(row, row + 2, (size_t)(n - 2) * sizeof(int64_t));
                    n -= 2;
                }
            }
        }
    }
    for (int64_t e = 0; e < E; ++e) { x[e] = eA[e]; x[E + e] = eB[e]; }
    *E_out = E;
    free(cnt); free(row); free(eA); free(eB);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Sieve kernels                                                                               */
/* ------------------------------------------------------------------------------------------ */

/* _hessenberg!(M, m, mult), src/hafnian.jl:210-258 (real).  M column-major, leading dim ld. */
static void hessenberg_real(double *M, int ld, int m, double *mult)
{
#define Mx(i, j) M[((j) - 1) * ld + ((i) - 1)]
    for (int k = 2; k <= m - 1; ++k) {
        int p = k;
        double big = fabs(Mx(k, k - 1));
        for (int i = k + 1; i <= m; ++i) {
            double a = fabs(Mx(i, k - 1));
            if (a > big) { big = a; p = i; }
        }
        if (p != k) {
            for (int j = k - 1; j <= m; ++j) { double t = Mx(p, j); Mx(p, j) = Mx(k, j); Mx(k, j) = t; }
            for (int i = 1; i <= m; ++i) { double t = Mx(i, p); Mx(i, p) = Mx(i, k); Mx(i, k) = t; }
        }
        double x = Mx(k, k - 1);
        if (x == 0.0) continue;
        for (int i = k + 1; i <= m; ++i) { mult[i - 1] = Mx(i, k - 1) / x; Mx(i, k - 1) = 0.0; }
        for (int j = k; j <= m; ++j) {
            double akj = Mx(k, j);
            if (akj == 0.0) continue;
            for (int i = k + 1; i <= m; ++i) Mx(i, j) -= mult[i - 1] * akj;
        }
        for (int i = k + 1; i <= m; ++i) {
            double mi = mult[i - 1];
            if (mi == 0.0) continue;
            for (int l = 1; l <= m; ++l) Mx(l, k) += mi * Mx(l, i);
        }
    }
#undef Mx
}

/* _hessenberg_split!(Mr, Mi, m, ur, ui), src/hafnian.jl:271-335 (complex, split storage). */
static void hessenberg_split(double *Mr, double *Mi, int ld, int m, double *ur, double *ui)
{
#define R(i, j) Mr[((j) - 1) * ld + ((i) - 1)]
#define I(i, j) Mi[((j) - 1) * ld + ((i) - 1)]
    for (int k = 2; k <= m - 1; ++k) {
        int p = k;
        double big = R(k, k - 1) * R(k, k - 1) + I(k, k - 1) * I(k, k - 1);
        for (int i = k + 1; i <= m; ++i) {
            double a = R(i, k - 1) * R(i, k - 1) + I(i, k - 1) * I(i, k - 1);
            if (a > big) { big = a; p = i; }
        }
        if (p != k) {
            for (int j = k - 1; j <= m; ++j) {
                double t = R(p, j); R(p, j) = R(k, j); R(k, j) = t;
                t = I(p, j); I(p, j) = I(k, j); I(k, j) = t;
            }
            for (int i = 1; i <= m; ++i) {
                double t = R(i, p); R(i, p) = R(i, k); R(i, k) = t;
                t = I(i, p); I(i, p) = I(i, k); I(i, k) = t;
            }
        }
        double xr = R(k, k - 1), xi = I(k, k - 1);
        double d = xr * xr + xi * xi;
        if (d == 0.0) continue;
        for (int i = k + 1; i <= m; ++i) {
            double ar = R(i, k - 1), ai = I(i, k - 1);
            ur[i - 1] = (ar * xr + ai * xi) / d;
            ui[i - 1] = (ai * xr - ar * xi) / d;
            R(i, k - 1) = 0.0;
            I(i, k - 1) = 0.0;
        }
        for (int j = k; j <= m; ++j) {
            double ar = R(k, j), ai = I(k, j);
            for (int i = k + 1; i <= m; ++i) {
                R(i, j) -= ur[i - 1] * ar - ui[i - 1] * ai;
                I(i, j) -= ur[i - 1] * ai + ui[i - 1] * ar;
            }
        }
        for (int i = k + 1; i <= m; ++i) {
            double mr = ur[i - 1], mi = ui[i - 1];
            for (int l = 1; l <= m; ++l) {
                R(l, k) += mr * R(l, i) - mi * I(l, i);
                I(l, k) += mr * I(l, i) + mi * R(l, i);
            }
        }
    }
#undef R
#undef I
}

/*
 * _charpoly_hessenberg!(C, H, m, n), src/hafnian.jl:454-492.  H column-major (ld), C is
 * (m+1) x (n+1) column-major with leading dim m+1.  Generic in T: real (im == NULL) or complex.
 */
static void charpoly_real(double *C, const double *H, int ld, int m, int n)
{
#define Hx(i, j) H[((j) - 1) * ld + ((i) - 1)]
#define Cx(i, j) C[((j) - 1) * (m + 1) + ((i) - 1)]
    Cx(1, 1) = 1.0;
    for (int t = 1; t <= n; ++t) Cx(1, t + 1) = 0.0;
    for (int k = 1; k <= m; ++k) {
        double hkk = Hx(k, k);
        int tmax = k < n ? k : n;
        int prevmax = (k - 1) < n ? (k - 1) : n;
        Cx(k + 1, 1) = Cx(k, 1);
        for (int t = 1; t <= tmax; ++t) {
            double a = t <= prevmax ? Cx(k, t + 1) : 0.0;
            Cx(k + 1, t + 1) = a - hkk * Cx(k, t);
        }
        for (int t = tmax + 1; t <= n; ++t) Cx(k + 1, t + 1) = 0.0;
        double beta = 1.0;
        int ilo = 1 > k - n + 1 ? 1 : k - n + 1;
        for (int i = k - 1; i >= ilo; --i) {
            beta *= Hx(i + 1, i);
            if (beta == 0.0) break;
            double coef = Hx(i, k) * beta;
            int d = k - i + 1;
            if (coef != 0.0) {
                int tt = n < d + i - 1 ? n : d + i - 1;
                for (int t = d; t <= tt; ++t) Cx(k + 1, t + 1) -= coef * Cx(i, t - d + 1);
            }
        }
    }
#undef Hx
#undef Cx
}

static void charpoly_cplx(c128 *C, const c128 *H, int ld, int m, int n)
{
#define Hx(i, j) H[((j) - 1) * ld + ((i) - 1)]
#define Cx(i, j) C[((j) - 1) * (m + 1) + ((i) - 1)]
    c128 one = {1.0, 0.0}, zero = {0.0, 0.0};
    Cx(1, 1) = one;
    for (int t = 1; t <= n; ++t) Cx(1, t + 1) = zero;
    for (int k = 1; k <= m; ++k) {
        c128 hkk = Hx(k, k);
        int tmax = k < n ? k : n;
        int prevmax = (k - 1) < n ? (k - 1) : n;
        Cx(k + 1, 1) = Cx(k, 1);
        for (int t = 1; t <= tmax; ++t) {
            c128 a = t <= prevmax ? Cx(k, t + 1) : zero;
            Cx(k + 1, t + 1) = c128_sub(a, c128_mul(hkk, Cx(k, t)));
        }
        for (int t = tmax + 1; t <= n; ++t) Cx(k + 1, t + 1) = zero;
        c128 beta = one;
        int ilo = 1 > k - n + 1 ? 1 : k - n + 1;
        for (int i = k - 1; i >= ilo; --i) {
            beta = c128_mul(beta, Hx(i + 1, i));
            if (beta.re == 0.0 && beta.im == 0.0) break;
            c128 coef = c128_mul(Hx(i, k), beta);
            int d = k - i + 1;
            if (!(coef.re == 0.0 && coef.im == 0.0)) {
                int tt = n < d + i - 1 ? n : d + i - 1;
                for (int t = d; t <= tt; ++t) Cx(k + 1, t + 1) = c128_sub(Cx(k + 1, t + 1), c128_mul(coef, Cx(i, t - d + 1)));
            }
        }
    }
#undef Hx
#undef Cx
}

/* _inv_sqrt_det_coeff!(f, q, m, n), src/hafnian.jl:502-514.  q[j] (0-based) = [lambda^j]. */
static double inv_sqrt_real(double *f, const double *q, int qstride, int m, int n)
{
    f[0] = 1.0;
    for (int t = 1; t <= n; ++t) {
        double s = 0.0;
        int jm = t < m ? t : m;
        for (int j = 1; j <= jm; ++j) s += ((double)(2 * t - j) * q[j * qstride]) * f[t - j];
        f[t] = -s / (double)(2 * t);
    }
    return f[n];
}

static c128 inv_sqrt_cplx(c128 *f, const c128 *q, int qstride, int m, int n)
{
    f[0].re = 1.0; f[0].im = 0.0;
    for (int t = 1; t <= n; ++t) {
        c128 s = {0.0, 0.0};
        int jm = t < m ? t : m;
        for (int j = 1; j <= jm; ++j) {
            double w = (double)(2 * t - j);
            c128 wq = {w * q[j * qstride].re, w * q[j * qstride].im};
            s = c128_add(s, c128_mul(wq, f[t - j]));
        }
        double dd = (double)(2 * t);
        f[t].re = -s.re / dd;
        f[t].im = -s.im / dd;
    }
    return f[n];
}

typedef struct {
    int E, n, glynn, cplx, maxrep;
    const void *Ax;     /* 2E x 2E column-major */
    const int64_t *edge_reps;
    const double *binoms; /* (maxrep+1) x (maxrep+1) column-major: binoms[a + b*(maxrep+1)] = C(a, b) */
} sieve_ctx;

typedef struct {
    double *M, *v, *Mr, *Mi, *ur, *ui, *C, *f;
    int64_t *kept, *idx, *rows;
} sieve_ws;

static int ws_alloc(sieve_ws *w, int E, int n)
{
    int m = 2 * E;
    w->M = malloc(sizeof(double) * 2 * (size_t)(m * m + 1));
    w->v = malloc(sizeof(double) * 2 * (size_t)(m + 1));
    w->Mr = malloc(sizeof(double) * (size_t)(m * m + 1));
    w->Mi = malloc(sizeof(double) * (size_t)(m * m + 1));
    w->ur = malloc(sizeof(double) * (size_t)(m + 1));
    w->ui = malloc(sizeof(double) * (size_t)(m + 1));
    w->C = malloc(sizeof(double) * 2 * (size_t)((m + 1) * (n + 1)));
    w->f = malloc(sizeof(double) * 2 * (size_t)(n + 1));
    w->kept = malloc(sizeof(int64_t) * (size_t)(E + 1));
    w->idx = malloc(sizeof(int64_t) * (size_t)(E + 1));
    w->rows = malloc(sizeof(int64_t) * (size_t)(m + 1));
    return (w->M && w->v && w->Mr && w->Mi && w->ur && w->ui && w->C && w->f && w->kept && w->idx && w->rows) ? 0 : -1;
}
static void ws_free(sieve_ws *w)
{
    free(w->M); free(w->v); free(w->Mr); free(w->Mi); free(w->ur); free(w->ui);
    free(w->C); free(w->f); free(w->kept); free(w->idx); free(w->rows);
}

/*
 * _glynn_term!(ws, Ax, edge_reps, n, j, binoms, glynn), src/hafnian.jl:528-602.
 * Writes the term value (real in out[0], complex in out[0..1]).
 */
static void glynn_term(const sieve_ctx *c, sieve_ws *w, int64_t j, double *out)
{
    int E = c->E, n = c->n, glynn = c->glynn;
    int64_t num = j, edge_sum = 0;
    double binom_prod = 1.0;
    int mr1 = c->maxrep + 1;
    for (int i = E; i >= 1; --i) {
        int64_t r = c->edge_reps[i - 1];
        int64_t b = r + 1;
        int64_t k = num % b;
        num /= b;
        w->kept[i - 1] = k;
        edge_sum += k;
        binom_prod *= c->binoms[r + k * mr1];
    }
    int mE = 0;
    for (int i = 1; i <= E; ++i) {
        int64_t k = glynn ? 2 * w->kept[i - 1] - c->edge_reps[i - 1] : w->kept[i - 1];
        w->kept[i - 1] = k;
        if (k != 0) { w->idx[mE] = i; ++mE; }
    }
    int m = 2 * mE;
    if (m == 0) { out[0] = 0.0; out[1] = 0.0; return; }
    double prefac = ((n - edge_sum) % 2 != 0) ? -binom_prod : binom_prod;
    if (glynn && w->kept[0] == 0) prefac /= 2;
    for (int a = 1; a <= mE; ++a) { w->rows[a - 1] = w->idx[a - 1]; w->rows[mE + a - 1] = w->idx[a - 1] + E; }
    int twoE = 2 * E;
    if (!c->cplx) {
        const double *Ax = c->Ax;
        double *M = w->M;
        for (int b = 1; b <= mE; ++b) {
            double kb = (double)w->kept[w->idx[b - 1] - 1];
            int64_t cb1 = w->idx[b - 1] + E, cb2 = w->idx[b - 1];
            for (int a = 1; a <= m; ++a) {
                int64_t ra = w->rows[a - 1];
                M[(b - 1) * m + (a - 1)] = kb * Ax[(cb1 - 1) * twoE + (ra - 1)];
                M[(mE + b - 1) * m + (a - 1)] = kb * Ax[(cb2 - 1) * twoE + (ra - 1)];
            }
        }
        hessenberg_real(M, m, m, w->v);
        charpoly_real(w->C, M, m, m, n);
        double val = inv_sqrt_real(w->f, w->C + m, m + 1, m, n); /* row m+1 of C */
        out[0] = prefac * val;
        out[1] = 0.0;
    } else {
        const c128 *Ax = c->Ax;
        c128 *M = (c128 *)w->M;
        for (int b = 1; b <= mE; ++b) {
            double kb = (double)w->kept[w->idx[b - 1] - 1];
            int64_t cb1 = w->idx[b - 1] + E, cb2 = w->idx[b - 1];
            for (int a = 1; a <= m; ++a) {
                int64_t ra = w->rows[a - 1];
                c128 z1 = Ax[(cb1 - 1) * twoE + (ra - 1)], z2 = Ax[(cb2 - 1) * twoE + (ra - 1)];
                c128 y1 = {kb * z1.re, kb * z1.im}, y2 = {kb * z2.re, kb * z2.im};
                M[(b - 1) * m + (a - 1)] = y1;
                M[(mE + b - 1) * m + (a - 1)] = y2;
            }
        }
        /* _reduce_hessenberg! for Complex{Float64}: split, reduce, copy back the band (:348-365). */
        for (int jj = 1; jj <= m; ++jj)
            for (int ii = 1; ii <= m; ++ii) {
                w->Mr[(jj - 1) * m + ii - 1] = M[(jj - 1) * m + ii - 1].re;
                w->Mi[(jj - 1) * m + ii - 1] = M[(jj - 1) * m + ii - 1].im;
            }
        hessenberg_split(w->Mr, w->Mi, m, m, w->ur, w->ui);
        for (int jj = 1; jj <= m; ++jj)
            for (int ii = 1; ii <= (jj + 1 < m ? jj + 1 : m); ++ii) {
                M[(jj - 1) * m + ii - 1].re = w->Mr[(jj - 1) * m + ii - 1];
                M[(jj - 1) * m + ii - 1].im = w->Mi[(jj - 1) * m + ii - 1];
            }
        c128 *C = (c128 *)w->C;
        charpoly_cplx(C, M, m, m, n);
        c128 val = inv_sqrt_cplx((c128 *)w->f, C + m, m + 1, m, n);
        out[0] = prefac * val.re;
        out[1] = prefac * val.im;
    }
}

/* _term_cost(E, n), src/hafnian.jl:626. */
static int64_t term_cost(int64_t E, int64_t n) { return (5 * (2 * E) * (2 * E) * (2 * E)) / 3 + 2 * E * n * n; }

static int64_t clamp_work(double x) { return x >= 9.0e18 ? INT64_MAX : (int64_t)nearbyint(x); }

/* _sieve_variant_cost(edge_reps, n, glynn), src/hafnian.jl:855-884. */
void orc_sieve_variant_cost(const int64_t *edge_reps, int E, int64_t n, int glynn, int64_t *work, int64_t *steps)
{
    if (E == 0) { *work = 0; *steps = 0; return; }
    double *counts = calloc((size_t)E + 2, sizeof(double));
    counts[0] = 1.0;
    for (int i = 1; i <= E; ++i) {
        int64_t r = edge_reps[i - 1];
        int64_t total = glynn ? (i == 1 ? (r + 2) / 2 : r + 1) : r + 1;
        int64_t nzero = glynn ? (r % 2 == 0 ? 1 : 0) : 1;
        int64_t nkeep = total - nzero;
        for (int cc = i - 1; cc >= 0; --cc) {
            double v = counts[cc];
            if (v == 0.0) continue;
            counts[cc] = v * (double)nzero;
            counts[cc + 1] += v * (double)nkeep;
        }
    }
    double wk = 0.0, st = 0.0;
    for (int cc = 0; cc <= E; ++cc) {
        if (counts[cc] == 0.0) continue;
        st += counts[cc];
        wk += counts[cc] * (double)term_cost(cc, n);
    }
    free(counts);
    *work = clamp_work(wk);
    *steps = clamp_work(st);
}

/* TwoSum-based double-double accumulation (Knuth); used by sum_mode 1. */
static inline void dd_add(double *hi, double *lo, double x)
{
    double s = *hi + x;
    double bp = s - *hi;
    double e = (*hi - (s - bp)) + (x - bp);
    double t = *lo + e;
    double h2 = s + t;
    *lo = t - (h2 - s);
    *hi = h2;
}

/*
 * _calc_hafnian(Ax, edge_reps; nthreads, glynn), src/hafnian.jl:684-738.
 *   sum_mode 0: the reference's own summation -- plain FP64 `+=` inside each of the
 *               _sieve_chunks(work, steps, nthreads) chunks, then the chunk sums in order.
 *   sum_mode 1: every term accumulated in double-double in term order (the GPU's accumulator
 *               is compared against this).
 * out: 1 (real) or 2 (complex) doubles.
 */
int orc_calc_hafnian(int cplx, const void *Ax, const int64_t *edge_reps, int E, int glynn, int nthreads,
                     int sum_mode, double *out)
{
    out[0] = 0.0; out[1] = 0.0;
    if (E == 0) { out[0] = 1.0; return 0; }
    int64_t n = 0, maxrep = 0;
    for (int i = 0; i < E; ++i) { n += edge_reps[i]; if (edge_reps[i] > maxrep) maxrep = edge_reps[i]; }
    int64_t work, steps;
    orc_sieve_variant_cost(edge_reps, E, n, glynn, &work, &steps);
    double *binoms = malloc(sizeof(double) * (size_t)((maxrep + 1) * (maxrep + 1)));
    for (int64_t a = 0; a <= maxrep; ++a)
        for (int64_t b = 0; b <= maxrep; ++b)
            binoms[a + b * (maxrep + 1)] = b <= a ? (double)binom_i64(a, b) : 0.0;
    sieve_ctx ctx = {E, (int)n, glynn, cplx, (int)maxrep, Ax, edge_reps, binoms};
    int64_t nchunks = (work < 90000) ? 1 : (nthreads < steps ? nthreads : steps); /* :646-647 */
    if (nchunks < 1) nchunks = 1;
    double *part = calloc((size_t)nchunks * 4, sizeof(double));
    int err = 0;
#pragma omp parallel for schedule(static, 1) num_threads((int)nchunks) reduction(| : err)
    for (int64_t c = 1; c <= nchunks; ++c) {
        int64_t lo = ((c - 1) * steps) / nchunks, hi = (c * steps) / nchunks - 1;
        sieve_ws w;
        if (ws_alloc(&w, E, (int)n)) { err |= 1; ws_free(&w); continue; }
        double hr = 0.0, hi_ = 0.0, lr = 0.0, li = 0.0, t[2];
        for (int64_t j = lo; j <= hi; ++j) {
            glynn_term(&ctx, &w, j, t);
            if (sum_mode == 0) { hr += t[0]; hi_ += t[1]; }
            else { dd_add(&hr, &lr, t[0]); dd_add(&hi_, &li, t[1]); }
        }
        part[4 * (c - 1) + 0] = hr; part[4 * (c - 1) + 1] = hi_;
        part[4 * (c - 1) + 2] = lr; part[4 * (c - 1) + 3] = li;
        ws_free(&w);
    }
    double Hr, Hi;
    if (sum_mode == 0) {
        /* sum(t -> fetch(t), tasks): Julia's sum over a short collection is a left fold. */
        Hr = part[0]; Hi = part[1];
        for (int64_t c = 1; c < nchunks; ++c) { Hr += part[4 * c]; Hi += part[4 * c + 1]; }
    } else {
        double ar = 0, al = 0, br = 0, bl = 0;
        for (int64_t c = 0; c < nchunks; ++c) {
            dd_add(&ar, &al, part[4 * c]); dd_add(&ar, &al, part[4 * c + 2]);
            dd_add(&br, &bl, part[4 * c + 1]); dd_add(&br, &bl, part[4 * c + 3]);
        }
        Hr = ar + al; Hi = br + bl;
    }
    if (glynn) {
        double s = 1.0;
        for (int64_t i = 0; i < n - 1; ++i) s *= 0.5; /* R(0.5)^(n-1), exact */
        Hr *= s; Hi *= s;
    }
    out[0] = Hr; out[1] = Hi;
    free(part); free(binoms);
    return err ? -1 : 0;
}

/* Individual term values j0..j0+cnt-1 of the sieve (for per-term parity checks). */
int orc_sieve_terms(int cplx, const void *Ax, const int64_t *edge_reps, int E, int glynn, int64_t j0, int64_t cnt,
                    double *out)
{
    int64_t n = 0, maxrep = 0;
    for (int i = 0; i < E; ++i) { n += edge_reps[i]; if (edge_reps[i] > maxrep) maxrep = edge_reps[i]; }
    double *binoms = malloc(sizeof(double) * (size_t)((maxrep + 1) * (maxrep + 1)));
    for (int64_t a = 0; a <= maxrep; ++a)
        for (int64_t b = 0; b <= maxrep; ++b)
            binoms[a + b * (maxrep + 1)] = b <= a ? (double)binom_i64(a, b) : 0.0;
    sieve_ctx ctx = {E, (int)n, glynn, cplx, (int)maxrep, Ax, edge_reps, binoms};
    sieve_ws w;
    if (ws_alloc(&w, E, (int)n)) { ws_free(&w); free(binoms); return -1; }
    for (int64_t j = 0; j < cnt; ++j) glynn_term(&ctx, &w, j0 + j, out + 2 * j);
    ws_free(&w);
    free(binoms);
    return 0;
}

/*
 * Gaussian vs Householder Hessenberg reductions on an arbitrary complex matrix (test/runtests.jl:
 * 160-191 compares them on the charpoly coefficients).  kind 0: Gaussian generic path (complex
 * arithmetic, src/hafnian.jl:210-258 applied to Complex{Float64}); kind 1: Householder
 * (:377-437).  Writes the n+1 coefficients of det(I - lambda*M), n = m/2.
 */
static void hessenberg_generic_c(c128 *M, int m, c128 *mult)
{
#define Mx(i, j) M[((j) - 1) * m + ((i) - 1)]
    for (int k = 2; k <= m - 1; ++k) {
        int p = k;
        double big = hypot(Mx(k, k - 1).re, Mx(k, k - 1).im);
        for (int i = k + 1; i <= m; ++i) {
            double a = hypot(Mx(i, k - 1).re, Mx(i, k - 1).im);
            if (a > big) { big = a; p = i; }
        }
        if (p != k) {
            for (int j = k - 1; j <= m; ++j) { c128 t = Mx(p, j); Mx(p, j) = Mx(k, j); Mx(k, j) = t; }
            for (int i = 1; i <= m; ++i) { c128 t = Mx(i, p); Mx(i, p) = Mx(i, k); Mx(i, k) = t; }
        }
        c128 x = Mx(k, k - 1);
        if (x.re == 0.0 && x.im == 0.0) continue;
        for (int i = k + 1; i <= m; ++i) {
            /* complex division; the precise formula only matters to the last ulp here */
            c128 a = Mx(i, k - 1);
            double den = x.re * x.re + x.im * x.im;
            c128 q = {(a.re * x.re + a.im * x.im) / den, (a.im * x.re - a.re * x.im) / den};
            mult[i - 1] = q;
            Mx(i, k - 1).re = 0.0; Mx(i, k - 1).im = 0.0;
        }
        for (int j = k; j <= m; ++j) {
            c128 akj = Mx(k, j);
            if (akj.re == 0.0 && akj.im == 0.0) continue;
            for (int i = k + 1; i <= m; ++i) Mx(i, j) = c128_sub(Mx(i, j), c128_mul(mult[i - 1], akj));
        }
        for (int i = k + 1; i <= m; ++i) {
            c128 mi = mult[i - 1];
            if (mi.re == 0.0 && mi.im == 0.0) continue;
            for (int l = 1; l <= m; ++l) Mx(l, k) = c128_add(Mx(l, k), c128_mul(mi, Mx(l, i)));
        }
    }
#undef Mx
}

static void hessenberg_householder_c(c128 *M, int m, c128 *v, c128 *w)
{
#define Mx(i, j) M[((j) - 1) * m + ((i) - 1)]
    for (int k = 1; k <= m - 2; ++k) {
        double nrm2 = 0.0;
        for (int i = k + 1; i <= m; ++i) nrm2 += Mx(i, k).re * Mx(i, k).re + Mx(i, k).im * Mx(i, k).im;
        if (nrm2 == 0.0) continue;
        c128 x1 = Mx(k + 1, k);
        double nrm = sqrt(nrm2);
        double ax1 = hypot(x1.re, x1.im);
        c128 sg;
        if (x1.re == 0.0 && x1.im == 0.0) { sg.re = nrm; sg.im = 0.0; }
        else { sg.re = nrm * (x1.re / ax1); sg.im = nrm * (x1.im / ax1); }
        for (int i = k + 1; i <= m; ++i) v[i - 1] = Mx(i, k);
        v[k] = c128_add(v[k], sg);
        double vn2 = 2 * (nrm2 + nrm * ax1);
        if (vn2 == 0.0) continue;
        double cc = 2 / vn2;
        Mx(k + 1, k).re = -sg.re; Mx(k + 1, k).im = -sg.im;
        for (int i = k + 2; i <= m; ++i) { Mx(i, k).re = 0.0; Mx(i, k).im = 0.0; }
        for (int j = k + 1; j <= m; ++j) {
            c128 s = {0, 0};
            for (int i = k + 1; i <= m; ++i) { c128 cv = {v[i - 1].re, -v[i - 1].im}; s = c128_add(s, c128_mul(cv, Mx(i, j))); }
            s.re *= cc; s.im *= cc;
            for (int i = k + 1; i <= m; ++i) Mx(i, j) = c128_sub(Mx(i, j), c128_mul(v[i - 1], s));
        }
        for (int i = 1; i <= m; ++i) { w[i - 1].re = 0; w[i - 1].im = 0; }
        for (int j = k + 1; j <= m; ++j) {
            c128 vj = v[j - 1];
            for (int i = 1; i <= m; ++i) w[i - 1] = c128_add(w[i - 1], c128_mul(Mx(i, j), vj));
        }
        for (int j = k + 1; j <= m; ++j) {
            c128 cv = {cc * v[j - 1].re, -cc * v[j - 1].im};
            for (int i = 1; i <= m; ++i) Mx(i, j) = c128_sub(Mx(i, j), c128_mul(w[i - 1], cv));
        }
    }
#undef Mx
}

int orc_charpoly_check(int kind, const c128 *M0, int m, c128 *coeffs)
{
    int n = m / 2;
    c128 *M = malloc(sizeof(c128) * (size_t)(m * m));
    c128 *v = malloc(sizeof(c128) * (size_t)(m + 1)), *w = malloc(sizeof(c128) * (size_t)(m + 1));
    c128 *C = malloc(sizeof(c128) * (size_t)((m + 1) * (n + 1)));
    memcpy(M, M0, sizeof(c128) * (size_t)(m * m));
    if (kind == 0) hessenberg_generic_c(M, m, v); else hessenberg_householder_c(M, m, v, w);
    charpoly_cplx(C, M, m, m, n);
    for (int t = 0; t <= n; ++t) coeffs[t] = C[t * (m + 1) + m];
    free(M); free(v); free(w); free(C);
    return 0;
}

/* Number of OpenMP threads available (for reporting the CPU baseline's core count). */
int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
