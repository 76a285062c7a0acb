// egg_sieve_tile.cuh -- one real sieve term on a register tile whose columns stay in logical order.
//
// The m x m matrix M = A_S X D of a term (src/hafnian.jl:583-593), m <= 32, is held one row per
// lane, one register per column.  The Gaussian similarity reduction to Hessenberg form
// (EISPACK elmhes, src/hafnian.jl:210-258) runs as m - 2 steps, each a separate instantiation of
// step_real<K> so that every column index is a compile-time constant:
//
//   * Rows are relabelled, not moved: each row carries its logical label, and swapping rows k and p
//     swaps two labels.
//   * Columns are moved: swapping columns k and p exchanges two registers in every lane.  The pivot
//     p is the same in all lanes, so the exchange is a branch tree on p (log2 of the live columns
//     deep) ending in a register swap, with no divergence.  Keeping columns in logical order is what
//     lets the work shrink with the step: step K updates only columns K .. m-1, and the column
//     update sums columns K+1 .. m-1 in ascending order, the reference's order.
//
// Two arithmetic forms share the tile:
//
//   * EXACT: every operation of the reference in its order and rounding -- the pivot is the first
//     row of largest |M[i, k-1]| (:212-221), multipliers are correctly rounded quotients, the row
//     update rounds the product and the difference separately (:239-245), and the column update
//     adds mult_i * M[l, i] for i ascending, each product and sum rounded (:248-255).  La Budde's
//     coefficients h_ik * beta are formed with beta multiplied down from h_{k,k-1} as the reference
//     walks i downwards (:476-490), and each coefficient row is accumulated i = k-1 first.  So each
//     term is bit-identical to _glynn_term! for finite inputs (a skipped zero multiplier or zero
//     pivot-row entry adds a signed zero here, which changes no nonzero value).
//   * FMA: fused multiply-adds, a Newton reciprocal for the multipliers, a pivot within 2^-13 of the
//     largest, and reassociated La Budde sums: faster, and within the rounding-error bound of the
//     reference's result.
//
// After the reduction the Hessenberg matrix is written to shared memory (its subdiagonal, its
// diagonal and the upper triangle by column), La Budde's coefficients are formed in place by one
// lane per order, and lane d computes diagonal d of the coefficient table in registers
// (labudde_diag*).  The caller turns q_1..q_n into the term value.
#pragma once

#include "egg_sieve_fast.cuh"

namespace egg {

// Shared-memory layout of one group's term workspace for the tile path, in doubles from the
// group's base: offsets depend only on the tile width mw (even), so every address is the base plus
// a constant.
//   prow  pivot row by column [64]            wv    column-update weights by row label [64]
//   cft   upper triangle by order k (cft_row_real(k) + i - 1), then La Budde's coefficients
//   hk    diagonal h_kk by order k             sub   subdiagonal h_{i+1,i} (1-based) at sub[i]
//   q     det(I - lambda H) coefficients q_j   kval  multiplicities of the surviving edges [32]
//   eidx  surviving edges, compacted (int) [32]
//   EXACT only: pre, jx, mx -- each buffered term's prefactor, index and size [32 each]; qbuf --
//   the buffered terms' q vectors, nmax + 1 doubles each (the series runs in batches).
__host__ __device__ constexpr int tile_off_cft() { return 128; }
__host__ __device__ constexpr int tile_off_hk(int mw) { return 128 + cft_row_real(mw + 1); }
__host__ __device__ constexpr int tile_off_sub(int mw) { return tile_off_hk(mw) + ((mw + 3) & ~1); }
__host__ __device__ constexpr int tile_off_q(int mw) { return tile_off_sub(mw) + ((mw + 3) & ~1); }
__host__ __device__ constexpr int tile_off_kval(int mw) { return tile_off_q(mw) + 32; }
__host__ __device__ constexpr int tile_off_eidx(int mw) { return tile_off_kval(mw) + 32; }
__host__ __device__ constexpr int tile_off_pre(int mw) { return tile_off_eidx(mw) + 16; }
__host__ __device__ constexpr int tile_off_jx(int mw) { return tile_off_pre(mw) + 32; }
__host__ __device__ constexpr int tile_off_mx(int mw) { return tile_off_jx(mw) + 32; }
__host__ __device__ constexpr int tile_off_qbuf(int mw) { return tile_off_mx(mw) + 16; }

__host__ __device__ inline size_t tile_ws_doubles(int nmax, int mhi, bool exact)
{
    const size_t d = exact ? (size_t)tile_off_qbuf(mhi) + 32 * (size_t)(nmax + 1) : (size_t)tile_off_pre(mhi);
    return (d + 1) & ~(size_t)1;  // keep every group's region 16-byte aligned
}

template <int MW>
struct TileWs {
    double *base;
    __device__ double *prow() const { return base; }
    __device__ double *wv() const { return base + 64; }
    __device__ double *cft() const { return base + tile_off_cft(); }
    __device__ double *hk() const { return base + tile_off_hk(MW); }
    __device__ double *sub() const { return base + tile_off_sub(MW); }
    __device__ double *q() const { return base + tile_off_q(MW); }
    __device__ double *kval() const { return base + tile_off_kval(MW); }
    __device__ int *eidx() const { return (int *)(base + tile_off_eidx(MW)); }
    __device__ double *pre() const { return base + tile_off_pre(MW); }
    __device__ long long *jx() const { return (long long *)(base + tile_off_jx(MW)); }
    __device__ int *mx() const { return (int *)(base + tile_off_mx(MW)); }
    __device__ double *qbuf() const { return base + tile_off_qbuf(MW); }
};

// The correctly rounded quotient a / b given y = RN(1/b), the same for every lane of a step
// (Markstein's division, "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Dev. 34(1), 1990; Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018,
// sec. 5.3): q0 = RN(a y) is within 1.5 ulp of a/b; one correction q1 = q0 + (a - b q0) y (the
// remainder exact in one fused multiply-add) brings it within 1 ulp; by Markstein's theorem a
// second correction from a reciprocal within half an ulp then yields RN(a/b).  Valid while nothing
// overflows or underflows: |b| and |a| within [2^-1000, 2^1000] and the quotient at least 2^-1000
// (here |a| <= |b|, the pivot being the largest entry); outside that, and for zero, Inf or NaN, the
// quotient comes from the correctly rounded division itself.  The parity tests hold every term of
// the N = 40 sieves to the reference's bits (the reference-order sum must equal the oracle's), so a
// quotient one ulp off anywhere would fail them.
__device__ __forceinline__ bool div_scale_ok(double v)
{
    const double av = fabs(v);
    return av >= 0x1p-1000 && av <= 0x1p+1000;
}
// The correctly rounded division itself, out of line: it is the rare path of every step, and kept
// inline it would sit between the hot instructions of consecutive steps (about 1 % of the N = 40
// exact sieve's time).
static __device__ __noinline__ double ddiv_cold(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double div_rn_shared(double a, double b, double y, bool b_ok)
{
    if (b_ok && div_scale_ok(a)) {
        const double q0 = __dmul_rn(a, y);
        const double r0 = __fma_rn(-b, q0, a);
        const double q1 = __fma_rn(r0, y, q0);
        const double r1 = __fma_rn(-b, q1, a);
        const double q2 = __fma_rn(r1, y, q1);
        if (fabs(q2) >= 0x1p-1000) return q2;
    }
    return ddiv_cold(a, b);
}

// 64-bit order key of |v| for the exact pivot search: non-negative doubles order as their bit
// patterns; +1 so that a candidate equal to zero still beats a non-candidate (key 0).  NaN never
// wins (key 0).
__device__ __forceinline__ unsigned long long abs_key(double a)
{
    if (a != a) return 0ull;
    return (unsigned long long)__double_as_longlong(fabs(a)) + 1ull;
}

// Exchange columns K and p (K < p < MW) of this lane's row: a branch tree on the warp-uniform p
// over the interval [LO, HI).
template <int K, int LO, int HI, int MW>
__device__ __forceinline__ void swap_cols(double (&R)[MW], int p)
{
    if constexpr (HI - LO == 1) {
        const double t = R[K];
        R[K] = R[LO];
        R[LO] = t;
    } else {
        constexpr int MID = (LO + HI) / 2;
        if (p < MID) swap_cols<K, LO, MID, MW>(R, p);
        else swap_cols<K, MID, HI, MW>(R, p);
    }
}

template <int MW, int G, bool EXACT>
struct TileCtx {
    double (&R)[MW];
    int &lab;
    const TileWs<MW> &ws;
    int m, lane;
    unsigned gm;
};

// Step K of the reduction (pivot row K, pivot column K - 1; 0-based), src/hafnian.jl:211-256.
template <int K, int MW, int G, bool EXACT>
__device__ __forceinline__ void step_real(TileCtx<MW, G, EXACT> &c)
{
    double (&R)[MW] = c.R;
    int &lab = c.lab;
    const int m = c.m;
    const bool cand = lab >= K && lab < m;
    // -- pivot: the row with label in [K, m) of largest |M[., K-1]|, and the lane pl holding it
    int plab, pl;
    if constexpr (EXACT) {
        // The first (lowest label) row achieving the maximum; if row K's own entry is NaN the
        // reference keeps it (no comparison with NaN succeeds, :212-218), so that row's key is the
        // largest there is, while any other NaN row's key is 0.
        const double v = R[K - 1];
        {
            unsigned long long key = cand ? abs_key(v) : 0ull;
            if (lab == K && v != v) key = ~0ull;
            const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
            const unsigned mhi = __reduce_max_sync(c.gm, hi);
            const unsigned mlo = __reduce_max_sync(c.gm, hi == mhi ? lo : 0u);
            const bool win = key != 0ull && hi == mhi && lo == mlo;
            // The lowest label among the maxima (one reduction serves the usual single maximum and
            // exact ties alike; the lane is found from the label below).
            plab = (int)__reduce_min_sync(c.gm, win ? (unsigned)lab : 0x7fffffffu);
            if (plab == 0x7fffffff) plab = K;
            pl = -1;
        }
    } else {
        const unsigned key = cand ? pivot_key(fabs(R[K - 1]), c.lane) : 0u;
        const unsigned best = __reduce_max_sync(c.gm, key);
        pl = 63 - (int)(best & 63u);
        plab = __shfl_sync(c.gm, lab, pl, G);
    }
    if (pl < 0) {
        pl = __ffs((int)__ballot_sync(c.gm, lab == plab)) - 1;
        if (G < 32) pl &= G - 1;
    }
    const double x = __shfl_sync(c.gm, R[K - 1], pl, G);
    // -- swap rows K and plab (relabel) and columns K and plab (move): a similarity (:222-229)
    if (lab == K) lab = plab;
    else if (lab == plab) lab = K;
    if (plab != K) swap_cols<K, K + 1, MW, MW>(R, plab);
    if (x == 0.0) return;  // column already clear below the subdiagonal (:231-232)
    // -- the multipliers of the rows below the pivot (:234-237)
    double mult = 0.0;
    if constexpr (EXACT) {
        // One correctly rounded reciprocal per step, shared by the lanes' quotients.
        const bool x_ok = div_scale_ok(x);
        const double y = x_ok ? __drcp_rn(x) : 0.0;
        if (lab > K && lab < m) mult = div_rn_shared(R[K - 1], x, y, x_ok);
    } else {
        const double rx = recip(x);
        if (lab > K && lab < m) mult = R[K - 1] * rx;
    }
    // -- broadcast the pivot row (columns K .. MW-1) and the weights by label, as 16-byte pairs from
    //    the even column at or below K (a pair's lower half below K is never read)
    constexpr int J0 = K & ~1;
    double *prow = c.ws.prow(), *wv = c.ws.wv();
    if (c.lane == pl) {
#pragma unroll
        for (int j = J0; j < MW; j += 2) *reinterpret_cast<double2 *>(prow + j) = make_double2(R[j], R[j + 1]);
    }
    wv[lab] = mult;
    __syncwarp(c.gm);
    // -- row update M[i, K:m] -= mult_i * M[K, K:m] (:239-245)
#pragma unroll
    for (int j = J0; j < MW; j += 2) {
        const double2 p2 = *reinterpret_cast<const double2 *>(prow + j);
        if constexpr (EXACT) {
            if (j >= K) R[j] = __dsub_rn(R[j], __dmul_rn(mult, p2.x));
            R[j + 1] = __dsub_rn(R[j + 1], __dmul_rn(mult, p2.y));
        } else {
            if (j >= K) R[j] = fma(-mult, p2.x, R[j]);
            R[j + 1] = fma(-mult, p2.y, R[j + 1]);
        }
    }
    // -- column update M[:, K] += sum_{i > K} mult_i M[:, i] (:248-255), i ascending
    constexpr int I0 = (K + 1) & ~1;
    if constexpr (EXACT) {
        double acc = R[K];
#pragma unroll
        for (int i = I0; i < MW; i += 2) {
            const double2 w2 = *reinterpret_cast<const double2 *>(wv + i);
            if (i > K) acc = __dadd_rn(acc, __dmul_rn(w2.x, R[i]));
            acc = __dadd_rn(acc, __dmul_rn(w2.y, R[i + 1]));
        }
        R[K] = acc;
    } else {
        double a0 = R[K], a1 = 0.0;
#pragma unroll
        for (int i = I0; i < MW; i += 2) {
            const double2 w2 = *reinterpret_cast<const double2 *>(wv + i);
            if (i > K) a0 = fma(w2.x, R[i], a0);
            a1 = fma(w2.y, R[i + 1], a1);
        }
        R[K] = a0 + a1;
    }
    __syncwarp(c.gm);
}

template <int K, int MW, int G, bool EXACT>
__device__ __forceinline__ void steps_real(TileCtx<MW, G, EXACT> &c)
{
    if constexpr (K <= MW - 2) {
        if (K > c.m - 2) return;
        step_real<K, MW, G, EXACT>(c);
        steps_real<K + 1, MW, G, EXACT>(c);
    }
}

// La Budde by diagonals in the reference's order and rounding (tiles of one row per lane): lane d
// holds D[r] = C[r][r - d] and forms, for order k,
//   D[k] = (C[k-1][k-d] - h_kk D[k-1]) - coef_{k-1,k} D[k-2] - ... - coef_{1,k} D[0]
// subtracting i = k-1 first (:470-490); coefficients whose D entry lies left of column 0 multiply an
// exact zero.
template <int MW, int G>
__device__ __forceinline__ void labudde_diag_exact(const double *__restrict__ cft, const double *__restrict__ hk, double *q,
                                                   int m, int n, int lane, unsigned gm)
{
    double D[MW + 1];
    D[0] = lane == 0 ? 1.0 : 0.0;
#pragma unroll
    for (int r = 1; r <= MW; ++r) D[r] = 0.0;
#pragma unroll
    for (int k = 1; k <= MW; ++k) {
        if (k > m) break;
        double up = __shfl_up_sync(gm, D[k - 1], 1, G);
        if (lane == 0) up = 0.0;
        const double *row = cft + cft_row_real(k);
        double v = __dsub_rn(up, __dmul_rn(hk[k], D[k - 1]));
#pragma unroll
        for (int i = k - 1; i >= 1; --i) v = __dsub_rn(v, __dmul_rn(row[i - 1], D[i - 1]));
        D[k] = v;
        if (k == m && lane < m && lane >= m - n) q[m - lane] = D[k];
    }
}

// One real term of mE surviving edges (m = 2 mE <= MW <= 32): build, reduce, La Budde.  Leaves
// q_1..q_min(m,n) in ws.q (the caller turns them into the term value).
template <int MW, int G, bool EXACT>
__device__ __forceinline__ void term_real_tile(const double *__restrict__ Ax, int lda, int E, int mE, int n,
                                               const TileWs<MW> &ws, int lane, unsigned gm)
{
    static_assert(MW <= 32, "one row per lane");
    static_assert(G == 32 || MW <= 16, "a group of 16 lanes holds up to 16 rows");
    const int m = 2 * mE;
    double R[MW];
    int lab = lane;
    {
        const bool live = lane < m;
        const int *eidx = ws.eidx();
        const double *kval = ws.kval();
        const int ra = live ? (lane < mE ? eidx[lane] : eidx[lane - mE] + E) : 0;
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            double v = 0.0;
            if (live && j < m) {
                const int b = j < mE ? j : j - mE;
                const int col = eidx[b] + (j < mE ? E : 0);
                v = kval[b] * __ldg(Ax + (size_t)col * lda + ra);  // M = A_S X D (:582-593)
            }
            R[j] = v;
        }
    }
    TileCtx<MW, G, EXACT> c{R, lab, ws, m, lane, gm};
    steps_real<1, MW, G, EXACT>(c);
    // The Hessenberg matrix to shared memory: the subdiagonal, the diagonal and, by column, the
    // entries above the diagonal (row label l of column j goes to order j+1's row at l).
    if (lab < m) {
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            if (j == lab - 1) ws.sub()[lab] = R[j];
            if (j == lab) ws.hk()[j + 1] = R[j];
            if (j > lab && j < m) ws.cft()[cft_row_real(j + 1) + lab] = R[j];
        }
    }
    __syncwarp(gm);
    // La Budde's coefficients h_ik * beta_ik, beta_ik = h_{k,k-1} h_{k-1,k-2} ... h_{i+1,i} multiplied
    // in that order (:476-481), one lane per order k.
    {
        const int k = lane + 1;
        if (k <= m) {
            double *row = ws.cft() + cft_row_real(k);
            double beta = 1.0;
            for (int i = k - 1; i >= 1; --i) {
                if constexpr (EXACT) {
                    beta = __dmul_rn(beta, ws.sub()[i]);
                    row[i - 1] = __dmul_rn(row[i - 1], beta);
                } else {
                    beta *= ws.sub()[i];
                    row[i - 1] *= beta;
                }
            }
        }
    }
    __syncwarp(gm);
    if constexpr (EXACT) labudde_diag_exact<MW, G>(ws.cft(), ws.hk(), ws.q(), m, n, lane, gm);
    else labudde_diag<MW, G>(ws.cft(), ws.hk(), ws.q(), m, n, lane, gm);
    __syncwarp(gm);
}

// [lambda^n] det(I - lambda H)^(-1/2) from q_1..q_min(m,n) in the reference's order and rounding
// (_inv_sqrt_det_coeff!, src/hafnian.jl:502-514): f_t = -s_t / (2t), s_t summed j = 1..min(t, m).
// One lane computes one term's series; f is that lane's scratch of n + 1 values.
__device__ __forceinline__ double series_exact(const double *q, double *f, int m, int n)
{
    f[0] = 1.0;
    for (int t = 1; t <= n; ++t) {
        double s = 0.0;
        const int jm = t < m ? t : m;
        for (int j = 1; j <= jm; ++j) s = __dadd_rn(s, __dmul_rn(__dmul_rn((double)(2 * t - j), q[j]), f[t - j]));
        f[t] = __ddiv_rn(-s, (double)(2 * t));
    }
    return f[n];
}

// ---- complex terms in the reference's arithmetic (_hessenberg_split!, src/hafnian.jl:271-335) ----
//
// The same tile with the real and imaginary parts of each row in two register arrays.  Pivot on the
// squared modulus (:277-286), multipliers ((ar xr + ai xi) / d, (ai xr - ar xi) / d) with
// d = xr^2 + xi^2 (:296-304), the row update Mr -= ur ar - ui ai, Mi -= ur ai + ui ar (:307-314) and
// the column update Mr += mr Mr_i - mi Mi_i, Mi += mr Mi_i + mi Mr_i (:317-324), every product and
// sum rounded separately; La Budde and the series use Julia's complex product
// (ar br - ai bi, ar bi + ai br).

// Layout in doubles from the group's base (complex arrays hold re, im pairs).
__host__ __device__ constexpr int ctile_off_cft() { return 256; }
__host__ __device__ constexpr int ctile_off_hk(int mw) { return 256 + 2 * cft_row_cplx(mw + 1); }
__host__ __device__ constexpr int ctile_off_sub(int mw) { return ctile_off_hk(mw) + 2 * (mw + 2); }
__host__ __device__ constexpr int ctile_off_q(int mw) { return ctile_off_sub(mw) + 2 * (mw + 2); }
__host__ __device__ constexpr int ctile_off_kval(int mw) { return ctile_off_q(mw) + 64; }
__host__ __device__ constexpr int ctile_off_eidx(int mw) { return ctile_off_kval(mw) + 32; }
__host__ __device__ constexpr int ctile_off_pre(int mw) { return ctile_off_eidx(mw) + 16; }
__host__ __device__ constexpr int ctile_off_jx(int mw) { return ctile_off_pre(mw) + 32; }
__host__ __device__ constexpr int ctile_off_mx(int mw) { return ctile_off_jx(mw) + 32; }
__host__ __device__ constexpr int ctile_off_qbuf(int mw) { return ctile_off_mx(mw) + 16; }

__host__ __device__ inline size_t ctile_ws_doubles(int nmax, int mhi)
{
    return ((size_t)ctile_off_qbuf(mhi) + 64 * (size_t)(nmax + 1) + 1) & ~(size_t)1;
}

template <int MW>
struct CTileWs {
    double *base;
    __device__ double *prr() const { return base; }
    __device__ double *pri() const { return base + 64; }
    __device__ double *wvr() const { return base + 128; }
    __device__ double *wvi() const { return base + 192; }
    __device__ cd *cft() const { return (cd *)(base + ctile_off_cft()); }
    __device__ cd *hk() const { return (cd *)(base + ctile_off_hk(MW)); }
    __device__ cd *sub() const { return (cd *)(base + ctile_off_sub(MW)); }
    __device__ cd *q() const { return (cd *)(base + ctile_off_q(MW)); }
    __device__ double *kval() const { return base + ctile_off_kval(MW); }
    __device__ int *eidx() const { return (int *)(base + ctile_off_eidx(MW)); }
    __device__ double *pre() const { return base + ctile_off_pre(MW); }
    __device__ long long *jx() const { return (long long *)(base + ctile_off_jx(MW)); }
    __device__ int *mx() const { return (int *)(base + ctile_off_mx(MW)); }
    __device__ cd *qbuf() const { return (cd *)(base + ctile_off_qbuf(MW)); }
};

template <int K, int LO, int HI, int MW>
__device__ __forceinline__ void swap_cols2(double (&A)[MW], double (&Bv)[MW], int p)
{
    if constexpr (HI - LO == 1) {
        const double t = A[K];
        A[K] = A[LO];
        A[LO] = t;
        const double u = Bv[K];
        Bv[K] = Bv[LO];
        Bv[LO] = u;
    } else {
        constexpr int MID = (LO + HI) / 2;
        if (p < MID) swap_cols2<K, LO, MID, MW>(A, Bv, p);
        else swap_cols2<K, MID, HI, MW>(A, Bv, p);
    }
}

template <int MW, int G>
struct CTileCtx {
    double (&Rr)[MW];
    double (&Ri)[MW];
    int &lab;
    const CTileWs<MW> &ws;
    int m, lane;
    unsigned gm;
};

// Step K of the split reduction (pivot row K, pivot column K - 1; 0-based).
template <int K, int MW, int G>
__device__ __forceinline__ void step_cplx(CTileCtx<MW, G> &c)
{
    double (&Rr)[MW] = c.Rr;
    double (&Ri)[MW] = c.Ri;
    int &lab = c.lab;
    const int m = c.m;
    const bool cand = lab >= K && lab < m;
    // -- pivot: the first row of largest squared modulus (:277-286); NaN as in the real form
    const double a = __dadd_rn(__dmul_rn(Rr[K - 1], Rr[K - 1]), __dmul_rn(Ri[K - 1], Ri[K - 1]));
    int plab, pl;
    {
        unsigned long long key = cand ? abs_key(a) : 0ull;
        if (lab == K && a != a) key = ~0ull;  // row K's NaN keeps row K, as in the real form
        const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
        const unsigned mhi = __reduce_max_sync(c.gm, hi);
        const unsigned mlo = __reduce_max_sync(c.gm, hi == mhi ? lo : 0u);
        const bool win = key != 0ull && hi == mhi && lo == mlo;
        plab = (int)__reduce_min_sync(c.gm, win ? (unsigned)lab : 0x7fffffffu);  // lowest label among the maxima
        if (plab == 0x7fffffff) plab = K;
    }
    pl = __ffs((int)__ballot_sync(c.gm, lab == plab)) - 1;
    if (G < 32) pl &= G - 1;
    const double xr = __shfl_sync(c.gm, Rr[K - 1], pl, G), xi = __shfl_sync(c.gm, Ri[K - 1], pl, G);
    // -- swap rows (relabel) and columns (move)
    if (lab == K) lab = plab;
    else if (lab == plab) lab = K;
    if (plab != K) swap_cols2<K, K + 1, MW, MW>(Rr, Ri, plab);
    const double d = __dadd_rn(__dmul_rn(xr, xr), __dmul_rn(xi, xi));
    if (d == 0.0) return;  // (:293)
    // -- multipliers (:296-304)
    double mr = 0.0, mi = 0.0;
    {
        const bool d_ok = div_scale_ok(d);
        const double y = d_ok ? __drcp_rn(d) : 0.0;
        if (lab > K && lab < m) {
            const double ar = Rr[K - 1], ai = Ri[K - 1];
            mr = div_rn_shared(__dadd_rn(__dmul_rn(ar, xr), __dmul_rn(ai, xi)), d, y, d_ok);
            mi = div_rn_shared(__dsub_rn(__dmul_rn(ai, xr), __dmul_rn(ar, xi)), d, y, d_ok);
        }
    }
    constexpr int J0 = K & ~1;
    double *prr = c.ws.prr(), *pri = c.ws.pri(), *wvr = c.ws.wvr(), *wvi = c.ws.wvi();
    if (c.lane == pl) {
#pragma unroll
        for (int j = J0; j < MW; j += 2) {
            *reinterpret_cast<double2 *>(prr + j) = make_double2(Rr[j], Rr[j + 1]);
            *reinterpret_cast<double2 *>(pri + j) = make_double2(Ri[j], Ri[j + 1]);
        }
    }
    wvr[lab] = mr;
    wvi[lab] = mi;
    __syncwarp(c.gm);
    // -- row update (:307-314)
#pragma unroll
    for (int j = J0; j < MW; j += 2) {
        const double2 ar2 = *reinterpret_cast<const double2 *>(prr + j);
        const double2 ai2 = *reinterpret_cast<const double2 *>(pri + j);
        if (j >= K) {
            Rr[j] = __dsub_rn(Rr[j], __dsub_rn(__dmul_rn(mr, ar2.x), __dmul_rn(mi, ai2.x)));
            Ri[j] = __dsub_rn(Ri[j], __dadd_rn(__dmul_rn(mr, ai2.x), __dmul_rn(mi, ar2.x)));
        }
        Rr[j + 1] = __dsub_rn(Rr[j + 1], __dsub_rn(__dmul_rn(mr, ar2.y), __dmul_rn(mi, ai2.y)));
        Ri[j + 1] = __dsub_rn(Ri[j + 1], __dadd_rn(__dmul_rn(mr, ai2.y), __dmul_rn(mi, ar2.y)));
    }
    // -- column update (:317-324), i ascending
    constexpr int I0 = (K + 1) & ~1;
    double accr = Rr[K], acci = Ri[K];
#pragma unroll
    for (int i = I0; i < MW; i += 2) {
        const double2 w_r = *reinterpret_cast<const double2 *>(wvr + i);
        const double2 w_i = *reinterpret_cast<const double2 *>(wvi + i);
        if (i > K) {
            accr = __dadd_rn(accr, __dsub_rn(__dmul_rn(w_r.x, Rr[i]), __dmul_rn(w_i.x, Ri[i])));
            acci = __dadd_rn(acci, __dadd_rn(__dmul_rn(w_r.x, Ri[i]), __dmul_rn(w_i.x, Rr[i])));
        }
        accr = __dadd_rn(accr, __dsub_rn(__dmul_rn(w_r.y, Rr[i + 1]), __dmul_rn(w_i.y, Ri[i + 1])));
        acci = __dadd_rn(acci, __dadd_rn(__dmul_rn(w_r.y, Ri[i + 1]), __dmul_rn(w_i.y, Rr[i + 1])));
    }
    Rr[K] = accr;
    Ri[K] = acci;
    __syncwarp(c.gm);
}

template <int K, int MW, int G>
__device__ __forceinline__ void steps_cplx(CTileCtx<MW, G> &c)
{
    if constexpr (K <= MW - 2) {
        if (K > c.m - 2) return;
        step_cplx<K, MW, G>(c);
        steps_cplx<K + 1, MW, G>(c);
    }
}

__device__ __forceinline__ cd c_sub_rn(cd a, cd b) { return cd{__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)}; }

// La Budde by diagonals, complex, in the reference's order and rounding (see labudde_diag_exact).
template <int MW, int G>
__device__ __forceinline__ void labudde_diag_cplx_exact(const cd *__restrict__ cft, const cd *__restrict__ hk, cd *q, int m,
                                                        int n, int lane, unsigned gm)
{
    cd D[MW + 1];
    D[0] = cd{lane == 0 ? 1.0 : 0.0, 0.0};
#pragma unroll
    for (int r = 1; r <= MW; ++r) D[r] = cd{0.0, 0.0};
#pragma unroll
    for (int k = 1; k <= MW; ++k) {
        if (k > m) break;
        cd up{__shfl_up_sync(gm, D[k - 1].re, 1, G), __shfl_up_sync(gm, D[k - 1].im, 1, G)};
        if (lane == 0) up = cd{0.0, 0.0};
        const cd *row = cft + cft_row_cplx(k);
        cd v = c_sub_rn(up, x_cmul(hk[k], D[k - 1]));
#pragma unroll
        for (int i = k - 1; i >= 1; --i) v = c_sub_rn(v, x_cmul(row[i - 1], D[i - 1]));
        D[k] = v;
        if (k == m && lane < m && lane >= m - n) q[m - lane] = D[k];
    }
}

// One complex term (m = 2 mE <= MW <= 32) in the reference's arithmetic: leaves q_1..q_min(m,n).
template <int MW, int G>
__device__ __forceinline__ void term_cplx_tile(const cd *__restrict__ Ax, int lda, int E, int mE, int n,
                                               const CTileWs<MW> &ws, int lane, unsigned gm)
{
    static_assert(MW <= 32, "one row per lane");
    static_assert(G == 32 || MW <= 16, "a group of 16 lanes holds up to 16 rows");
    const int m = 2 * mE;
    double Rr[MW], Ri[MW];
    int lab = lane;
    {
        const int *eidx = ws.eidx();
        const double *kval = ws.kval();
        const bool live = lane < m;
        const int ra = live ? (lane < mE ? eidx[lane] : eidx[lane - mE] + E) : 0;
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            double vr = 0.0, vi = 0.0;
            if (live && j < m) {
                const int b = j < mE ? j : j - mE;
                const int col = eidx[b] + (j < mE ? E : 0);
                const double2 z = __ldg(reinterpret_cast<const double2 *>(Ax + (size_t)col * lda + ra));
                vr = __dmul_rn(kval[b], z.x);  // M = A_S X D (:582-593)
                vi = __dmul_rn(kval[b], z.y);
            }
            Rr[j] = vr;
            Ri[j] = vi;
        }
    }
    CTileCtx<MW, G> c{Rr, Ri, lab, ws, m, lane, gm};
    steps_cplx<1, MW, G>(c);
    if (lab < m) {
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            const cd v{Rr[j], Ri[j]};
            if (j == lab - 1) ws.sub()[lab] = v;
            if (j == lab) ws.hk()[j + 1] = v;
            if (j > lab && j < m) ws.cft()[cft_row_cplx(j + 1) + lab] = v;
        }
    }
    __syncwarp(gm);
    {
        const int k = lane + 1;
        if (k <= m) {
            cd *row = ws.cft() + cft_row_cplx(k);
            cd beta{1.0, 0.0};
            for (int i = k - 1; i >= 1; --i) {
                beta = x_cmul(beta, ws.sub()[i]);
                row[i - 1] = x_cmul(row[i - 1], beta);
            }
        }
    }
    __syncwarp(gm);
    labudde_diag_cplx_exact<MW, G>(ws.cft(), ws.hk(), ws.q(), m, n, lane, gm);
    __syncwarp(gm);
}

// _inv_sqrt_det_coeff! for a complex term, in the reference's order and rounding, on one lane.
__device__ __forceinline__ cd series_cplx_exact(const cd *q, cd *f, int m, int n)
{
    f[0] = cd{1.0, 0.0};
    for (int t = 1; t <= n; ++t) {
        cd s{0.0, 0.0};
        const int jm = t < m ? t : m;
        for (int j = 1; j <= jm; ++j) {
            const double wt = (double)(2 * t - j);
            const cd wq{__dmul_rn(wt, q[j].re), __dmul_rn(wt, q[j].im)};
            const cd pr = x_cmul(wq, f[t - j]);
            s.re = __dadd_rn(s.re, pr.re);
            s.im = __dadd_rn(s.im, pr.im);
        }
        const double d2 = (double)(2 * t);
        f[t] = cd{__ddiv_rn(-s.re, d2), __ddiv_rn(-s.im, d2)};
    }
    return f[n];
}

}  // namespace egg
