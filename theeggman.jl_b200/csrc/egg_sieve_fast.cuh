// egg_sieve_fast.cuh -- register-resident sieve terms (the fast path of the device sieve).
//
// One warp evaluates one term at a time, as in the exact kernel, but the m x m matrix
// M = A_S X D (src/hafnian.jl:583-593) lives in registers: lane l owns row l (and row l + 32 for
// real terms with m > 32), one register per physical column slot, so every loop over columns has
// a compile-time trip count.  The Gaussian similarity reduction to Hessenberg form (EISPACK
// elmhes, src/hafnian.jl:210-335) is done without moving data:
//
//   * Pivoting relabels.  Each row carries its logical label; swapping logical rows/columns p and k
//     (a similarity, so both) swaps two labels.  Physical column j always carries the label of
//     physical row j, so a lane knows every column's label from the rows' labels.
//   * The pivot search is one redux.sync.max over a 32-bit key: the high 24 bits of |pivot|'s
//     magnitude (sign-free double bits) above the candidate's physical slot.  Entries within 2^-13
//     of each other may pick either; any near-maximal pivot keeps the multipliers bounded by ~1.
//   * The current pivot column (logical s-1) is kept in a scalar per row, `pc`.  The row update
//     M[i, :] -= mult_i * M[piv, :] runs over all slots with mult_i = 0 for rows that are not below
//     the pivot (so they are left bit-for-bit unchanged); slots of finished columns hold values that
//     are never read again except multiplied by zero.
//   * The column update M[:, s] += sum_i mult_i M[:, i] is a dot product of each row with a weight
//     vector that is mult_i on the live rows' slots and exactly 1 on the pivot slot, which yields
//     the updated column s directly -- the next step's `pc` -- with no dynamic register index.
//
// La Budde's recurrence (src/hafnian.jl:454-492): each finished Hessenberg column stores its
// order-k coefficients; after the reduction lane d computes diagonal d of the coefficient table in
// registers (labudde_diag), and diagonal d + 32 too for tiles of two rows per lane
// (labudde_diag2).  The [lambda^n] series coefficient
// (src/hafnian.jl:502-514) is accumulated push-style: once f_s is known every lane t > s adds its
// (t+s) q_{t-s} f_s, so each order costs one multiply-add per lane and one broadcast.  All arithmetic
// is FP64 with fused multiply-adds; terms are accumulated in double-double per warp.
//
// Terms whose size exceeds the register tiles (complex m > 32, real m > 48) or whose order n
// exceeds 31 are left to the exact kernel, which sums them into separate partials.
#pragma once
#include <atomic>

#include "egg_sieve.cuh"

namespace egg {

static constexpr unsigned FULL = 0xffffffffu;

// Tables in constant memory, computed at compile time and placed in the module image, so that
// every device that loads the library holds them from the start (nothing to upload).
struct FastTables {
    double neg_inv_2t[64];   // -1 / (2t) for t = 1..63, correctly rounded (entry 0 unused)
    uint32_t binom[33 * 33]; // C(x, i) for x, i <= 32 at [x * 33 + i] (C(32, 16) < 2^32)
};
static constexpr FastTables make_fast_tables()
{
    FastTables t{};
    for (int i = 1; i < 64; ++i) t.neg_inv_2t[i] = -1.0 / (2.0 * i);
    for (int x = 0; x <= 32; ++x)
        for (int i = 0; i <= 32; ++i)
            t.binom[x * 33 + i] = i == 0 ? 1u : (x == 0 ? 0u : t.binom[(x - 1) * 33 + i - 1] + t.binom[(x - 1) * 33 + i]);
    return t;
}
static __constant__ const FastTables c_fast = make_fast_tables();
static_assert(make_fast_tables().binom[32 * 33 + 16] == 601080390u, "C(32, 16)");

// The k-subset of [0, E) with colex rank R: x_i is the largest x with C(x, i) <= what is left.
__device__ __forceinline__ uint32_t subset_unrank(int E, int k, uint32_t R)
{
    uint32_t S = 0;
    int x = E - 1;
    for (int i = k; i >= 1; --i) {
        while (c_fast.binom[x * 33 + i] > R) --x;
        S |= 1u << x;
        R -= c_fast.binom[x * 33 + i];
        --x;
    }
    return S;
}

// The colex successor of a subset mask (the next larger integer with the same popcount).
__device__ __forceinline__ uint32_t subset_next(uint32_t v)
{
    const uint32_t t = v | (v - 1);
    return (t + 1) | (((~t & (0u - ~t)) - 1) >> (__ffs((int)v)));
}

// 1/x by Newton-Raphson iteration from the single-precision reciprocal: each step
// y <- y + y(1 - xy) doubles the number of correct bits (24 -> 48 -> full).  Outside the range
// where the float seed is representable, fall back to IEEE division.
__device__ __forceinline__ double recip(double x)
{
    float xf = __double2float_rn(x);
    float ax = fabsf(xf);
    if (!(ax > 1e-36f && ax < 1e36f)) return 1.0 / x;
    double y = (double)__frcp_rn(xf);
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// Candidate key: magnitude bits above bit 7, then a set bit 6 (so every candidate beats the
// non-candidates' 0), then 63 - slot (ties go to the lowest slot).  a >= 0; NaN never wins.
__device__ __forceinline__ unsigned pivot_key(double a, int slot)
{
    unsigned hi = (unsigned)__double2hiint(a);
    if (a != a) hi = 0;
    return (hi & ~127u) | 64u | (unsigned)(63 - slot);
}

// Per-warp shared scratch of the fast path.
struct FastWs {
    double *prow;  // pivot row, by physical slot [64]
    double *wv;    // column-update weights, by physical slot [64]
    double *cft;   // La Budde coefficients of every order k, a triangle (see labudde_diag)
    double *hk;    // Hessenberg diagonal h_kk by k [mhi + 1]
    double *q;     // det(I - lambda H) coefficients q_j by j [32]
    double *kval;  // multiplicities of the surviving edges after the Glynn substitution [32]
    int *eidx;     // surviving edges, compacted [32]
};

// Start of order k's row in the coefficient triangle (k = 1..mhi, k - 1 coefficients each).  Real
// rows are padded to an even length so that each starts on a 16-byte boundary.
__host__ __device__ constexpr int cft_row_real(int k) { return (k - 1) * (k - 2) / 2 + (k - 1) / 2; }
__host__ __device__ constexpr int cft_row_cplx(int k) { return (k - 1) * (k - 2) / 2; }

__host__ __device__ inline size_t fast_body_doubles(int cplx, int mhi)
{
    const size_t v = cplx ? 2 : 1;  // doubles per value
    const size_t tri = cplx ? 2 * (size_t)cft_row_cplx(mhi + 1) : (size_t)cft_row_real(mhi + 1);
    return tri + v * (size_t)((mhi + 2) & ~1) + v * 32;
}

__host__ __device__ inline size_t fast_ws_doubles(int nmax, int cplx, int mhi)
{
    size_t d = 64 * 2 + fast_body_doubles(cplx, mhi) + 32 /*kval*/ + 16 /*eidx*/;
    return (d + 1) & ~(size_t)1;  // keep every warp's region 16-byte aligned
}

__device__ inline FastWs fast_carve(double *base, int nmax, int cplx, int mhi)
{
    const size_t v = cplx ? 2 : 1;
    FastWs w;
    double *p = base;
    w.prow = p; p += 64;
    w.wv = p; p += 64;
    w.cft = p;
    w.hk = w.cft + (cplx ? 2 * (size_t)cft_row_cplx(mhi + 1) : (size_t)cft_row_real(mhi + 1));
    w.q = w.hk + v * (size_t)((mhi + 2) & ~1);
    p += fast_body_doubles(cplx, mhi);
    w.kval = p; p += 32;
    w.eidx = (int *)p;
    return w;
}

// ---- La Budde by diagonals, in registers (tiles of one row per lane) ------------------------------
// La Budde's recurrence over the leading minors (src/hafnian.jl:454-492), with C[k][t] the
// coefficient of lambda^t in det(I - lambda H_k), run after the Hessenberg reduction from the
// coefficients it stored: for order k, cft[cft_row(k) + i - 1] = h_{i,k} prod_{l=i+1..k} h_{l,l-1}
// (i = 1..k-1) and hk[k] = h_{k,k}.  Lane d owns diagonal d of the table, D[r] = C[r][r - d], zero
// left of column 0:
//   C[k][t] = C[k-1][t] - h_kk C[k-1][t-1] - sum_{i=1}^{k-1} cf_k[i] C[i-1][t-1-(k-i)],
// where C[k-1][t] lies on diagonal d - 1 (one shuffle) and every other entry on the lane's own
// diagonal, so with k unrolled every index is a compile-time register.  Columns beyond n are
// computed too but never read by the columns <= n.  The depth sum runs over all i: entries left of
// column 0 are exact zeros.  Diagonal 32 (only C[32][0] = 1, never read) has no lane.
// q_j = C[m][j] (j = 1..min(m, n)) goes to q[j] for the series.
template <int MW, int G>
__device__ __forceinline__ void labudde_diag(const double *__restrict__ cft, const double *__restrict__ hk, double *q,
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
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int i = 1; i < k; i += 2) {
            const double2 c2 = *reinterpret_cast<const double2 *>(row + (i - 1));
            s0 = fma(c2.x, D[i - 1], s0);
            if (i + 1 < k) s1 = fma(c2.y, D[i], s1);
        }
        D[k] = fma(-hk[k], D[k - 1], up) - (s0 + s1);
        if (k == m && lane < m && lane >= m - n) q[m - lane] = D[k];
    }
}

// Tiles of two rows per lane (33 <= m <= 48): lane l owns diagonals l and l + 32.  The upper one
// has entries only in rows r >= 32 (at Dh[r - 32]); its entry above-right lies on diagonal l + 31,
// lane l - 1's upper diagonal, or lane 31's lower one for l = 0.
template <int MW>
__device__ __forceinline__ void labudde_diag2(const double *__restrict__ cft, const double *__restrict__ hk, double *q,
                                              int m, int n, int lane)
{
    static_assert(MW > 32 && MW <= 64, "two diagonals per lane");
    double Dl[MW + 1], Dh[MW - 31];
    Dl[0] = lane == 0 ? 1.0 : 0.0;
#pragma unroll
    for (int r = 1; r <= MW; ++r) Dl[r] = 0.0;
#pragma unroll
    for (int r = 0; r < MW - 31; ++r) Dh[r] = 0.0;
#pragma unroll
    for (int k = 1; k <= MW; ++k) {
        if (k > m) break;
        const double h = hk[k];
        const double *row = cft + cft_row_real(k);
        double up = __shfl_up_sync(FULL, Dl[k - 1], 1);
        if (lane == 0) up = 0.0;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int i = 1; i < k; i += 2) {
            const double2 c2 = *reinterpret_cast<const double2 *>(row + (i - 1));
            s0 = fma(c2.x, Dl[i - 1], s0);
            if (i + 1 < k) s1 = fma(c2.y, Dl[i], s1);
        }
        if (k >= 32) {
            // Upper diagonal, row k (k - 1 >= 31: Dh[k - 33] is row k - 1 when k >= 33).
            const double prev = k >= 33 ? Dh[k - 33] : 0.0;
            double uh = __shfl_up_sync(FULL, prev, 1);
            const double from31 = __shfl_sync(FULL, Dl[k - 1], 31);
            if (lane == 0) uh = from31;
            double t = 0.0;
#pragma unroll
            for (int i = 33; i < k; ++i) t = fma(row[i - 1], Dh[i - 33], t);  // rows i - 1 >= 32
            Dh[k - 32] = fma(-h, prev, uh) - t;
        }
        Dl[k] = fma(-h, Dl[k - 1], up) - (s0 + s1);
        if (k == m) {
            const int jl = m - lane, jh = m - lane - 32;
            if (jl >= 1 && jl <= n) q[jl] = Dl[k];
            if (jh >= 1 && jh <= n) q[jh] = Dh[k - 32];
        }
    }
}

template <int MW, int G>
__device__ __forceinline__ void labudde_diag_c(const cd *__restrict__ cft, const cd *__restrict__ hk, cd *q, int m, int n,
                                               int lane, unsigned gm)
{
    double Dr[MW + 1], Di[MW + 1];
    Dr[0] = lane == 0 ? 1.0 : 0.0;
    Di[0] = 0.0;
#pragma unroll
    for (int r = 1; r <= MW; ++r) {
        Dr[r] = 0.0;
        Di[r] = 0.0;
    }
#pragma unroll
    for (int k = 1; k <= MW; ++k) {
        if (k > m) break;
        double ur = __shfl_up_sync(gm, Dr[k - 1], 1, G), ui = __shfl_up_sync(gm, Di[k - 1], 1, G);
        if (lane == 0) {
            ur = 0.0;
            ui = 0.0;
        }
        const cd h = hk[k];
        const double vr = fma(-h.re, Dr[k - 1], fma(h.im, Di[k - 1], ur));
        const double vi = fma(-h.re, Di[k - 1], fma(-h.im, Dr[k - 1], ui));
        const cd *row = cft + cft_row_cplx(k);
        double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
#pragma unroll
        for (int i = 1; i < k; ++i) {
            const cd c = row[i - 1];
            if (i & 1) {
                sr0 = fma(c.re, Dr[i - 1], fma(-c.im, Di[i - 1], sr0));
                si0 = fma(c.re, Di[i - 1], fma(c.im, Dr[i - 1], si0));
            } else {
                sr1 = fma(c.re, Dr[i - 1], fma(-c.im, Di[i - 1], sr1));
                si1 = fma(c.re, Di[i - 1], fma(c.im, Dr[i - 1], si1));
            }
        }
        Dr[k] = vr - (sr0 + sr1);
        Di[k] = vi - (si0 + si1);
        if (k == m && lane < m && lane >= m - n) q[m - lane] = cd{Dr[k], Di[k]};
    }
}

// [lambda^n] det(I - lambda H)^(-1/2) from q_1..q_min(m,n), push-style: the lane of coefficient t
// accumulates S_t = sum_j (2t-j) q_j f_{t-j} as the f's become known; f_t = -S_t / (2t).  In a
// group of G lanes, lane l holds t = l + G c for c < 32 / G (n <= 31).  All lanes return f_n.
template <int G>
__device__ __forceinline__ double series_q(const double *q, int m, int n, int lane, unsigned gm)
{
    constexpr int NC = 32 / G;
    double S[NC], fs = 1.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) S[c] = 0.0;
    for (int s = 0; s < n; ++s) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int t = lane + G * c, j = t - s;
            if (j >= 1 && j <= m && t <= n) S[c] = fma((double)(t + s) * q[j], fs, S[c]);
        }
        const int t1 = s + 1;
        const double own = (NC > 1 && t1 >= G) ? S[NC - 1] : S[0];
        fs = __shfl_sync(gm, own, t1 & (G - 1), G) * c_fast.neg_inv_2t[t1];
    }
    return fs;
}

template <int G>
__device__ __forceinline__ cd series_q_c(const cd *q, int m, int n, int lane, unsigned gm)
{
    constexpr int NC = 32 / G;
    double Sr[NC], Si[NC], fr = 1.0, fi = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        Sr[c] = 0.0;
        Si[c] = 0.0;
    }
    for (int s = 0; s < n; ++s) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int t = lane + G * c, j = t - s;
            if (j >= 1 && j <= m && t <= n) {
                const double w = (double)(t + s);
                const cd qj = q[j];
                const double ar = w * qj.re, ai = w * qj.im;
                Sr[c] = fma(ar, fr, fma(-ai, fi, Sr[c]));
                Si[c] = fma(ar, fi, fma(ai, fr, Si[c]));
            }
        }
        const int t1 = s + 1;
        const double c1 = c_fast.neg_inv_2t[t1];
        const double ownr = (NC > 1 && t1 >= G) ? Sr[NC - 1] : Sr[0];
        const double owni = (NC > 1 && t1 >= G) ? Si[NC - 1] : Si[0];
        fr = __shfl_sync(gm, ownr, t1 & (G - 1), G) * c1;
        fi = __shfl_sync(gm, owni, t1 & (G - 1), G) * c1;
    }
    return cd{fr, fi};
}

// ---- one real term, m <= 32 * RPL, register tile of MW columns ----------------------------------
template <int MW, int RPL, int G>
__device__ __forceinline__ double term_real(const double *__restrict__ Ax, int lda, int E, int mE, int n,
                                            const FastWs &ws, int lane, unsigned gm)
{
    static_assert(G == 32 || (G == 16 && RPL == 1 && MW <= 16), "a group of 16 lanes holds up to 16 rows");
    const int m = 2 * mE;
    double *prow = ws.prow, *wv = ws.wv;
    double R[RPL][MW];
    int lab[RPL];
    double pc[RPL], bet[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
        const int r = lane + 32 * q;
        lab[q] = r;
        bet[q] = 0.0;
        const bool live = r < m;
        const int ra = live ? (r < mE ? ws.eidx[r] : ws.eidx[r - mE] + E) : 0;
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            double v = 0.0;
            if (live && j < m) {
                const int b = j < mE ? j : j - mE;
                const int col = ws.eidx[b] + (j < mE ? E : 0);
                v = ws.kval[b] * __ldg(Ax + (size_t)col * lda + ra);
            }
            R[q][j] = v;
        }
        pc[q] = R[q][0];
    }
    double xprev = 0.0;  // subdiagonal entry h_{s,s-1} of the previous step
    for (int s = 1; s <= m - 2; ++s) {
        // -- pivot among rows with s <= label < m
        unsigned key = 0;
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lab[q] >= s && lab[q] < m) {
                const unsigned k2 = pivot_key(fabs(pc[q]), lane + 32 * q);
                key = k2 > key ? k2 : key;
            }
        const unsigned best = __reduce_max_sync(gm, key);
        const int pslot = 63 - (int)(best & 63u);
        const int plane = pslot & 31, pq = pslot >> 5;
        const double pcp = (RPL > 1 && pq == 1) ? pc[RPL - 1] : pc[0];
        const int labp = (RPL > 1 && pq == 1) ? lab[RPL - 1] : lab[0];
        const double x = __shfl_sync(gm, pcp, plane, G);
        const int plab = __shfl_sync(gm, labp, plane, G);
        // -- column s-1 is final for rows with label <= s-1 plus the pivot: store La Budde's order
        //    k = s coefficients for labudde_diag, which runs once the reduction is done
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            if (lab[q] <= s - 3) bet[q] *= xprev;
            else if (lab[q] == s - 2) bet[q] = xprev;
            if (lab[q] <= s - 2) ws.cft[cft_row_real(s) + lab[q]] = pc[q] * bet[q];
            if (lab[q] == s - 1) ws.hk[s] = pc[q];
        }
        // -- relabel (similarity swap of logical s and plab)
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            if (lab[q] == s) lab[q] = plab;
            else if (lab[q] == plab) lab[q] = s;
        }
        xprev = x;
        if (x == 0.0) {
            // Nothing to eliminate (:231-232): the next pivot column is the physical slot of label s.
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                double v = 0.0;
#pragma unroll
                for (int j = 0; j < MW; ++j)
                    if (j == pslot) v = R[q][j];
                pc[q] = v;
            }
            __syncwarp(gm);
            continue;
        }
        const double rx = recip(x);
        double mult[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) mult[q] = (lab[q] > s && lab[q] < m) ? pc[q] * rx : 0.0;
        if (lane == plane) {
#pragma unroll
            for (int j = 0; j < MW; j += 2)
                *reinterpret_cast<double2 *>(prow + j) =
                    (RPL > 1 && pq == 1) ? make_double2(R[RPL - 1][j], R[RPL - 1][j + 1]) : make_double2(R[0][j], R[0][j + 1]);
        }
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int r = lane + 32 * q;
            if (r < MW) wv[r] = r == pslot ? 1.0 : mult[q];
        }
        __syncwarp(gm);
        // -- row update: M[i, :] -= mult_i * M[piv, :]
#pragma unroll
        for (int j = 0; j < MW; j += 2) {
            const double2 p2 = *reinterpret_cast<const double2 *>(prow + j);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                R[q][j] = fma(-mult[q], p2.x, R[q][j]);
                R[q][j + 1] = fma(-mult[q], p2.y, R[q][j + 1]);
            }
        }
        // -- column update: pc <- M[:, piv] + sum_i mult_i M[:, i]
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int j = 0; j < MW; j += 2) {
                const double2 w0 = *reinterpret_cast<const double2 *>(wv + j);
                if ((j & 2) == 0) {
                    a0 = fma(w0.x, R[q][j], a0);
                    a1 = fma(w0.y, R[q][j + 1], a1);
                } else {
                    a2 = fma(w0.x, R[q][j], a2);
                    a3 = fma(w0.y, R[q][j + 1], a3);
                }
            }
            pc[q] = (a0 + a1) + (a2 + a3);
        }
        __syncwarp(gm);
    }
    // Last two columns: m-2 is `pc`, m-1 is the physical slot carrying label m-1.  Feed La Budde
    // steps k = m-1 and k = m (for m == 2 the loop above did not run and k = 1, 2 remain).
    int lastslot;
    {
        int mine = -1;
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lab[q] == m - 1) mine = lane + 32 * q;
        lastslot = (int)__reduce_max_sync(gm, (unsigned)(mine + 1)) - 1;
    }
    double colm1[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
        double v = 0.0;
#pragma unroll
        for (int j = 0; j < MW; ++j)
            if (j == lastslot) v = R[q][j];
        colm1[q] = v;
    }
    for (int k = (m >= 3 ? m - 1 : 1); k <= m; ++k) {
        const bool last = k == m;
        // h_{k,k-1}: for k = m-1 the last pivot value; for k = m the entry of the row labelled m-1
        // in column m-2, i.e. that row's pc.
        double sub = xprev;
        if (last && k >= 2) {
            const double cand = (RPL > 1 && (lastslot >> 5) == 1) ? pc[RPL - 1] : pc[0];
            sub = __shfl_sync(gm, cand, lastslot & 31, G);
        }
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const double colv = last ? colm1[q] : pc[q];
            if (k >= 2) {
                if (lab[q] <= k - 3) bet[q] *= sub;
                else if (lab[q] == k - 2) bet[q] = sub;
                if (lab[q] <= k - 2) ws.cft[cft_row_real(k) + lab[q]] = colv * bet[q];
            }
            if (lab[q] == k - 1) ws.hk[k] = colv;
        }
    }
    __syncwarp(gm);
    if constexpr (RPL == 1) labudde_diag<MW, G>(ws.cft, ws.hk, ws.q, m, n, lane, gm);
    else labudde_diag2<MW>(ws.cft, ws.hk, ws.q, m, n, lane);
    __syncwarp(gm);
    return series_q<G>(ws.q, m, n, lane, gm);
}

// ---- one complex term, m <= 32 --------------------------------------------------------------------
template <int MW, int G>
__device__ __forceinline__ cd term_cplx(const cd *__restrict__ Ax, int lda, int E, int mE, int n, const FastWs &ws,
                                        int lane, unsigned gm)
{
    static_assert(G == 32 || (G == 16 && MW <= 16), "a group of 16 lanes holds up to 16 rows");
    const int m = 2 * mE;
    double Rr[MW], Ri[MW];
    int lab = lane;
    const bool live = lane < m;
    {
        const int ra = live ? (lane < mE ? ws.eidx[lane] : ws.eidx[lane - mE] + E) : 0;
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            double vr = 0.0, vi = 0.0;
            if (live && j < m) {
                const int b = j < mE ? j : j - mE;
                const int col = ws.eidx[b] + (j < mE ? E : 0);
                const double2 z = __ldg(reinterpret_cast<const double2 *>(Ax + (size_t)col * lda + ra));
                const double kb = ws.kval[b];
                vr = kb * z.x;
                vi = kb * z.y;
            }
            Rr[j] = vr;
            Ri[j] = vi;
        }
    }
    double pcr = Rr[0], pci = Ri[0];
    cd bet{0.0, 0.0};
    cd *cft = (cd *)ws.cft, *hk = (cd *)ws.hk;
    double *prr = ws.prow, *pri = ws.prow + 32, *wvr = ws.wv, *wvi = ws.wv + 32;
    cd xprev{0.0, 0.0};
    // Store La Budde's order-k coefficients for labudde_diag_c, which runs once the reduction is done.
    auto feed = [&](int k, double colr, double coli, cd sub) {
        if (k >= 2) {
            if (lab <= k - 3) bet = cd{fma(bet.re, sub.re, -bet.im * sub.im), fma(bet.re, sub.im, bet.im * sub.re)};
            else if (lab == k - 2) bet = sub;
            if (lab <= k - 2)
                cft[cft_row_cplx(k) + lab] = cd{fma(colr, bet.re, -coli * bet.im), fma(colr, bet.im, coli * bet.re)};
        }
        if (lab == k - 1) hk[k] = cd{colr, coli};
    };
    for (int s = 1; s <= m - 2; ++s) {
        unsigned key = 0;
        if (lab >= s && lab < m) key = pivot_key(fma(pcr, pcr, pci * pci), lane);
        const unsigned best = __reduce_max_sync(gm, key);
        const int plane = 63 - (int)(best & 63u);
        const double xr = __shfl_sync(gm, pcr, plane, G), xi = __shfl_sync(gm, pci, plane, G);
        const int plab = __shfl_sync(gm, lab, plane, G);
        feed(s, pcr, pci, xprev);
        if (lab == s) lab = plab;
        else if (lab == plab) lab = s;
        xprev = cd{xr, xi};
        const double d = fma(xr, xr, xi * xi);
        if (d == 0.0) {
            double vr = 0.0, vi = 0.0;
#pragma unroll
            for (int j = 0; j < MW; ++j)
                if (j == plane) {
                    vr = Rr[j];
                    vi = Ri[j];
                }
            pcr = vr;
            pci = vi;
            continue;
        }
        const double rd = recip(d);
        double mr = 0.0, mi = 0.0;
        if (lab > s && lab < m) {
            mr = fma(pcr, xr, pci * xi) * rd;
            mi = fma(pci, xr, -pcr * xi) * rd;
        }
        if (lane == plane) {
#pragma unroll
            for (int j = 0; j < MW; j += 2) {
                *reinterpret_cast<double2 *>(prr + j) = make_double2(Rr[j], Rr[j + 1]);
                *reinterpret_cast<double2 *>(pri + j) = make_double2(Ri[j], Ri[j + 1]);
            }
        }
        if (lane < MW) {
            wvr[lane] = lane == plane ? 1.0 : mr;
            wvi[lane] = lane == plane ? 0.0 : mi;
        }
        __syncwarp(gm);
#pragma unroll
        for (int j = 0; j < MW; j += 2) {
            const double2 ar = *reinterpret_cast<const double2 *>(prr + j);
            const double2 ai = *reinterpret_cast<const double2 *>(pri + j);
            Rr[j] = fma(-mr, ar.x, fma(mi, ai.x, Rr[j]));
            Ri[j] = fma(-mr, ai.x, fma(-mi, ar.x, Ri[j]));
            Rr[j + 1] = fma(-mr, ar.y, fma(mi, ai.y, Rr[j + 1]));
            Ri[j + 1] = fma(-mr, ai.y, fma(-mi, ar.y, Ri[j + 1]));
        }
        double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
#pragma unroll
        for (int j = 0; j < MW; j += 2) {
            const double2 wr = *reinterpret_cast<const double2 *>(wvr + j);
            const double2 wi = *reinterpret_cast<const double2 *>(wvi + j);
            sr0 = fma(wr.x, Rr[j], fma(-wi.x, Ri[j], sr0));
            si0 = fma(wr.x, Ri[j], fma(wi.x, Rr[j], si0));
            sr1 = fma(wr.y, Rr[j + 1], fma(-wi.y, Ri[j + 1], sr1));
            si1 = fma(wr.y, Ri[j + 1], fma(wi.y, Rr[j + 1], si1));
        }
        pcr = sr0 + sr1;
        pci = si0 + si1;
        __syncwarp(gm);
    }
    const int lastslot = (int)__reduce_max_sync(gm, lab == m - 1 ? (unsigned)(lane + 1) : 0u) - 1;
    double cr = 0.0, ci = 0.0;
#pragma unroll
    for (int j = 0; j < MW; ++j)
        if (j == lastslot) {
            cr = Rr[j];
            ci = Ri[j];
        }
    for (int k = (m >= 3 ? m - 1 : 1); k <= m; ++k) {
        cd sub = xprev;
        if (k == m && k >= 2) sub = cd{__shfl_sync(gm, pcr, lastslot, G), __shfl_sync(gm, pci, lastslot, G)};
        if (k == m) feed(k, cr, ci, sub);
        else feed(k, pcr, pci, sub);
    }
    __syncwarp(gm);
    labudde_diag_c<MW, G>(cft, hk, (cd *)ws.q, m, n, lane, gm);
    __syncwarp(gm);
    return series_q_c<G>((const cd *)ws.q, m, n, lane, gm);
}

}  // namespace egg
