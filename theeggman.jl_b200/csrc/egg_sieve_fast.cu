// egg_sieve_fast.cu -- register-resident sieve terms (the fast path of the device sieve).
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
// Each finished Hessenberg column feeds La Budde's recurrence (src/hafnian.jl:454-492) at once:
// lanes own coefficient orders t and walk the coefficient table (shared memory, one row per order
// of leading minor) along a diagonal, one address step per term of the depth sum.  The [lambda^n] series coefficient
// (src/hafnian.jl:502-514) is accumulated push-style: once f_s is known every lane t > s adds its
// (t+s) q_{t-s} f_s, so each order costs one multiply-add per lane and one broadcast.  All arithmetic
// is FP64 with fused multiply-adds; terms are accumulated in double-double per warp.
//
// Terms whose size exceeds the register tiles (complex m > 32, real m > 48) or whose order n
// exceeds 31 are left to the exact kernel, which sums them into separate partials.
#include "egg_sieve.cuh"

namespace egg {

static constexpr unsigned FULL = 0xffffffffu;

// -1 / (2t) for t = 0..63, rounded on the host (entry 0 unused).
__constant__ double c_neg_inv_2t[64];

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
    double *cf;    // La Budde coefficients coef_i, by i [64] (complex: 32 values)
    double *C;     // La Budde coefficient table by diagonals, (mhi+1) x (mhi+1) values (see labudde_row)
    double *kval;  // multiplicities of the surviving edges after the Glynn substitution [32]
    int *eidx;     // surviving edges, compacted [32]
};

__host__ __device__ inline size_t fast_ws_doubles(int nmax, int cplx, int mhi)
{
    const size_t v = cplx ? 2 : 1;  // doubles per value
    size_t d = 64 * 3 + v * (size_t)(mhi + 1) * (mhi + 1) + 32 /*kval*/ + 16 /*eidx*/;
    return (d + 1) & ~(size_t)1;  // keep every warp's region 16-byte aligned
}

__device__ inline FastWs fast_carve(double *base, int nmax, int cplx, int mhi)
{
    const size_t v = cplx ? 2 : 1;
    FastWs w;
    double *p = base;
    w.prow = p; p += 64;
    w.wv = p; p += 64;
    w.cf = p; p += 64;
    w.C = p; p += v * (size_t)(mhi + 1) * (mhi + 1);
    w.kval = p; p += 32;
    w.eidx = (int *)p;
    return w;
}

// ---- La Budde row k (1-based); lane t (0..n) owns coefficient t ----------------------------------
//   C[k][t] = (t <= min(k-1,n) ? C[k-1][t] : 0) - hkk C[k-1][t-1] - sum_{j=1}^{jmax} cf[k-j] C[k-1-j][t-1-j]
// (j = k - i of the reference's i loop, which runs i = k-1 .. max(1, k-n+1)).  The table is stored
// by diagonals: C[r][c] at T[(r - c) * rs + r].  Every entry of lane t's depth sum lies on its
// diagonal d = k - t, at rows k-2, k-3, ..., so the sum walks one contiguous run.  Entries left of
// column 0 (r < d) are zero -- they are cleared once per warp and never written -- so the walk
// needs no bounds test; entries right of the diagonal (c > r) are never read.  Every entry read
// in a term was written earlier in the same term.
__device__ __forceinline__ void labudde_row(double *T, const double *cf, int k, int n, int rs, double hkk, int lane)
{
    const int t = lane;
    const int tmax = k < n ? k : n;
    const int d = k - t;  // negative for lanes past row k: clamped below, their result is not stored
    double v = 0.0;
    if (t <= tmax) {
        const double a = t <= k - 1 ? T[(d - 1) * rs + (k - 1)] : 0.0;  // C[k-1][t]
        const double b = t >= 1 ? T[d * rs + (k - 1)] : 0.0;            // C[k-1][t-1]
        v = a - hkk * b;
    }
    const int jmax = (k - 1) < (n - 1) ? (k - 1) : (n - 1);
    const double *cfk = cf + k;
    const double *Td = T + (d > 0 ? d : 0) * rs + (k - 2);  // C[k-1-j][t-1-j] at Td[1 - j]
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
    for (int j = 1; j <= 31; ++j) {
        if (j > jmax) break;
        const double c = cfk[-j];
        const double x = Td[1 - j];
        if ((j & 3) == 1) a0 = fma(c, x, a0);
        else if ((j & 3) == 2) a1 = fma(c, x, a1);
        else if ((j & 3) == 3) a2 = fma(c, x, a2);
        else a3 = fma(c, x, a3);
    }
    if (t <= tmax) T[d * rs + k] = v - ((a0 + a1) + (a2 + a3));
}

// [lambda^n] det(I - lambda H)^(-1/2), push-style: lane t accumulates S_t = sum_j (2t-j) q_j f_{t-j}
// as the f's become known; f_t = -S_t / (2t).  q_j = C[m][j] = T[(m - j) * rs + m].  All lanes
// return f_n.
__device__ __forceinline__ double series_coeff(const double *T, int m, int n, int rs, int lane)
{
    double S = 0.0, fs = 1.0;  // fs = f_s, starting at f_0 = 1
    for (int s = 0; s < n; ++s) {
        const int j = lane - s;
        if (j >= 1 && j <= m && lane <= n) S = fma((double)(lane + s) * T[(m - j) * rs + m], fs, S);
        fs = __shfl_sync(FULL, S, s + 1) * c_neg_inv_2t[s + 1];
    }
    return fs;
}

__device__ __forceinline__ void labudde_row_c(cd *T, const cd *cf, int k, int n, int rs, cd hkk, int lane)
{
    const int t = lane;
    const int tmax = k < n ? k : n;
    const int d = k - t;
    cd v{0.0, 0.0};
    if (t <= tmax) {
        const cd a = t <= k - 1 ? T[(d - 1) * rs + (k - 1)] : cd{0.0, 0.0};
        const cd b = t >= 1 ? T[d * rs + (k - 1)] : cd{0.0, 0.0};
        v.re = a.re - fma(hkk.re, b.re, -hkk.im * b.im);
        v.im = a.im - fma(hkk.re, b.im, hkk.im * b.re);
    }
    const int jmax = (k - 1) < (n - 1) ? (k - 1) : (n - 1);
    const cd *cfk = cf + k;
    const cd *Td = T + (d > 0 ? d : 0) * rs + (k - 2);
    double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
#pragma unroll
    for (int j = 1; j <= 31; ++j) {
        if (j > jmax) break;
        const cd c = cfk[-j];
        const cd x = Td[1 - j];
        if (j & 1) {
            sr0 = fma(c.re, x.re, fma(-c.im, x.im, sr0));
            si0 = fma(c.re, x.im, fma(c.im, x.re, si0));
        } else {
            sr1 = fma(c.re, x.re, fma(-c.im, x.im, sr1));
            si1 = fma(c.re, x.im, fma(c.im, x.re, si1));
        }
    }
    if (t <= tmax) T[d * rs + k] = cd{v.re - (sr0 + sr1), v.im - (si0 + si1)};
}

__device__ __forceinline__ cd series_coeff_c(const cd *T, int m, int n, int rs, int lane)
{
    double Sr = 0.0, Si = 0.0, fr = 1.0, fi = 0.0;
    for (int s = 0; s < n; ++s) {
        const int j = lane - s;
        if (j >= 1 && j <= m && lane <= n) {
            const double w = (double)(lane + s);
            const cd q = T[(m - j) * rs + m];
            const double ar = w * q.re, ai = w * q.im;
            Sr = fma(ar, fr, fma(-ai, fi, Sr));
            Si = fma(ar, fi, fma(ai, fr, Si));
        }
        const double c = c_neg_inv_2t[s + 1];
        fr = __shfl_sync(FULL, Sr, s + 1) * c;
        fi = __shfl_sync(FULL, Si, s + 1) * c;
    }
    return cd{fr, fi};
}

// ---- one real term, m <= 32 * RPL, register tile of MW columns ----------------------------------
template <int MW, int RPL>
__device__ __forceinline__ double term_real(const double *__restrict__ Ax, int lda, int E, int mE, int n,
                                            const FastWs &ws, int lane)
{
    constexpr int rs = MW + 1;  // La Budde table row stride
    const int m = 2 * mE;
    double *prow = ws.prow, *wv = ws.wv, *cf = ws.cf, *C = ws.C;
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
    if (lane == 0) C[0] = 1.0;  // La Budde row 0: C[0][0] = 1
    int hslot = 0;       // physical slot of label s-1 (label 0 never moves)
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
        const unsigned best = __reduce_max_sync(FULL, key);
        const int pslot = 63 - (int)(best & 63u);
        const int plane = pslot & 31, pq = pslot >> 5;
        const double pcp = (RPL > 1 && pq == 1) ? pc[RPL - 1] : pc[0];
        const int labp = (RPL > 1 && pq == 1) ? lab[RPL - 1] : lab[0];
        const double x = __shfl_sync(FULL, pcp, plane);
        const int plab = __shfl_sync(FULL, labp, plane);
        // -- column s-1 is final for rows with label <= s-1 plus the pivot; feed La Budde step k = s
        {
            const double hcand = (RPL > 1 && (hslot >> 5) == 1) ? pc[RPL - 1] : pc[0];
            const double hkk = __shfl_sync(FULL, hcand, hslot & 31);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                if (lab[q] <= s - 3) bet[q] *= xprev;
                else if (lab[q] == s - 2) bet[q] = xprev;
                if (lab[q] <= s - 2) cf[lab[q] + 1] = pc[q] * bet[q];
            }
            __syncwarp();
            labudde_row(C, cf, s, n, rs, hkk, lane);
        }
        // -- relabel (similarity swap of logical s and plab)
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            if (lab[q] == s) lab[q] = plab;
            else if (lab[q] == plab) lab[q] = s;
        }
        hslot = pslot;
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
            __syncwarp();
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
        __syncwarp();
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
            for (int j = 0; j < MW; j += 4) {
                const double2 w0 = *reinterpret_cast<const double2 *>(wv + j);
                const double2 w1 = *reinterpret_cast<const double2 *>(wv + j + 2);
                a0 = fma(w0.x, R[q][j], a0);
                a1 = fma(w0.y, R[q][j + 1], a1);
                a2 = fma(w1.x, R[q][j + 2], a2);
                a3 = fma(w1.y, R[q][j + 3], a3);
            }
            pc[q] = (a0 + a1) + (a2 + a3);
        }
        __syncwarp();
    }
    // Last two columns: m-2 is `pc`, m-1 is the physical slot carrying label m-1.  Feed La Budde
    // steps k = m-1 and k = m (for m == 2 the loop above did not run and k = 1, 2 remain).
    int lastslot;
    {
        int mine = -1;
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lab[q] == m - 1) mine = lane + 32 * q;
        lastslot = (int)__reduce_max_sync(FULL, (unsigned)(mine + 1)) - 1;
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
            sub = __shfl_sync(FULL, cand, lastslot & 31);
        }
        double hkk = 0.0;
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const double colv = last ? colm1[q] : pc[q];
            if (k >= 2) {
                if (lab[q] <= k - 3) bet[q] *= sub;
                else if (lab[q] == k - 2) bet[q] = sub;
                if (lab[q] <= k - 2) cf[lab[q] + 1] = colv * bet[q];
            }
            if (lab[q] == k - 1) hkk = colv;
        }
        const int hs = last ? lastslot : hslot;
        hkk = __shfl_sync(FULL, hkk, hs & 31);
        __syncwarp();
        labudde_row(C, cf, k, n, rs, hkk, lane);
        __syncwarp();
    }
    return series_coeff(C, m, n, rs, lane);
}

// ---- one complex term, m <= 32 --------------------------------------------------------------------
template <int MW>
__device__ __forceinline__ cd term_cplx(const cd *__restrict__ Ax, int lda, int E, int mE, int n, const FastWs &ws,
                                        int lane)
{
    constexpr int rs = MW + 1;  // La Budde table row stride
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
    cd *C = (cd *)ws.C;
    cd *cfc = (cd *)ws.cf;  // 32 complex coefficients
    double *prr = ws.prow, *pri = ws.prow + 32, *wvr = ws.wv, *wvi = ws.wv + 32;
    if (lane == 0) C[0] = cd{1.0, 0.0};  // La Budde row 0: C[0][0] = 1
    int hslot = 0;
    cd xprev{0.0, 0.0};
    auto feed = [&](int k, double colr, double coli, cd sub, int hs) {
        if (k >= 2) {
            if (lab <= k - 3) bet = cd{fma(bet.re, sub.re, -bet.im * sub.im), fma(bet.re, sub.im, bet.im * sub.re)};
            else if (lab == k - 2) bet = sub;
            if (lab <= k - 2) cfc[lab + 1] = cd{fma(colr, bet.re, -coli * bet.im), fma(colr, bet.im, coli * bet.re)};
        }
        const cd hkk{__shfl_sync(FULL, colr, hs), __shfl_sync(FULL, coli, hs)};
        __syncwarp();
        labudde_row_c(C, cfc, k, n, rs, hkk, lane);
        __syncwarp();
    };
    for (int s = 1; s <= m - 2; ++s) {
        unsigned key = 0;
        if (lab >= s && lab < m) key = pivot_key(fma(pcr, pcr, pci * pci), lane);
        const unsigned best = __reduce_max_sync(FULL, key);
        const int plane = 63 - (int)(best & 63u);
        const double xr = __shfl_sync(FULL, pcr, plane), xi = __shfl_sync(FULL, pci, plane);
        const int plab = __shfl_sync(FULL, lab, plane);
        feed(s, pcr, pci, xprev, hslot);
        if (lab == s) lab = plab;
        else if (lab == plab) lab = s;
        hslot = plane;
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
        __syncwarp();
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
        __syncwarp();
    }
    const int lastslot = (int)__reduce_max_sync(FULL, lab == m - 1 ? (unsigned)(lane + 1) : 0u) - 1;
    double cr = 0.0, ci = 0.0;
#pragma unroll
    for (int j = 0; j < MW; ++j)
        if (j == lastslot) {
            cr = Rr[j];
            ci = Ri[j];
        }
    for (int k = (m >= 3 ? m - 1 : 1); k <= m; ++k) {
        cd sub = xprev;
        if (k == m && k >= 2) sub = cd{__shfl_sync(FULL, pcr, lastslot), __shfl_sync(FULL, pci, lastslot)};
        if (k == m) feed(k, cr, ci, sub, lastslot);
        else feed(k, pcr, pci, sub, hslot);
    }
    return series_coeff_c(C, m, n, rs, lane);
}

// ---- kernels -----------------------------------------------------------------------------------

// Size classes: terms with MLO < m <= MHI, each evaluated on one register tile of MHI columns
// (two rows per lane above 32).  Each class is its own kernel with its own register budget, so the
// small tiles run at high occupancy and each kernel holds one copy of the term code; every class
// walks all of the instance's terms (a few dozen instructions per term) and evaluates its own.
template <bool CPLX, int MHI>
struct SizeClass {
    // Block size and blocks kept resident per SM, i.e. the register budget per thread
    // (65536 / (threads * min_blocks)): sized so each class's tile fits without spilling.  The
    // real m <= 24 tile fits 96 registers, which 128-thread blocks turn into 20 resident warps
    // per SM (256-thread blocks would round down to 16).
    static constexpr int threads = (!CPLX && MHI > 16 && MHI <= 24) ? 128 : 256;
    static constexpr int min_blocks = CPLX ? (MHI <= 16 ? 2 : 1)
                                           : (MHI <= 8 ? 4 : (MHI <= 16 ? 3 : (MHI <= 24 ? 5 : (MHI <= 32 ? 2 : 1))));
};

template <bool CPLX, int MLO, int MHI>
__global__ void __launch_bounds__((SizeClass<CPLX, MHI>::threads), (SizeClass<CPLX, MHI>::min_blocks))
    sieve_fast_kernel(SieveArgs a, const int64_t *__restrict__ strides, int warps_per_block, dd *partial)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    const int E = in.E, n = in.n;
    const FastWs w = fast_carve(smem + (size_t)wib * fast_ws_doubles(a.nmax, CPLX, MHI), a.nmax, CPLX, MHI);
    // The La Budde table's entries left of column 0 must read as zero; nothing ever writes them.
    for (int i = lane; i < (CPLX ? 2 : 1) * (MHI + 1) * (MHI + 1); i += 32) w.C[i] = 0.0;
    __syncwarp();
    const int wslot = blockIdx.x * warps_per_block + wib;
    const int64_t W = a.warps_per_inst;
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    const int *reps = a.reps + in.reps_off;
    const int mr1 = a.maxrep + 1;
    const bool unit = a.maxrep <= 1;  // all multiplicities 1: every binomial factor is 1
    // Odometer: lane i holds digit i (edge E-1 least significant); digit 0 clipped under Glynn.
    int r = 0, base = 1, digit = 0;
    if (lane < E) {
        r = reps[lane];
        base = (in.glynn && lane == 0) ? (r + 2) / 2 : r + 1;
    }
    // Terms are dealt to warps in runs of kRunTerms consecutive indices, round robin.  A term's size
    // is set by its digits, and a long contiguous range fixes the high digits, so contiguous ranges
    // would hand some warps almost all of a size class and others none of it.
    constexpr int64_t kRunTerms = 16;
    for (int64_t j0 = wslot * kRunTerms; j0 < in.steps; j0 += W * kRunTerms) {
        const int64_t j1 = j0 + kRunTerms < in.steps ? j0 + kRunTerms : in.steps;
        if (lane < E) digit = (int)((j0 / strides[in.reps_off + lane]) % base);
        for (int64_t j = j0; j < j1; ++j) {
            if (j > j0) {
                const unsigned notmax = __ballot_sync(FULL, lane < E && digit != base - 1);
                const int h = 31 - __clz(notmax);
                if (lane == h) ++digit;
                else if (lane > h && lane < E) digit = 0;
            }
            const int kk = lane < E ? (in.glynn ? 2 * digit - r : digit) : 0;
            const bool nz = lane < E && kk != 0;
            const unsigned mask = __ballot_sync(FULL, nz);
            const int mE = __popc(mask);
            const int m = 2 * mE;
            if (m <= MLO || m > MHI) continue;  // another size class (or an empty term, which vanishes)
            const int esum = __reduce_add_sync(FULL, lane < E ? digit : 0);
            double bp = 1.0;
            if (!unit) {
                bp = lane < E ? a.binoms[r + digit * mr1] : 1.0;
                for (int off = 16; off > 0; off >>= 1) bp *= __shfl_xor_sync(FULL, bp, off);
            }
            double prefac = ((n - esum) & 1) ? -bp : bp;
            const int k0 = __shfl_sync(FULL, kk, 0);
            if (in.glynn && k0 == 0) prefac *= 0.5;
            if (nz) {
                const int pos = __popc(mask & ((1u << lane) - 1u));
                w.eidx[pos] = lane;
                w.kval[pos] = (double)kk;
            }
            __syncwarp();
            if constexpr (!CPLX) {
                const double val = term_real<MHI, (MHI > 32 ? 2 : 1)>((const double *)a.Ax + in.ax_off, in.lda, E, mE, n, w,
                                                                      lane);
                if (lane == 0) dd_add(acc_re, prefac * val);
            } else {
                const cd val = term_cplx<MHI>((const cd *)a.Ax + in.ax_off, in.lda, E, mE, n, w, lane);
                if (lane == 0) {
                    dd_add(acc_re, prefac * val.re);
                    dd_add(acc_im, prefac * val.im);
                }
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        dd *out = partial + ((size_t)b * W + wslot) * 2;
        out[0] = acc_re;
        out[1] = acc_im;
    }
}

size_t fast_smem_bytes(int nmax, int cplx, int cls, int warps)
{
    return (size_t)warps * fast_ws_doubles(nmax, cplx, kFastClasses[cls][1]) * sizeof(double);
}

template <bool CPLX, int MLO, int MHI>
static int launch_one(const SieveArgs &a, const int64_t *strides, dim3 grid, int wpb, int cls, dd *partial,
                      cudaStream_t st)
{
    // The same warps per instance as every class (grid.x * wpb), in this class's block size.
    constexpr int cw = SizeClass<CPLX, MHI>::threads / 32;
    grid.x = (unsigned)((int64_t)grid.x * wpb / cw);
    const size_t smem = fast_smem_bytes(a.nmax, CPLX, cls, cw);
    auto k = sieve_fast_kernel<CPLX, MLO, MHI>;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, cw * 32, smem, st>>>(a, strides, cw, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

const int kFastClasses[][2] = {{0, 8}, {8, 16}, {16, 24}, {24, 32}, {32, 40}, {40, 48}};

static int upload_tables(cudaStream_t st)
{
    // -1/(2t), computed with IEEE division on the host.
    static double host_tab[64];
    if (host_tab[1] == 0.0)
        for (int t = 1; t < 64; ++t) host_tab[t] = -1.0 / (2.0 * t);
    EGG_CUDA_TRY(cudaMemcpyToSymbolAsync(c_neg_inv_2t, host_tab, sizeof(host_tab), 0, cudaMemcpyHostToDevice, st));
    return EGG_OK;
}

int launch_fast(const SieveArgs &a, const int64_t *strides, int B, int cplx, int cls, dd *partial, int wpb,
                int blocks_x, cudaStream_t st)
{
    int rc = upload_tables(st);
    if (rc) return rc;
    dim3 grid((unsigned)blocks_x, (unsigned)B);
    if (cplx) {
        switch (cls) {
        case 0: return launch_one<true, 0, 8>(a, strides, grid, wpb, cls, partial, st);
        case 1: return launch_one<true, 8, 16>(a, strides, grid, wpb, cls, partial, st);
        case 2: return launch_one<true, 16, 24>(a, strides, grid, wpb, cls, partial, st);
        case 3: return launch_one<true, 24, 32>(a, strides, grid, wpb, cls, partial, st);
        }
    } else {
        switch (cls) {
        case 0: return launch_one<false, 0, 8>(a, strides, grid, wpb, cls, partial, st);
        case 1: return launch_one<false, 8, 16>(a, strides, grid, wpb, cls, partial, st);
        case 2: return launch_one<false, 16, 24>(a, strides, grid, wpb, cls, partial, st);
        case 3: return launch_one<false, 24, 32>(a, strides, grid, wpb, cls, partial, st);
        case 4: return launch_one<false, 32, 40>(a, strides, grid, wpb, cls, partial, st);
        case 5: return launch_one<false, 40, 48>(a, strides, grid, wpb, cls, partial, st);
        }
    }
    return fail(EGG_ERR_ARGUMENT, "no such sieve size class");
}

}  // namespace egg
