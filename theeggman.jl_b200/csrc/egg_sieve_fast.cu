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
//     magnitude (sign-free double bits) above 7 bits of (127 - label), so ties go to the smallest
//     logical index as in the reference.  Entries within 2^-13 of each other may pick either; any
//     near-maximal pivot keeps the multipliers bounded by ~1.
//   * The current pivot column (logical s-1) is kept in a scalar per row, `pc`.  The row update
//     M[i, :] -= mult_i * M[piv, :] runs over all slots with mult_i = 0 for rows that are not below
//     the pivot (so they are left bit-for-bit unchanged); slots of finished columns hold values that
//     are never read again except multiplied by zero.
//   * The column update M[:, s] += sum_i mult_i M[:, i] is a dot product of each row with a weight
//     vector that is mult_i on the live rows' slots and exactly 1 on the pivot slot, which yields
//     the updated column s directly -- the next step's `pc` -- with no dynamic register index.
//
// Each finished Hessenberg column feeds La Budde's recurrence (src/hafnian.jl:454-492) at once,
// so only the last n+1 rows of the coefficient table are kept (a ring in shared memory), and the
// [lambda^n] series coefficient (src/hafnian.jl:502-514) is a warp reduction per order.  All
// arithmetic is FP64 with fused multiply-adds; terms are accumulated in double-double per warp.
//
// Terms whose size exceeds the register tile (complex m > 32) are left to the exact kernel, which
// sums them into separate partials.
#include "egg_sieve.cuh"

namespace egg {

static constexpr unsigned FULL = 0xffffffffu;

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

__device__ __forceinline__ unsigned pivot_key(double a, int lab)
{
    // a >= 0 (a magnitude); NaN never wins
    unsigned hi = (unsigned)__double2hiint(a);
    if (a != a) hi = 0;
    return (hi & ~127u) | (unsigned)(127 - lab);
}

// Per-warp shared scratch of the fast path.
struct FastWs {
    double *prow;  // pivot row, by physical slot [64]
    double *wv;    // column-update weights, by physical slot [64]
    double *cf;    // La Budde coefficients coef_i, by i [64]
    double *C;     // ring of n+1 coefficient rows, (n+1) x (n+1)
    double *f;     // series coefficients [n+1]
    int *eidx;     // surviving edges, compacted [32]
    double *kval;  // their multiplicities after the Glynn substitution [32]
};

// Rows of the La Budde table live in a ring of RR = 2^p >= n+1 rows (row r in slot r & (RR-1)):
// row k reads rows k-1 .. k-n only.
__host__ __device__ inline int ring_rows(int nmax)
{
    int rr = 1;
    while (rr < nmax + 1) rr <<= 1;
    return rr;
}

__host__ __device__ inline size_t fast_ws_doubles(int nmax, int cplx)
{
    const size_t v = cplx ? 2 : 1;  // doubles per value
    size_t d = 64 * 3 + v * (size_t)ring_rows(nmax) * (nmax + 1) + v * (nmax + 1) + 32 /*kval*/ + 16 /*eidx*/;
    return (d + 1) & ~(size_t)1;  // keep every warp's region 16-byte aligned
}

__device__ inline FastWs fast_carve(double *base, int nmax, int cplx)
{
    const size_t v = cplx ? 2 : 1;
    FastWs w;
    double *p = base;
    w.prow = p; p += 64;
    w.wv = p; p += 64;
    w.cf = p; p += 64;
    w.C = p; p += v * (size_t)ring_rows(nmax) * (nmax + 1);
    w.f = p; p += v * (nmax + 1);
    w.kval = p; p += 32;
    w.eidx = (int *)p;
    return w;
}

// ---- La Budde step k (1-based), lanes over t --------------------------------------------------------
//   C[k][t] = (t <= min(k-1,n) ? C[k-1][t] : 0) - hkk C[k-1][t-1] - sum_{i=ilo}^{k-1} cf[i] C[i-1][t-k+i-1]
// Row r of C lives in ring slot (r & rm) with row stride cs = n+1.
__device__ __forceinline__ void labudde_row(double *C, const double *cf, int k, int n, int rm, double hkk, int lane)
{
    const int cs = n + 1;
    const double *Cp = C + (size_t)((k - 1) & rm) * cs;
    double *Ck = C + (size_t)(k & rm) * cs;
    const int tmax = k < n ? k : n, prevmax = (k - 1) < n ? (k - 1) : n;
    const int ilo = 1 > k - n + 1 ? 1 : k - n + 1;
    for (int t = lane; t <= n; t += 32) {
        double v;
        if (t == 0) v = Cp[0];
        else if (t <= tmax) v = (t <= prevmax ? Cp[t] : 0.0) - hkk * Cp[t - 1];
        else v = 0.0;
        if (t >= 1 && t <= tmax) {
            // term i reads row i-1 at column u = t-k+i-1; as i steps down by one, so do both
            const int i0 = ilo > k - t + 1 ? ilo : k - t + 1;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            int i = k - 1;
            for (; i - 3 >= i0; i -= 4) {
                const int u = t - k + i - 1;
                a0 = fma(cf[i], C[(size_t)((i - 1) & rm) * cs + u], a0);
                a1 = fma(cf[i - 1], C[(size_t)((i - 2) & rm) * cs + u - 1], a1);
                a2 = fma(cf[i - 2], C[(size_t)((i - 3) & rm) * cs + u - 2], a2);
                a3 = fma(cf[i - 3], C[(size_t)((i - 4) & rm) * cs + u - 3], a3);
            }
            for (; i >= i0; --i) a0 = fma(cf[i], C[(size_t)((i - 1) & rm) * cs + (t - k + i - 1)], a0);
            v -= (a0 + a1) + (a2 + a3);
        }
        Ck[t] = v;
    }
}

// [lambda^n] det(I - lambda H)^(-1/2) from q_j = C[m][j]; warp-parallel over j for each order t.
__device__ double series_coeff(const double *C, int m, int n, int rm, double *f, int lane)
{
    const int cs = n + 1;
    const double *q = C + (size_t)(m & rm) * cs;
    if (lane == 0) f[0] = 1.0;
    __syncwarp();
    double ft = 1.0;
    for (int t = 1; t <= n; ++t) {
        const int jm = t < m ? t : m;
        double s = 0.0;
        for (int j = 1 + lane; j <= jm; j += 32) s = fma((double)(2 * t - j) * q[j], f[t - j], s);
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
        ft = -s / (double)(2 * t);
        if (lane == 0) f[t] = ft;
        __syncwarp();
    }
    return ft;
}

// Complex versions (values interleaved as cd in the same ring layout).
__device__ __forceinline__ void labudde_row_c(cd *C, const cd *cf, int k, int n, int rm, cd hkk, int lane)
{
    const int cs = n + 1;
    const cd *Cp = C + (size_t)((k - 1) & rm) * cs;
    cd *Ck = C + (size_t)(k & rm) * cs;
    const int tmax = k < n ? k : n, prevmax = (k - 1) < n ? (k - 1) : n;
    const int ilo = 1 > k - n + 1 ? 1 : k - n + 1;
    for (int t = lane; t <= n; t += 32) {
        cd v;
        if (t == 0) v = Cp[0];
        else if (t <= tmax) {
            cd a = t <= prevmax ? Cp[t] : cd{0.0, 0.0};
            cd b = Cp[t - 1];
            v.re = a.re - (hkk.re * b.re - hkk.im * b.im);
            v.im = a.im - (hkk.re * b.im + hkk.im * b.re);
        } else v = cd{0.0, 0.0};
        if (t >= 1 && t <= tmax) {
            int i0 = ilo > k - t + 1 ? ilo : k - t + 1;
            double sr = 0.0, si = 0.0, tr = 0.0, ti = 0.0;
            int i = k - 1;
            for (; i - 1 >= i0; i -= 2) {
                const int u = t - k + i - 1;
                const cd c = cf[i], x = C[(size_t)((i - 1) & rm) * cs + u];
                const cd c2 = cf[i - 1], x2 = C[(size_t)((i - 2) & rm) * cs + u - 1];
                sr = fma(c.re, x.re, fma(-c.im, x.im, sr));
                si = fma(c.re, x.im, fma(c.im, x.re, si));
                tr = fma(c2.re, x2.re, fma(-c2.im, x2.im, tr));
                ti = fma(c2.re, x2.im, fma(c2.im, x2.re, ti));
            }
            if (i >= i0) {
                const cd c = cf[i], x = C[(size_t)((i - 1) & rm) * cs + (t - k + i - 1)];
                sr = fma(c.re, x.re, fma(-c.im, x.im, sr));
                si = fma(c.re, x.im, fma(c.im, x.re, si));
            }
            v.re -= sr + tr;
            v.im -= si + ti;
        }
        Ck[t] = v;
    }
}

__device__ cd series_coeff_c(const cd *C, int m, int n, int rm, cd *f, int lane)
{
    const int cs = n + 1;
    const cd *q = C + (size_t)(m & rm) * cs;
    if (lane == 0) f[0] = cd{1.0, 0.0};
    __syncwarp();
    cd ft{1.0, 0.0};
    for (int t = 1; t <= n; ++t) {
        const int jm = t < m ? t : m;
        double sr = 0.0, si = 0.0;
        for (int j = 1 + lane; j <= jm; j += 32) {
            const double w = (double)(2 * t - j);
            const cd a{w * q[j].re, w * q[j].im}, b = f[t - j];
            sr = fma(a.re, b.re, fma(-a.im, b.im, sr));
            si = fma(a.re, b.im, fma(a.im, b.re, si));
        }
        for (int off = 16; off > 0; off >>= 1) {
            sr += __shfl_xor_sync(FULL, sr, off);
            si += __shfl_xor_sync(FULL, si, off);
        }
        const double d2 = 1.0 / (double)(2 * t);
        ft = cd{-sr * d2, -si * d2};
        if (lane == 0) f[t] = ft;
        __syncwarp();
    }
    return ft;
}

// ---- one real term, m <= 32 * RPL, register tile of MW columns ----------------------------------
template <int MW, int RPL>
__device__ __noinline__ double term_real(const double *__restrict__ Axs, int lda, int E, int mE, int n, int rm,
                                         FastWs &w, int lane)
{
    const int m = 2 * mE;
    double R[RPL][MW];
    int lab[RPL];
    double pc[RPL], bet[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
        const int r = lane + 32 * q;
        lab[q] = r;
        bet[q] = 0.0;
        const bool live = r < m;
        const int ra = live ? (r < mE ? w.eidx[r] : w.eidx[r - mE] + E) : 0;
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            double v = 0.0;
            if (live && j < m) {
                const int b = j < mE ? j : j - mE;
                const int col = w.eidx[b] + (j < mE ? E : 0);
                v = w.kval[b] * __ldg(Axs + (size_t)col * lda + ra);
            }
            R[q][j] = v;
        }
        pc[q] = R[q][0];
    }
    // La Budde row 0
    for (int t = lane; t <= n; t += 32) w.C[t] = t == 0 ? 1.0 : 0.0;
    double xprev = 0.0;  // subdiagonal entry of the previous step
    for (int s = 1; s <= m - 2; ++s) {
        // -- pivot among rows with s <= label < m
        unsigned key = 0;
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lab[q] >= s && lab[q] < m) {
                unsigned k2 = pivot_key(fabs(pc[q]), lab[q]);
                key = k2 > key ? k2 : key;
            }
        const unsigned best = __reduce_max_sync(FULL, key);
        const int plab = 127 - (int)(best & 127u);
        int mine = -1;
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lab[q] == plab) mine = q;
        const unsigned own = __ballot_sync(FULL, mine >= 0);
        const int plane = __ffs(own) - 1;
        const int pq = __shfl_sync(FULL, mine, plane);
        const int pslot = plane + 32 * pq;
        const double x = __shfl_sync(FULL, (RPL > 1 && mine == RPL - 1) ? pc[RPL - 1] : pc[0], plane);
        // -- relabel (similarity swap of logical s and plab)
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            if (lab[q] == s) lab[q] = plab;
            else if (lab[q] == plab) lab[q] = s;
        }
        // -- column s-1 is final for rows with label <= s: feed La Budde step k = s
        {
            // beta_{i,s} for i = lab+1: multiply by the subdiagonal h_{s,s-1} = xprev (s >= 2)
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                if (lab[q] <= s - 3) bet[q] *= xprev;
                else if (lab[q] == s - 2) bet[q] = xprev;
                if (lab[q] <= s - 2) w.cf[lab[q] + 1] = pc[q] * bet[q];
            }
            double hkk = 0.0;
#pragma unroll
            for (int q = 0; q < RPL; ++q)
                if (lab[q] == s - 1) hkk = pc[q];
            const unsigned hown = __ballot_sync(FULL, [&] {
                bool o = false;
#pragma unroll
                for (int q = 0; q < RPL; ++q) o |= lab[q] == s - 1;
                return o;
            }());
            hkk = __shfl_sync(FULL, hkk, __ffs(hown) - 1);
            __syncwarp();
            labudde_row(w.C, w.cf, s, n, rm, hkk, lane);
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
            __syncwarp();
            continue;
        }
        const double rx = recip(x);
        double mult[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) mult[q] = (lab[q] > s && lab[q] < m) ? pc[q] * rx : 0.0;
        if (lane == plane) {
#pragma unroll
            for (int j = 0; j < MW; ++j) w.prow[j] = (RPL > 1 && pq == RPL - 1) ? R[RPL - 1][j] : R[0][j];
        }
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int r = lane + 32 * q;
            if (r < MW) w.wv[r] = r == pslot ? 1.0 : mult[q];
        }
        __syncwarp();
        // -- row update: M[i, :] -= mult_i * M[piv, :]
#pragma unroll
        for (int j = 0; j < MW; j += 2) {
            const double2 p2 = *reinterpret_cast<const double2 *>(w.prow + j);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                R[q][j] = fma(-mult[q], p2.x, R[q][j]);
                if (j + 1 < MW) R[q][j + 1] = fma(-mult[q], p2.y, R[q][j + 1]);
            }
        }
        // -- column update: pc <- M[:, piv] + sum_i mult_i M[:, i]
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int j = 0; j < MW; j += 4) {
                const double2 w0 = *reinterpret_cast<const double2 *>(w.wv + j);
                a0 = fma(w0.x, R[q][j], a0);
                if (j + 1 < MW) a1 = fma(w0.y, R[q][j + 1], a1);
                if (j + 2 < MW) {
                    const double2 w1 = *reinterpret_cast<const double2 *>(w.wv + j + 2);
                    a2 = fma(w1.x, R[q][j + 2], a2);
                    if (j + 3 < MW) a3 = fma(w1.y, R[q][j + 3], a3);
                }
            }
            pc[q] = (a0 + a1) + (a2 + a3);
        }
        __syncwarp();
    }
    // Last two columns: m-2 is `pc`, m-1 is the physical slot carrying label m-1.  Feed La Budde
    // steps k = m-1 and k = m (for m == 2 the loop above did not run and k = 1, 2 remain).
    int lastslot = 0;
    {
        int mine = -1;
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lab[q] == m - 1) mine = q;
        const unsigned own = __ballot_sync(FULL, mine >= 0);
        const int ln = __ffs(own) - 1;
        lastslot = ln + 32 * __shfl_sync(FULL, mine, ln);
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
        // column k-1 is `pc` for k = m-1 (or k = 1 when m == 2), `colm1` for k = m
        const bool last = (k == m);
        double sub = xprev;  // h_{k,k-1}
        if (k >= 2) {
            // h_{k,k-1} = H[k-1][k-2]: for k = m-1 that is the last pivot value; for k = m it is the
            // entry of the row labelled m-1 in column m-2 (= pc of that row).
            if (k == m) {
                double v = 0.0;
#pragma unroll
                for (int q = 0; q < RPL; ++q)
                    if (lab[q] == m - 1) v = pc[q];
                const unsigned o = __ballot_sync(FULL, [&] {
                    bool b = false;
#pragma unroll
                    for (int q = 0; q < RPL; ++q) b |= lab[q] == m - 1;
                    return b;
                }());
                sub = __shfl_sync(FULL, v, __ffs(o) - 1);
            }
        }
        double hkk = 0.0;
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const double colv = last ? colm1[q] : pc[q];
            if (k >= 2) {
                if (lab[q] <= k - 3) bet[q] *= sub;
                else if (lab[q] == k - 2) bet[q] = sub;
                if (lab[q] <= k - 2) w.cf[lab[q] + 1] = colv * bet[q];
            }
            if (lab[q] == k - 1) hkk = colv;
        }
        const unsigned hown = __ballot_sync(FULL, [&] {
            bool o = false;
#pragma unroll
            for (int q = 0; q < RPL; ++q) o |= lab[q] == k - 1;
            return o;
        }());
        hkk = __shfl_sync(FULL, hkk, __ffs(hown) - 1);
        __syncwarp();
        labudde_row(w.C, w.cf, k, n, rm, hkk, lane);
        __syncwarp();
    }
    return series_coeff(w.C, m, n, rm, w.f, lane);
}

// ---- one complex term, m <= 32 --------------------------------------------------------------------
template <int MW>
__device__ __noinline__ cd term_cplx(const cd *__restrict__ Axs, int lda, int E, int mE, int n, int rm, FastWs &w,
                                     int lane)
{
    const int m = 2 * mE;
    double Rr[MW], Ri[MW];
    int lab = lane;
    const bool live = lane < m;
    {
        const int ra = live ? (lane < mE ? w.eidx[lane] : w.eidx[lane - mE] + E) : 0;
#pragma unroll
        for (int j = 0; j < MW; ++j) {
            double vr = 0.0, vi = 0.0;
            if (live && j < m) {
                const int b = j < mE ? j : j - mE;
                const int col = w.eidx[b] + (j < mE ? E : 0);
                const double2 z2 = __ldg(reinterpret_cast<const double2 *>(Axs + (size_t)col * lda + ra));
                const cd z{z2.x, z2.y};
                const double kb = w.kval[b];
                vr = kb * z.re;
                vi = kb * z.im;
            }
            Rr[j] = vr;
            Ri[j] = vi;
        }
    }
    double pcr = Rr[0], pci = Ri[0];
    cd bet{0.0, 0.0};
    cd *C = (cd *)w.C;
    cd *cfc = (cd *)w.cf;  // complex coefficients need 2 doubles each: cf and prow regions are adjacent
    double *prr = w.prow, *pri = w.prow + 32, *wvr = w.wv, *wvi = w.wv + 32;
    for (int t = lane; t <= n; t += 32) C[t] = t == 0 ? cd{1.0, 0.0} : cd{0.0, 0.0};
    cd xprev{0.0, 0.0};
    auto feed = [&](int k, double colr, double coli, cd sub) {
        if (k >= 2) {
            if (lab <= k - 3) bet = cd{bet.re * sub.re - bet.im * sub.im, bet.re * sub.im + bet.im * sub.re};
            else if (lab == k - 2) bet = sub;
            if (lab <= k - 2) cfc[lab + 1] = cd{colr * bet.re - coli * bet.im, colr * bet.im + coli * bet.re};
        }
        const unsigned hown = __ballot_sync(FULL, lab == k - 1);
        const int hl = __ffs(hown) - 1;
        cd hkk{__shfl_sync(FULL, colr, hl), __shfl_sync(FULL, coli, hl)};
        __syncwarp();
        labudde_row_c(C, cfc, k, n, rm, hkk, lane);
        __syncwarp();
    };
    for (int s = 1; s <= m - 2; ++s) {
        unsigned key = 0;
        if (lab >= s && lab < m) key = pivot_key(fma(pcr, pcr, pci * pci), lab);
        const unsigned best = __reduce_max_sync(FULL, key);
        const int plab = 127 - (int)(best & 127u);
        const unsigned own = __ballot_sync(FULL, lab == plab);
        const int plane = __ffs(own) - 1;
        const double xr = __shfl_sync(FULL, pcr, plane), xi = __shfl_sync(FULL, pci, plane);
        if (lab == s) lab = plab;
        else if (lab == plab) lab = s;
        feed(s, pcr, pci, xprev);
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
            for (int j = 0; j < MW; ++j) {
                prr[j] = Rr[j];
                pri[j] = Ri[j];
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
            if (j + 1 < MW) {
                Rr[j + 1] = fma(-mr, ar.y, fma(mi, ai.y, Rr[j + 1]));
                Ri[j + 1] = fma(-mr, ai.y, fma(-mi, ar.y, Ri[j + 1]));
            }
        }
        double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
#pragma unroll
        for (int j = 0; j < MW; j += 2) {
            const double2 wr = *reinterpret_cast<const double2 *>(wvr + j);
            const double2 wi = *reinterpret_cast<const double2 *>(wvi + j);
            sr0 = fma(wr.x, Rr[j], fma(-wi.x, Ri[j], sr0));
            si0 = fma(wr.x, Ri[j], fma(wi.x, Rr[j], si0));
            if (j + 1 < MW) {
                sr1 = fma(wr.y, Rr[j + 1], fma(-wi.y, Ri[j + 1], sr1));
                si1 = fma(wr.y, Ri[j + 1], fma(wi.y, Rr[j + 1], si1));
            }
        }
        pcr = sr0 + sr1;
        pci = si0 + si1;
        __syncwarp();
    }
    const unsigned lown = __ballot_sync(FULL, lab == m - 1);
    const int lastslot = __ffs(lown) - 1;
    double cr = 0.0, ci = 0.0;
#pragma unroll
    for (int j = 0; j < MW; ++j)
        if (j == lastslot) {
            cr = Rr[j];
            ci = Ri[j];
        }
    for (int k = (m >= 3 ? m - 1 : 1); k <= m; ++k) {
        cd sub = xprev;
        if (k == m && k >= 2) {
            const unsigned o = __ballot_sync(FULL, lab == m - 1);
            const int l = __ffs(o) - 1;
            sub = cd{__shfl_sync(FULL, pcr, l), __shfl_sync(FULL, pci, l)};
        }
        if (k == m) feed(k, cr, ci, sub);
        else feed(k, pcr, pci, sub);
    }
    return series_coeff_c(C, m, n, rm, (cd *)w.f, lane);
}

// ---- kernel ------------------------------------------------------------------------------------

// Size classes: terms with MLO < m <= MHI (RPL rows per lane).  Each class is its own kernel with
// its own register budget, so the small tiles run at high occupancy; every class walks all of the
// instance's terms (the walk costs a few dozen instructions per term) and evaluates its own.
template <bool CPLX, int RPL, int MLO, int MHI>
struct SizeClass {
    // Blocks of 256 threads kept resident per SM, i.e. the register budget per thread
    // (65536 / (256 * min_blocks)): sized so each class's tiles fit without spilling in the
    // elimination loops.
    static constexpr int min_blocks = CPLX ? (MHI <= 16 ? 2 : 1) : (MHI <= 16 ? 3 : (MHI <= 32 ? 2 : 1));
};

template <bool CPLX, int RPL, int MLO, int MHI>
__device__ __forceinline__ void eval_term(const void *Ax, int lda, int E, int mE, int n, int rm, FastWs &w, int lane,
                                          double prefac, dd &acc_re, dd &acc_im)
{
    const int mw = (2 * mE + 3) & ~3;  // register tile: the next multiple of 4 (MLO < m <= MHI)
    if constexpr (!CPLX) {
        const double *A = (const double *)Ax;
        double val = 0.0;
#define EGG_TILE(MWV)                                                                  \
    if constexpr (MLO < MWV && MWV <= MHI) {                                            \
        if (mw <= MWV) {                                                                \
            val = term_real<MWV, (MWV > 32 ? 2 : 1)>(A, lda, E, mE, n, rm, w, lane);    \
            goto done_real;                                                             \
        }                                                                               \
    }
        EGG_TILE(4) EGG_TILE(8) EGG_TILE(12) EGG_TILE(16) EGG_TILE(20) EGG_TILE(24)
        EGG_TILE(28) EGG_TILE(32) EGG_TILE(36) EGG_TILE(40) EGG_TILE(44) EGG_TILE(48)
#undef EGG_TILE
    done_real:
        if (lane == 0) dd_add(acc_re, prefac * val);
    } else {
        const cd *A = (const cd *)Ax;
        cd val{0.0, 0.0};
#define EGG_TILE(MWV)                                                        \
    if constexpr (MLO < MWV && MWV <= MHI) {                                  \
        if (mw <= MWV) {                                                      \
            val = term_cplx<MWV>(A, lda, E, mE, n, rm, w, lane);              \
            goto done_cplx;                                                   \
        }                                                                     \
    }
        EGG_TILE(4) EGG_TILE(8) EGG_TILE(12) EGG_TILE(16) EGG_TILE(20) EGG_TILE(24) EGG_TILE(28) EGG_TILE(32)
#undef EGG_TILE
    done_cplx:
        if (lane == 0) {
            dd_add(acc_re, prefac * val.re);
            dd_add(acc_im, prefac * val.im);
        }
    }
    (void)RPL;
}

template <bool CPLX, int RPL, int MLO, int MHI>
__global__ void __launch_bounds__(256, (SizeClass<CPLX, RPL, MLO, MHI>::min_blocks))
    sieve_fast_kernel(SieveArgs a, const int64_t *__restrict__ strides, int warps_per_block, dd *partial)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    const int E = in.E, n = in.n;
    const int rm = ring_rows(a.nmax) - 1;
    FastWs w = fast_carve(smem + (size_t)wib * fast_ws_doubles(a.nmax, CPLX), a.nmax, CPLX);
    const int wslot = blockIdx.x * warps_per_block + wib;
    const int64_t W = a.warps_per_inst;
    const int64_t chunk = (in.steps + W - 1) / W;
    const int64_t j0 = wslot * chunk;
    const int64_t j1 = j0 + chunk < in.steps ? j0 + chunk : in.steps;
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    const int *reps = a.reps + in.reps_off;
    const int mr1 = a.maxrep + 1;
    const void *Ax = CPLX ? (const void *)((const cd *)a.Ax + in.ax_off) : (const void *)((const double *)a.Ax + in.ax_off);
    // Odometer: lane i holds digit i (edge E-1 least significant); digit 0 clipped under Glynn.
    int r = 0, base = 1, digit = 0;
    if (lane < E) {
        r = reps[lane];
        base = (in.glynn && lane == 0) ? (r + 2) / 2 : r + 1;
        if (j0 < j1) digit = (int)((j0 / strides[in.reps_off + lane]) % base);
    }
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
        double bp = lane < E ? a.binoms[r + digit * mr1] : 1.0;
        for (int off = 16; off > 0; off >>= 1) bp *= __shfl_xor_sync(FULL, bp, off);
        double prefac = ((n - esum) & 1) ? -bp : bp;
        const int k0 = __shfl_sync(FULL, kk, 0);
        if (in.glynn && k0 == 0) prefac *= 0.5;
        if (nz) {
            const int pos = __popc(mask & ((1u << lane) - 1u));
            w.eidx[pos] = lane;
            w.kval[pos] = (double)kk;
        }
        __syncwarp();
        eval_term<CPLX, RPL, MLO, MHI>(Ax, in.lda, E, mE, n, rm, w, lane, prefac, acc_re, acc_im);
        __syncwarp();
    }
    if (lane == 0) {
        dd *out = partial + ((size_t)b * W + wslot) * 2;
        out[0] = acc_re;
        out[1] = acc_im;
    }
}

size_t fast_smem_bytes(int nmax, int cplx, int warps)
{
    return (size_t)warps * fast_ws_doubles(nmax, cplx) * sizeof(double);
}

template <bool CPLX, int RPL, int MLO, int MHI>
static int launch_one(const SieveArgs &a, const int64_t *strides, dim3 grid, int wpb, size_t smem, dd *partial,
                      cudaStream_t st)
{
    auto k = sieve_fast_kernel<CPLX, RPL, MLO, MHI>;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, wpb * 32, smem, st>>>(a, strides, wpb, partial);
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

const int kFastClasses[][2] = {{0, 16}, {16, 24}, {24, 32}, {32, 40}, {40, 48}};

int launch_fast(const SieveArgs &a, const int64_t *strides, int B, int cplx, int cls, dd *partial, int wpb,
                int blocks_x, cudaStream_t st)
{
    const size_t smem = fast_smem_bytes(a.nmax, cplx, wpb);
    dim3 grid((unsigned)blocks_x, (unsigned)B);
    if (cplx) {
        switch (cls) {
        case 0: return launch_one<true, 1, 0, 16>(a, strides, grid, wpb, smem, partial, st);
        case 1: return launch_one<true, 1, 16, 24>(a, strides, grid, wpb, smem, partial, st);
        case 2: return launch_one<true, 1, 24, 32>(a, strides, grid, wpb, smem, partial, st);
        }
    } else {
        switch (cls) {
        case 0: return launch_one<false, 1, 0, 16>(a, strides, grid, wpb, smem, partial, st);
        case 1: return launch_one<false, 1, 16, 24>(a, strides, grid, wpb, smem, partial, st);
        case 2: return launch_one<false, 1, 24, 32>(a, strides, grid, wpb, smem, partial, st);
        case 3: return launch_one<false, 2, 32, 40>(a, strides, grid, wpb, smem, partial, st);
        case 4: return launch_one<false, 2, 40, 48>(a, strides, grid, wpb, smem, partial, st);
        }
    }
    return fail(EGG_ERR_ARGUMENT, "no such sieve size class");
}

}  // namespace egg
