// egg_sieve.cu -- the Bjorklund/Glynn sieve (src/hafnian.jl:528-738) on the device.
//
// The reference has no device sieve (README.md:144-148: "roughly a 40 KB workspace per term").
// Here one warp evaluates one term at a time with its workspace in shared memory; lanes split the
// independent element updates of each step, and every element is updated in exactly the order and
// rounding of the reference loop (__dmul_rn/__dadd_rn, no contraction), so each term's value is
// bit-identical to the CPU's _glynn_term!.  Where the reference sums terms with a plain `+=`
// (:618-622), each warp keeps a double-double accumulator; the per-warp partials are then summed
// in a fixed tree, so results do not depend on scheduling.
//
// Work layout of this exact kernel.  Instance b's terms are dealt to that instance's warps
// (grid.y = instance): round robin over j = 0..steps-1, decoding the mixed-radix odometer per term
// (edge E least significant, the leading digit clipped to its lower half under Glynn, :655-657),
// or, for distinct-row inclusion-exclusion, as equal shares of each popcount level.  The fast
// register-tile kernels (egg_sieve_fast.cuh, egg_sieve_level*.cu) take every term that fits their
// tiles unless the exact mode is asked for; this driver launches both and the fixed-order
// reduction.  One small distinct-row instance instead takes a single all-levels launch of the
// register-tile kernel, which sums its own blocks' partials in a fixed order.
#include <cmath>
#include <cstring>
#include <map>

#include "egg_sieve.cuh"

namespace egg {

// Per-warp shared workspace, carved from dynamic shared memory.
struct WarpWs {
    double *M;   // real: M; complex: Mr
    double *Mi;  // complex: Mi
    double *u;   // multipliers (real) / ur
    double *ui;  // ui
    double *C;   // (m+1) x (n+1) rows of charpoly coefficients (complex: interleaved)
    double *f;   // n+1 series coefficients (complex: interleaved)
    int *kept, *idx, *rows;
    int ldm;
};

__host__ __device__ inline size_t ws_doubles(int Emax, int nmax, int cplx)
{
    size_t MM = 2 * (size_t)Emax, ld = MM + 1;
    size_t d = (cplx ? 2 : 1) * ld * MM + 2 * MM + (cplx ? 2 : 1) * (MM + 1) * (nmax + 1) + 2 * (nmax + 1);
    size_t ints = 2 * (size_t)Emax + MM;
    return d + (ints + 1) / 2 + 2;
}

__device__ inline WarpWs carve(double *base, int Emax, int nmax, int cplx)
{
    WarpWs w;
    int MM = 2 * Emax, ld = MM + 1;
    w.ldm = ld;
    double *p = base;
    w.M = p; p += (size_t)ld * MM;
    w.Mi = cplx ? p : nullptr; if (cplx) p += (size_t)ld * MM;
    w.u = p; p += MM;
    w.ui = p; p += MM;
    w.C = p; p += (size_t)(cplx ? 2 : 1) * (MM + 1) * (nmax + 1);
    w.f = p; p += 2 * (nmax + 1);
    int *ip = (int *)p;
    w.kept = ip; ip += Emax;
    w.idx = ip; ip += Emax;
    w.rows = ip;
    return w;
}

// Warp argmax with the reference's tie rule (the first index achieving the maximum, :212-221):
// returns the winning row.  a is this lane's candidate value (NaN entries must never win).
__device__ __forceinline__ int warp_first_argmax(double a, int i)
{
    for (int off = 16; off > 0; off >>= 1) {
        double a2 = __shfl_down_sync(0xffffffffu, a, off);
        int i2 = __shfl_down_sync(0xffffffffu, i, off);
        if (a2 > a || (a2 == a && i2 < i)) {
            a = a2;
            i = i2;
        }
    }
    return __shfl_sync(0xffffffffu, i, 0);
}

// _hessenberg!(M, m, mult), src/hafnian.jl:210-258, one warp, exact order, m <= 32 * NP.
// Each lane keeps its rows' multipliers (rows k+1+lane+32p) and its column-update sums (rows
// lane+32p) in registers, so that every element's chain of separately rounded operations runs in
// registers, in the reference's order, instead of through shared memory; the row update's skip of
// a zero M[k, j] is a select (the same value), so that four columns' loads overlap.
template <int NP>
__device__ void hessenberg_real_exact_np(WarpWs &w, int m, int lane)
{
    double *M = w.M;
    const int ld = w.ldm;
#define MX(i, j) M[(size_t)(j) * ld + (i)]
    for (int k = 1; k <= m - 2; ++k) {  // 0-based pivot row k, pivot column k-1
        const int col = k - 1;
        double a0 = fabs(MX(k, col));
        int p = k;
        if (a0 == a0) {
            double best = -1.0;
            int bi = 0x7fffffff;
            for (int i = k + lane; i < m; i += 32) {
                double a = fabs(MX(i, col));
                if (a != a) a = -1.0;
                if (a > best) {
                    best = a;
                    bi = i;
                }
            }
            p = warp_first_argmax(best, bi);
        }
        if (p != k) {
            for (int j = col + lane; j < m; j += 32) {
                double t = MX(p, j);
                MX(p, j) = MX(k, j);
                MX(k, j) = t;
            }
            __syncwarp();
            for (int i = lane; i < m; i += 32) {
                double t = MX(i, p);
                MX(i, p) = MX(i, k);
                MX(i, k) = t;
            }
            __syncwarp();
        }
        const double x = MX(k, col);
        if (x == 0.0) continue;
        double ui[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int i = k + 1 + lane + 32 * p;
            ui[p] = 0.0;
            if (i < m) {
                ui[p] = __ddiv_rn(MX(i, col), x);
                w.u[i] = ui[p];
                MX(i, col) = 0.0;
            }
        }
        __syncwarp();
        // Rows k+1.. minus u[i] * M[k, j], for j = k..m-1; a zero M[k, j] leaves its column as it is.
        int j = k;
        for (; j + 4 <= m; j += 4) {
            double a4[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) a4[q] = MX(k, j + q);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int i = k + 1 + lane + 32 * p;
                if (i < m) {
                    double v[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) v[q] = MX(i, j + q);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        MX(i, j + q) = a4[q] == 0.0 ? v[q] : __dsub_rn(v[q], __dmul_rn(ui[p], a4[q]));
                }
            }
        }
        for (; j < m; ++j) {
            const double akj = MX(k, j);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int i = k + 1 + lane + 32 * p;
                if (i < m) {
                    const double v = MX(i, j);
                    MX(i, j) = akj == 0.0 ? v : __dsub_rn(v, __dmul_rn(ui[p], akj));
                }
            }
        }
        __syncwarp();
        // Column k plus u[i] * column i for i = k+1..m-1 in order; a zero u[i] adds nothing.
        double acc[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int l = lane + 32 * p;
            acc[p] = l < m ? MX(l, k) : 0.0;
        }
#pragma unroll 4
        for (int i = k + 1; i < m; ++i) {
            const double mi = w.u[i];
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int l = lane + 32 * p;
                if (l < m) {
                    const double s = __dadd_rn(acc[p], __dmul_rn(mi, MX(l, i)));
                    acc[p] = mi == 0.0 ? acc[p] : s;
                }
            }
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int l = lane + 32 * p;
            if (l < m) MX(l, k) = acc[p];
        }
        __syncwarp();
    }
#undef MX
}

__device__ void hessenberg_real_exact(WarpWs &w, int m, int lane)
{
    if (m <= 32) hessenberg_real_exact_np<1>(w, m, lane);
    else if (m <= 64) hessenberg_real_exact_np<2>(w, m, lane);
    else if (m <= 96) hessenberg_real_exact_np<3>(w, m, lane);
    else hessenberg_real_exact_np<4>(w, m, lane);
}

// _hessenberg_split!(Mr, Mi, m, ur, ui), src/hafnian.jl:271-335, one warp, exact order, m <= 32 * NP;
// multipliers and column-update sums in registers as in the real form.
template <int NP>
__device__ void hessenberg_split_exact_np(WarpWs &w, int m, int lane)
{
    double *R = w.M, *I = w.Mi;
    const int ld = w.ldm;
#define RX(i, j) R[(size_t)(j) * ld + (i)]
#define IX(i, j) I[(size_t)(j) * ld + (i)]
    for (int k = 1; k <= m - 2; ++k) {
        const int col = k - 1;
        double a0 = __dadd_rn(__dmul_rn(RX(k, col), RX(k, col)), __dmul_rn(IX(k, col), IX(k, col)));
        int p = k;
        if (a0 == a0) {
            double best = -1.0;
            int bi = 0x7fffffff;
            for (int i = k + lane; i < m; i += 32) {
                double a = __dadd_rn(__dmul_rn(RX(i, col), RX(i, col)), __dmul_rn(IX(i, col), IX(i, col)));
                if (a != a) a = -1.0;
                if (a > best) {
                    best = a;
                    bi = i;
                }
            }
            p = warp_first_argmax(best, bi);
        }
        if (p != k) {
            for (int j = col + lane; j < m; j += 32) {
                double t = RX(p, j); RX(p, j) = RX(k, j); RX(k, j) = t;
                t = IX(p, j); IX(p, j) = IX(k, j); IX(k, j) = t;
            }
            __syncwarp();
            for (int i = lane; i < m; i += 32) {
                double t = RX(i, p); RX(i, p) = RX(i, k); RX(i, k) = t;
                t = IX(i, p); IX(i, p) = IX(i, k); IX(i, k) = t;
            }
            __syncwarp();
        }
        const double xr = RX(k, col), xi = IX(k, col);
        const double d = __dadd_rn(__dmul_rn(xr, xr), __dmul_rn(xi, xi));
        if (d == 0.0) continue;
        double ur[NP], uim[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int i = k + 1 + lane + 32 * p;
            ur[p] = 0.0;
            uim[p] = 0.0;
            if (i < m) {
                const double ar = RX(i, col), ai = IX(i, col);
                ur[p] = __ddiv_rn(__dadd_rn(__dmul_rn(ar, xr), __dmul_rn(ai, xi)), d);
                uim[p] = __ddiv_rn(__dsub_rn(__dmul_rn(ai, xr), __dmul_rn(ar, xi)), d);
                w.u[i] = ur[p];
                w.ui[i] = uim[p];
                RX(i, col) = 0.0;
                IX(i, col) = 0.0;
            }
        }
        __syncwarp();
#pragma unroll 2
        for (int j = k; j < m; ++j) {
            const double ar = RX(k, j), ai = IX(k, j);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int i = k + 1 + lane + 32 * p;
                if (i < m) {
                    const double vr = RX(i, j), vi = IX(i, j);
                    RX(i, j) = __dsub_rn(vr, __dsub_rn(__dmul_rn(ur[p], ar), __dmul_rn(uim[p], ai)));
                    IX(i, j) = __dsub_rn(vi, __dadd_rn(__dmul_rn(ur[p], ai), __dmul_rn(uim[p], ar)));
                }
            }
        }
        __syncwarp();
        double sr[NP], si[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int l = lane + 32 * p;
            sr[p] = l < m ? RX(l, k) : 0.0;
            si[p] = l < m ? IX(l, k) : 0.0;
        }
#pragma unroll 2
        for (int i = k + 1; i < m; ++i) {
            const double mr = w.u[i], mi = w.ui[i];
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int l = lane + 32 * p;
                if (l < m) {
                    const double r = RX(l, i), im = IX(l, i);
                    sr[p] = __dadd_rn(sr[p], __dsub_rn(__dmul_rn(mr, r), __dmul_rn(mi, im)));
                    si[p] = __dadd_rn(si[p], __dadd_rn(__dmul_rn(mr, im), __dmul_rn(mi, r)));
                }
            }
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int l = lane + 32 * p;
            if (l < m) {
                RX(l, k) = sr[p];
                IX(l, k) = si[p];
            }
        }
        __syncwarp();
    }
#undef RX
#undef IX
}

__device__ void hessenberg_split_exact(WarpWs &w, int m, int lane)
{
    if (m <= 32) hessenberg_split_exact_np<1>(w, m, lane);
    else if (m <= 64) hessenberg_split_exact_np<2>(w, m, lane);
    else if (m <= 96) hessenberg_split_exact_np<3>(w, m, lane);
    else hessenberg_split_exact_np<4>(w, m, lane);
}

// _charpoly_hessenberg!(C, H, m, n), src/hafnian.jl:454-492 (real), exact order.  Row k of C
// (k = 0..m) holds p_k; C[k*(n+1) + t] is the coefficient of lambda^(k-t).  Lane <-> t is fixed
// (t = lane + 32p, n <= 63), and each lane keeps its coefficients of row k in registers while the
// i loop updates them in the reference's order (i descending); the row is stored once at the end.
__device__ void charpoly_real_exact(WarpWs &w, int m, int n, int lane)
{
    const double *H = w.M;
    const int ld = w.ldm, cs = n + 1;
    double *C = w.C;
#define HX(i, j) H[(size_t)(j) * ld + (i)]
    for (int t = lane; t <= n; t += 32) C[t] = t == 0 ? 1.0 : 0.0;
    __syncwarp();
    for (int k = 1; k <= m; ++k) {
        const double hkk = HX(k - 1, k - 1);
        const int tmax = k < n ? k : n, prevmax = (k - 1) < n ? (k - 1) : n;
        const double *Cp = C + (size_t)(k - 1) * cs;
        double *Ck = C + (size_t)k * cs;
        double ck[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int t = lane + 32 * p;
            ck[p] = 0.0;
            if (t == 0) ck[p] = Cp[0];
            else if (t <= tmax) ck[p] = __dsub_rn(t <= prevmax ? Cp[t] : 0.0, __dmul_rn(hkk, Cp[t - 1]));
        }
        double beta = 1.0;
        const int ilo = 1 > k - n + 1 ? 1 : k - n + 1;
        for (int i = k - 1; i >= ilo; --i) {
            beta = __dmul_rn(beta, HX(i, i - 1));
            if (beta == 0.0) break;
            const double coef = __dmul_rn(HX(i - 1, k - 1), beta);
            const int d = k - i + 1;
            if (coef != 0.0) {
                const int tt = n < d + i - 1 ? n : d + i - 1;
                const double *Ci = C + (size_t)(i - 1) * cs;
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const int t = lane + 32 * p;
                    if (t >= d && t <= tt) ck[p] = __dsub_rn(ck[p], __dmul_rn(coef, Ci[t - d]));
                }
            }
        }
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int t = lane + 32 * p;
            if (t <= n) Ck[t] = ck[p];
        }
        __syncwarp();
    }
#undef HX
}

__device__ __forceinline__ cd c_mul_x(cd a, cd b) { return x_cmul(a, b); }
__device__ __forceinline__ cd c_sub_x(cd a, cd b) { return cd{__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)}; }

// Complex charpoly on the split storage (the band of Mr/Mi equals the copied-back M, :358-363);
// row k's coefficients in registers as in the real form.
__device__ void charpoly_cplx_exact(WarpWs &w, int m, int n, int lane)
{
    const int ld = w.ldm, cs = n + 1;
    cd *C = (cd *)w.C;
    auto H = [&](int i, int j) { return cd{w.M[(size_t)j * ld + i], w.Mi[(size_t)j * ld + i]}; };
    for (int t = lane; t <= n; t += 32) C[t] = t == 0 ? cd{1.0, 0.0} : cd{0.0, 0.0};
    __syncwarp();
    for (int k = 1; k <= m; ++k) {
        const cd hkk = H(k - 1, k - 1);
        const int tmax = k < n ? k : n, prevmax = (k - 1) < n ? (k - 1) : n;
        const cd *Cp = C + (size_t)(k - 1) * cs;
        cd *Ck = C + (size_t)k * cs;
        cd ck[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int t = lane + 32 * p;
            ck[p] = cd{0.0, 0.0};
            if (t == 0) ck[p] = Cp[0];
            else if (t <= tmax) ck[p] = c_sub_x(t <= prevmax ? Cp[t] : cd{0.0, 0.0}, c_mul_x(hkk, Cp[t - 1]));
        }
        cd beta{1.0, 0.0};
        const int ilo = 1 > k - n + 1 ? 1 : k - n + 1;
        for (int i = k - 1; i >= ilo; --i) {
            beta = c_mul_x(beta, H(i, i - 1));
            if (beta.re == 0.0 && beta.im == 0.0) break;
            const cd coef = c_mul_x(H(i - 1, k - 1), beta);
            const int d = k - i + 1;
            if (!(coef.re == 0.0 && coef.im == 0.0)) {
                const int tt = n < d + i - 1 ? n : d + i - 1;
                const cd *Ci = C + (size_t)(i - 1) * cs;
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const int t = lane + 32 * p;
                    if (t >= d && t <= tt) ck[p] = c_sub_x(ck[p], c_mul_x(coef, Ci[t - d]));
                }
            }
        }
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int t = lane + 32 * p;
            if (t <= n) Ck[t] = ck[p];
        }
        __syncwarp();
    }
}

// _inv_sqrt_det_coeff!(f, q, m, n), src/hafnian.jl:502-514, on lane 0.
__device__ double inv_sqrt_real_exact(const double *q, double *f, int m, int n)
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

__device__ cd inv_sqrt_cplx_exact(const cd *q, cd *f, int m, int n)
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
        const double dd2 = (double)(2 * t);
        f[t] = cd{__ddiv_rn(-s.re, dd2), __ddiv_rn(-s.im, dd2)};
    }
    return f[n];
}

// One instance's share of terms for this warp, exact order.  Returns the warp's double-double
// partial sums (re, im) on lane 0.
template <bool CPLX>
__device__ void sieve_warp_exact(const SieveArgs &a, const SieveInst &in, WarpWs &w, int wslot, int lane, dd &acc_re,
                                 dd &acc_im)
{
    const int E = in.E, n = in.n, glynn = in.glynn, lda = in.lda;
    const int *reps = a.reps + in.reps_off;
    const int mr1 = a.maxrep + 1;
    // Term j: decode, build, reduce, accumulate.
    auto term = [&](int64_t j) {
        // Mixed-radix decode, Glynn substitution, surviving edges (:542-580), on lane 0.
        int mE = 0;
        double prefac = 0.0;
        if (lane == 0) {
            int64_t num = j, edge_sum = 0;
            double bp = 1.0;
            for (int i = E - 1; i >= 0; --i) {
                const int r = reps[i];
                const int64_t b = r + 1;
                const int k = (int)(num % b);
                num /= b;
                w.kept[i] = k;
                edge_sum += k;
                bp = __dmul_rn(bp, a.binoms[r + k * mr1]);
            }
            for (int i = 0; i < E; ++i) {
                const int k = glynn ? 2 * w.kept[i] - reps[i] : w.kept[i];
                w.kept[i] = k;
                if (k != 0) w.idx[mE++] = i;
            }
            prefac = ((n - edge_sum) % 2 != 0) ? -bp : bp;
            if (glynn && w.kept[0] == 0) prefac = __ddiv_rn(prefac, 2.0);
            for (int q = 0; q < mE; ++q) {
                w.rows[q] = w.idx[q];
                w.rows[mE + q] = w.idx[q] + E;
            }
        }
        mE = __shfl_sync(0xffffffffu, mE, 0);
        prefac = __shfl_sync(0xffffffffu, prefac, 0);
        __syncwarp();
        const int m = 2 * mE;
        if (m == 0) {                   // empty submatrix contributes zero (:566-567)
            if (a.terms && lane == 0) {
                if (CPLX) {
                    a.terms[2 * j] = 0.0;
                    a.terms[2 * j + 1] = 0.0;
                } else {
                    a.terms[j] = 0.0;
                }
            }
            return;
        }
        if (m <= a.skip_le) return;   // evaluated by the fast kernels
        const int ld = w.ldm;
        // M = A_S X D (:582-593).
        if (!CPLX) {
            const double *Ax = (const double *)a.Ax + in.ax_off;
            for (int b = 0; b < mE; ++b) {
                const double kb = (double)w.kept[w.idx[b]];
                const int cb1 = w.idx[b] + E, cb2 = w.idx[b];
                for (int r = lane; r < m; r += 32) {
                    const int ra = w.rows[r];
                    w.M[(size_t)b * ld + r] = __dmul_rn(kb, Ax[(size_t)cb1 * lda + ra]);
                    w.M[(size_t)(mE + b) * ld + r] = __dmul_rn(kb, Ax[(size_t)cb2 * lda + ra]);
                }
            }
            __syncwarp();
            hessenberg_real_exact(w, m, lane);
            charpoly_real_exact(w, m, n, lane);
            if (lane == 0) {
                const double val = inv_sqrt_real_exact(w.C + (size_t)m * (n + 1), w.f, m, n);
                if (a.terms) a.terms[j] = __dmul_rn(prefac, val);
                else dd_add(acc_re, __dmul_rn(prefac, val));
            }
        } else {
            const cd *Ax = (const cd *)a.Ax + in.ax_off;
            for (int b = 0; b < mE; ++b) {
                const double kb = (double)w.kept[w.idx[b]];
                const int cb1 = w.idx[b] + E, cb2 = w.idx[b];
                for (int r = lane; r < m; r += 32) {
                    const int ra = w.rows[r];
                    const cd z1 = Ax[(size_t)cb1 * lda + ra], z2 = Ax[(size_t)cb2 * lda + ra];
                    w.M[(size_t)b * ld + r] = __dmul_rn(kb, z1.re);
                    w.Mi[(size_t)b * ld + r] = __dmul_rn(kb, z1.im);
                    w.M[(size_t)(mE + b) * ld + r] = __dmul_rn(kb, z2.re);
                    w.Mi[(size_t)(mE + b) * ld + r] = __dmul_rn(kb, z2.im);
                }
            }
            __syncwarp();
            hessenberg_split_exact(w, m, lane);
            charpoly_cplx_exact(w, m, n, lane);
            if (lane == 0) {
                const cd val = inv_sqrt_cplx_exact((const cd *)w.C + (size_t)m * (n + 1), (cd *)w.f, m, n);
                if (a.terms) {
                    a.terms[2 * j] = __dmul_rn(prefac, val.re);
                    a.terms[2 * j + 1] = __dmul_rn(prefac, val.im);
                } else {
                    dd_add(acc_re, __dmul_rn(prefac, val.re));
                    dd_add(acc_im, __dmul_rn(prefac, val.im));
                }
            }
        }
        __syncwarp();
    };
    if (in.subset) {
        // All multiplicities 1 under inclusion-exclusion: term j is the edge subset whose bit E-1-i
        // is edge i.  Each warp takes an equal share of every popcount level it evaluates (colex
        // unrank, then successors; bit i = edge i here, reversed into j), so that when only the
        // largest terms are left to this kernel they are spread evenly over the warps.
        const int k0 = a.skip_le > 0 ? a.skip_le / 2 + 1 : 0;
        const uint64_t W = (uint64_t)a.warps_per_inst;
        for (int k = k0; k <= E; ++k) {
            const uint64_t cnt = a.binom32[E * 65 + k];
            const uint64_t lo = (uint64_t)wslot * cnt / W, hi = ((uint64_t)wslot + 1) * cnt / W;
            if (lo >= hi) continue;
            uint32_t S = 0;
            {
                uint32_t R = (uint32_t)lo;
                int x = E - 1;
                for (int i = k; i >= 1; --i) {
                    while (a.binom32[x * 65 + i] > R) --x;
                    S |= 1u << x;
                    R -= a.binom32[x * 65 + i];
                    --x;
                }
            }
            for (uint64_t rk = lo; rk < hi; ++rk) {
                if (rk > lo) {
                    const uint32_t t = S | (S - 1);
                    S = (t + 1) | (((~t & (0u - ~t)) - 1) >> (__ffs((int)S)));
                }
                term((int64_t)(__brev(S) >> (32 - E)));
            }
        }
    } else {
        for (int64_t j = wslot; j < in.steps; j += a.warps_per_inst) term(j);
    }
}

template <bool CPLX>
__global__ void __launch_bounds__(256) sieve_exact_kernel(SieveArgs a, int warps_per_block)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    WarpWs w = carve(smem + (size_t)wib * ws_doubles(a.Emax, a.nmax, CPLX), a.Emax, a.nmax, CPLX);
    const int wslot = blockIdx.x * warps_per_block + wib;
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    if (wslot < a.warps_per_inst) sieve_warp_exact<CPLX>(a, in, w, wslot, lane, acc_re, acc_im);
    if (lane == 0 && wslot < a.warps_per_inst) {
        dd *out = a.partial + ((size_t)b * a.warps_per_inst + wslot) * 2;
        out[0] = acc_re;
        out[1] = acc_im;
    }
}

// Sums each instance's per-warp partials (one array per kernel that evaluated some of its terms) in a fixed tree, applies the Glynn rescaling 2^-(n-1) (:737) and writes the result.
// One block of 256 threads per instance.
constexpr int kReduceThreads = 512;

struct PartialSet {
    const dd *p[kMaxPartials];  // exact kernel, then the register-tile level launches
    int w[kMaxPartials];
};

template <bool CPLX>
__global__ void __launch_bounds__(kReduceThreads) sieve_reduce_kernel(PartialSet ps, const SieveInst *inst, void *out)
{
    __shared__ dd sre[kReduceThreads], sim[CPLX ? kReduceThreads : 1];
    const int b = blockIdx.x, t = threadIdx.x;
    dd r{0.0, 0.0}, i{0.0, 0.0};
    for (int a = 0; a < kMaxPartials; ++a) {
        if (!ps.p[a]) continue;
        const dd *p = ps.p[a] + (size_t)b * ps.w[a] * 2;
        for (int w = t; w < ps.w[a]; w += kReduceThreads) {
            dd_add(r, p[2 * w]);
            if (CPLX) dd_add(i, p[2 * w + 1]);
        }
    }
    sre[t] = r;
    if (CPLX) sim[t] = i;
    __syncthreads();
    for (int s = kReduceThreads / 2; s > 0; s >>= 1) {
        if (t < s) {
            dd_add(sre[t], sre[t + s]);
            if (CPLX) dd_add(sim[t], sim[t + s]);
        }
        __syncthreads();
    }
    if (t == 0) {
        const SieveInst in = inst[b];
        double hr, hi;
        if (in.E == 0) {
            hr = 1.0;  // E == 0: one(T) (:691)
            hi = 0.0;
        } else {
            hr = __dadd_rn(sre[0].hi, sre[0].lo);
            hi = CPLX ? __dadd_rn(sim[0].hi, sim[0].lo) : 0.0;
            if (in.glynn) {
                const double s = ldexp(1.0, -(in.n - 1));
                hr = __dmul_rn(hr, s);
                hi = __dmul_rn(hi, s);
            }
        }
        if (CPLX) ((cd *)out)[b] = cd{hr, hi};
        else ((double *)out)[b] = hr;
    }
}

// ---- host side ---------------------------------------------------------------------------------

static int64_t maxrep_of(const int64_t *reps, int64_t E)
{
    int64_t m = 0;
    for (int64_t i = 0; i < E; ++i) m = reps[i] > m ? reps[i] : m;
    return m;
}

static int64_t term_count(const int64_t *reps, int64_t E, int glynn)
{
    // The odometer's range: prod(r_i + 1), the leading digit clipped to (r_1 + 2) / 2 under Glynn
    // (the `total` of _sieve_variant_cost, src/hafnian.jl:865).
    int64_t steps = 1;
    for (int64_t i = 0; i < E; ++i) {
        int64_t f = (glynn && i == 0) ? (reps[i] + 2) / 2 : reps[i] + 1;
        if (f <= 0) return -1;
        if (steps > INT64_MAX / f) return -1;
        steps *= f;
    }
    return E == 0 ? 0 : steps;
}

static int64_t align256(int64_t x) { return (x + 255) & ~(int64_t)255; }

// Rounds of terms (the level's terms over the machine's warps in lockstep blocks) below which a
// level runs in blocks of four warps instead: complex and real tiles.
constexpr double kLockstepMinRoundsCplx = 8.0, kLockstepMinRoundsReal = 3.0;

int sieve_batch_run(int dtype, int prec, int64_t B, int64_t Emax, const void *dAx, const int64_t *E,
                    const int64_t *edge_reps, const int32_t *glynn, void *dout, cudaStream_t st,
                    const FixedScratch *fixed, double *terms, void *stage, size_t stage_cap)
{
    // terms: instead of summing, store every term of the single instance (exact kernel).
    if (terms && (B != 1 || prec != EGG_PREC_EXACT)) return fail(EGG_ERR_ARGUMENT, "term output needs one instance in exact mode");
    Context &c = ctx();
    const int num_sms = fixed ? fixed->num_sms : c.num_sms;
    const int cplx = dtype == EGG_C128;
    if (prec != EGG_PREC_EXACT && prec != EGG_PREC_FMA) return fail(EGG_ERR_ARGUMENT, "the sieve takes EGG_PREC_EXACT or EGG_PREC_FMA");
    if (B > 65535) return fail(EGG_ERR_ARGUMENT, "batch too large for one launch (max 65535)");
    std::vector<SieveInst> inst((size_t)B);
    std::vector<int> reps;
    std::vector<int64_t> strides;
    int maxrep = 0, nmax = 0;
    int64_t maxsteps = 0;
    int mmax_all = 0;  // the largest term size any instance can produce
    const int lda = (int)(2 * Emax);
    for (int64_t b = 0; b < B; ++b) {
        SieveInst &s = inst[(size_t)b];
        s.E = (int)E[b];
        s.glynn = glynn[b] ? 1 : 0;
        s.lda = lda > 0 ? lda : 1;
        s.ax_off = b * (int64_t)lda * lda;
        s.reps_off = (int64_t)reps.size();
        int64_t n = 0;
        for (int64_t i = 0; i < s.E; ++i) {
            int64_t r = edge_reps[b * Emax + i];
            if (r < 0 || r > 1000000) return fail(EGG_ERR_ARGUMENT, "edge multiplicities must be non-negative");
            reps.push_back((int)r);
            n += r;
            if (r > maxrep) maxrep = (int)r;
        }
        if (n > 63) return fail(EGG_ERR_TOO_LARGE, "the device sieve extracts coefficients up to lambda^63");
        s.n = (int)n;
        s.subset = (!s.glynn && s.E > 0 && s.E <= 32 && n == s.E && maxrep_of(edge_reps + b * Emax, s.E) == 1) ? 1 : 0;
        s.pattern = -1;
        nmax = s.n > nmax ? s.n : nmax;
        s.steps = term_count(edge_reps + b * Emax, s.E, s.glynn);
        if (s.steps < 0) return fail(EGG_ERR_TOO_LARGE, "the sieve's term count overflows Int64");
        maxsteps = s.steps > maxsteps ? s.steps : maxsteps;
        // mixed-radix place values, edge E-1 least significant
        std::vector<int64_t> pv((size_t)s.E);
        int64_t acc = 1;
        for (int64_t i = s.E - 1; i >= 0; --i) {
            pv[(size_t)i] = acc;
            int64_t r = edge_reps[b * Emax + i];
            acc *= (s.glynn && i == 0) ? (r + 2) / 2 : r + 1;
        }
        strides.insert(strides.end(), pv.begin(), pv.end());
        if (s.steps > 0) {
            mmax_all = 2 * s.E > mmax_all ? 2 * s.E : mmax_all;
        }
    }
    std::vector<double> binoms((size_t)(maxrep + 1) * (maxrep + 1), 0.0);
    for (int aa = 0; aa <= maxrep; ++aa) {
        double v = 1.0;  // C(aa, bb), exact for the small multiplicities used here
        for (int bb = 0; bb <= aa; ++bb) {
            binoms[(size_t)aa + (size_t)bb * (maxrep + 1)] = v;
            v = v * (double)(aa - bb) / (double)(bb + 1);
        }
    }
    const int Ews = (int)(Emax > 0 ? Emax : 1);

    // Which kernels run: each popcount level that some instance has terms in, on the register tiles
    // (orders n <= 31, one lane per coefficient) -- with fused multiply-adds, or for terms of up to
    // 32 rows in the reference's arithmetic -- and the shared-memory exact kernel for whatever
    // exceeds the tiles.
    const bool exact = prec == EGG_PREC_EXACT;
    const bool fast_ok = nmax <= 31;
    bool all_subset = true;
    for (const SieveInst &si : inst) all_subset = all_subset && si.subset;
    const int fast_hi = cplx ? 32 : (exact ? 32 : 48);

    // Term lists for the fast kernels: instances that share a multiplicity pattern (a batch of
    // hafnian_repeated(B, rpt) with one rpt) share one list per level of their terms' digits, so
    // that the level kernels deal the terms evenly instead of walking the whole odometer at every
    // level.  Only patterns of at least two instances, small ones (E <= 16 edges, digits below 16,
    // all lists within 2^22 terms), and not with caller-provided scratch, whose size must not depend
    // on this.
    std::vector<uint64_t> lists;
    std::vector<int64_t> list_off;
    const int list_stride = (int)Emax + 2;
    if (fast_ok && !fixed && B > 1) {
        constexpr int64_t kListTerms = (int64_t)1 << 22;
        auto list_key = [&](int64_t b, std::vector<int64_t> &key) -> bool {
            const SieveInst &si = inst[(size_t)b];
            const int64_t *er = edge_reps + b * Emax;
            if (si.subset || si.E == 0 || si.E > 16 || maxrep_of(er, si.E) > 15) return false;
            key.assign(er, er + si.E);
            key.push_back(si.glynn);
            return true;
        };
        // Only patterns that at least two instances share: a list costs a host walk of the odometer.
        std::map<std::vector<int64_t>, int> uses;
        std::vector<int64_t> key;
        for (int64_t b = 0; b < B; ++b)
            if (list_key(b, key)) ++uses[key];
        std::map<std::vector<int64_t>, int> pid;
        for (int64_t b = 0; b < B; ++b) {
            SieveInst &si = inst[(size_t)b];
            const int64_t *er = edge_reps + b * Emax;
            if (!list_key(b, key) || uses[key] < 2) continue;
            auto it = pid.find(key);
            if (it != pid.end()) {
                si.pattern = it->second;
                continue;
            }
            if ((int64_t)lists.size() + si.steps > kListTerms) continue;
            // Walk the odometer once (edge E-1 least significant, digit 0 clipped under Glynn).
            const int E = si.E;
            std::vector<int> d((size_t)E, 0), base((size_t)E), r((size_t)E);
            for (int i = 0; i < E; ++i) {
                r[(size_t)i] = (int)er[i];
                base[(size_t)i] = (si.glynn && i == 0) ? (r[(size_t)i] + 2) / 2 : r[(size_t)i] + 1;
            }
            std::vector<std::vector<uint64_t>> lvl((size_t)E + 1);
            for (int64_t j = 0; j < si.steps; ++j) {
                uint64_t word = 0;
                int k = 0;
                for (int i = 0; i < E; ++i) {
                    word |= (uint64_t)d[(size_t)i] << (4 * i);
                    const int kk = si.glynn ? 2 * d[(size_t)i] - r[(size_t)i] : d[(size_t)i];
                    k += kk != 0;
                }
                lvl[(size_t)k].push_back(word);
                for (int i = E - 1; i >= 0; --i) {
                    if (++d[(size_t)i] < base[(size_t)i]) break;
                    d[(size_t)i] = 0;
                }
            }
            const int p = (int)pid.size();
            pid[key] = p;
            list_off.resize((size_t)(p + 1) * list_stride, 0);
            for (int k = 0; k < list_stride; ++k) {
                list_off[(size_t)p * list_stride + k] = (int64_t)lists.size();
                if (k <= E) lists.insert(lists.end(), lvl[(size_t)k].begin(), lvl[(size_t)k].end());
            }
            si.pattern = p;
        }
    }
    bool all_balanced = true;  // every instance's terms dealt in equal shares (subsets or lists)
    for (const SieveInst &si : inst) all_balanced = all_balanced && (si.subset || si.pattern >= 0);
    const bool run_ex = !fast_ok || mmax_all > fast_hi || mmax_all == 0;
    const int skip_le = fast_ok ? fast_hi : 0;

    // Launch shapes.
    auto per_inst_blocks = [&](int wpb) {
        int64_t target = (int64_t)num_sms * 32;  // resident-warp budget across the machine
        int64_t per = (target + B - 1) / B;
        if (per > maxsteps) per = maxsteps;
        if (per < 1) per = 1;
        return (int)((per + wpb - 1) / wpb);
    };
    const size_t ex_per_warp = ws_doubles(Ews, nmax, cplx) * sizeof(double);
    int ex_wpb = (int)((200 * 1024) / ex_per_warp);
    if (ex_wpb > 8) ex_wpb = 8;
    if (run_ex && ex_wpb < 1) return fail(EGG_ERR_TOO_LARGE, "sieve workspace exceeds shared memory");
    int ex_bx = 0;
    if (run_ex && all_subset) {
        // Terms dealt as equal shares of each popcount level: one wave of resident blocks.
        int nb = 0;
        const void *ek = cplx ? (const void *)sieve_exact_kernel<true> : (const void *)sieve_exact_kernel<false>;
        int rc0 = smem_limit_at_least(ek, ex_wpb * ex_per_warp);
        if (!rc0) rc0 = blocks_per_sm(ek, ex_wpb * 32, ex_wpb * ex_per_warp, &nb);
        if (rc0) return rc0;
        int64_t per = ((int64_t)num_sms * (nb > 0 ? nb : 1) + B - 1) / B;
        const int64_t cap = (maxsteps + ex_wpb - 1) / ex_wpb;
        ex_bx = (int)(per < cap ? (per > 0 ? per : 1) : cap);
    } else if (run_ex) {
        ex_bx = per_inst_blocks(ex_wpb);
    }
    // The fast launches: one per popcount level with terms.  A level of distinct-row instances runs
    // as one wave of its resident blocks across the machine, shared among the instances (every
    // group of lanes gets the same share of the level's terms, so a second, partial wave would
    // leave most of the machine idle while it ran); odometer levels get about four waves.  A level
    // whose terms number at most two per resident term slot is latency-bound: it runs on a side
    // stream, overlapping the main stream's launches, as does the exact kernel when it only takes
    // the terms too large for the tiles.
    struct FastLaunch {
        int level, cw, bx;
        bool side, narrow;
    };
    std::vector<FastLaunch> fl;
    int64_t f_parts = 0;  // sum over launches of partials (one per block) per instance
    // One small distinct-row instance: all its terms in one launch (every nonzero edge subset on the
    // tile of its largest size) instead of a launch per popcount level, whose fixed costs would
    // outweigh its few terms.
    const bool fused = fast_ok && B == 1 && all_subset && inst[0].E >= 1 && inst[0].E <= kFusedMaxE;
    if (fused) {
        const int k = inst[0].E;
        const bool narrow = 2 * k <= 16;
        int cw = 0, bps = 0;
        int rc0 = cplx ? level_shape_cplx(nmax, k, narrow, exact, true, &cw, &bps)
                       : level_shape_real(nmax, k, narrow, exact, true, &cw, &bps);
        if (rc0) return rc0;
        if (bps < 1) return fail(EGG_ERR_TOO_LARGE, "sieve workspace exceeds shared memory");
        const int64_t terms_all = ((int64_t)1 << k) - 1, per_block = (int64_t)cw * (narrow ? 2 : 1);
        int64_t bx = (terms_all + per_block - 1) / per_block;
        if (bx > (int64_t)num_sms * bps) bx = (int64_t)num_sms * bps;
        fl.push_back(FastLaunch{k, cw, (int)bx, false, narrow});
        f_parts += bx;
    } else if (fast_ok) {
        // Terms per level over all instances: the `counts` recursion of the cost model
        // (src/hafnian.jl:855-884), per instance.
        const int kmax = (int)(Emax < fast_hi / 2 ? Emax : fast_hi / 2);
        std::vector<double> lvl((size_t)kmax + 1, 0.0);
        for (int64_t b = 0; b < B; ++b) {
            const SieveInst &si = inst[(size_t)b];
            std::vector<double> cnt((size_t)si.E + 1, 0.0);
            cnt[0] = 1.0;
            for (int i = 0; i < si.E; ++i) {
                const int64_t r = edge_reps[b * Emax + i];
                const double total = (double)(si.glynn ? (i == 0 ? (r + 2) / 2 : r + 1) : r + 1);
                const double nzero = si.glynn ? (r % 2 == 0 ? 1.0 : 0.0) : 1.0;
                for (int c = i + 1; c >= 1; --c) cnt[(size_t)c] = cnt[(size_t)c] * nzero + cnt[(size_t)c - 1] * (total - nzero);
                cnt[0] *= nzero;
            }
            for (int k = 1; k <= kmax && k <= si.E; ++k) lvl[(size_t)k] += cnt[(size_t)k];
        }
        // Tiles of up to 16 rows take two terms per warp when every odometer instance has at most 16
        // edges (one lane per digit); distinct-row instances need no digits.
        int64_t e_odo = 0, tot_steps = 0;
        for (const SieveInst &si : inst) tot_steps += si.steps;
        const int64_t avg_steps = B > 0 ? tot_steps / B : 0;
        for (const SieveInst &si : inst) e_odo = (!si.subset && si.E > e_odo) ? si.E : e_odo;
        for (int k = 1; k <= kmax; ++k) {
            if (lvl[(size_t)k] <= 0.0) continue;
            const bool narrow = 2 * k <= 16 && e_odo <= 16;
            int cw = 0, bps = 0;
            int rc0 = cplx ? level_shape_cplx(nmax, k, narrow, exact, false, &cw, &bps)
                           : level_shape_real(nmax, k, narrow, exact, false, &cw, &bps);
            if (rc0) return rc0;
            // A lockstep shape (one block of all an SM's warps) pays off over many rounds of terms;
            // a level with fewer runs in blocks of four warps, several per SM, as the other shapes
            // do.  The complex N = 40 sieve took 30.77 -> 29.87 ms with its large levels in
            // lockstep (at N = 24 and 32, whose levels have few rounds, lockstep blocks were 10 %
            // and 3.5 % slower); the real N = 32 sieve 0.686 -> 0.656 ms with its levels of under
            // three rounds in four-warp blocks (N = 40 unchanged; under eight rounds, 1 % slower).
            const double min_rounds = cplx ? kLockstepMinRoundsCplx : kLockstepMinRoundsReal;
            if (cw > 4 && lvl[(size_t)k] < min_rounds * (double)num_sms * cw) {
                bps = cw / 4;
                cw = 4;
            }
            if (bps < 1 || (size_t)cw * (narrow ? 2 : 1) * level_ws_bytes(nmax, cplx, k, exact) > 220 * 1024)
                return fail(EGG_ERR_TOO_LARGE, "sieve workspace exceeds shared memory");
            // Distinct-row levels deal equal shares: one wave.  Odometer runs are only balanced on
            // average and instances differ in size, so those levels get several waves of blocks for
            // the block scheduler to even out: four for long odometers, two for short ones (a
            // batch of 1,458-term instances ran 6 % faster on two, one of 90 k-term instances 23 %
            // faster on four), where each block's fixed costs weigh more.
            const int64_t waves = all_subset ? 1 : (avg_steps >= 16384 ? 4 : 2);
            int64_t per = ((int64_t)num_sms * bps * waves + B - 1) / B;
            if (all_balanced && B > 1) {
                // Equal shares within each instance: the only loss is a last, partial wave of
                // blocks, so take the fewest blocks per instance whose waves end at least 90 % full.
                const double res = (double)num_sms * bps;
                int64_t best = 1;
                double best_eff = 0.0;
                for (int64_t p = 1; p <= 8; ++p) {
                    const double w = (double)(B * p) / res, eff = w / std::ceil(w);
                    if (eff > best_eff + 1e-9) {
                        best = p;
                        best_eff = eff;
                    }
                    if (eff >= 0.9) {
                        best = p;
                        break;
                    }
                }
                per = best;
            }
            const int64_t cap = (maxsteps + cw - 1) / cw;  // no more warps than terms
            if (per > cap) per = cap;
            if (per < 1) per = 1;
            const double slots = (double)num_sms * bps * cw * (narrow ? 2 : 1);  // terms in flight
            fl.push_back(FastLaunch{k, cw, (int)per, lvl[(size_t)k] <= 2.0 * slots, narrow});
            f_parts += per;
        }
    }
    if ((int)fl.size() + 1 > kMaxPartials) return fail(EGG_ERR_TOO_LARGE, "too many sieve launches");

    // Device staging: instance table, reps, strides, binoms, partials -- one scratch allocation.
    int64_t off = 0;
    const int64_t off_inst = off; off = align256(off + (int64_t)(inst.size() * sizeof(SieveInst)));
    const int64_t off_reps = off; off = align256(off + (int64_t)((reps.size() + 1) * sizeof(int)));
    const int64_t off_str = off; off = align256(off + (int64_t)((strides.size() + 1) * sizeof(int64_t)));
    const int64_t off_bin = off; off = align256(off + (int64_t)(binoms.size() * sizeof(double)));
    const int64_t off_done = off; off = align256(off + (int64_t)sizeof(unsigned));  // zero in the image
    const int64_t off_loff = off; off = align256(off + (int64_t)((list_off.size() + 1) * sizeof(int64_t)));
    const int64_t off_lst = off; off = align256(off + (int64_t)((lists.size() + 1) * sizeof(uint64_t)));
    const int64_t off_pex = off; off = align256(off + (run_ex ? B * ex_bx * ex_wpb * 2 * (int64_t)sizeof(dd) : 0));
    const int64_t off_pf = off; off = align256(off + B * f_parts * 2 * (int64_t)sizeof(dd));
    char *base;
    int rc;
    if (fixed) {
        if ((size_t)off + 256 > fixed->bytes)
            return fail(EGG_ERR_TOO_LARGE, "this sieve needs " + std::to_string((size_t)off + 256) +
                                               " bytes of scratch; the fixed scratch region holds " +
                                               std::to_string(fixed->bytes));
        base = (char *)fixed->ptr;
    } else {
        rc = ensure_buf(c.scratch[5], (size_t)off + 256);
        if (rc) return rc;
        base = (char *)c.scratch[5].ptr;
    }
    {
        // The instance table, reps, strides, binomials and term lists in their device layout, sent
        // as one copy (each copy from pageable memory has a fixed staging cost).
        // A synchronous caller's page-locked stage takes the image when it fits.
        const size_t img = (size_t)(off_lst + (int64_t)(lists.size() * sizeof(uint64_t)));
        std::vector<char> hv;
        char *h;
        if (stage && img <= stage_cap) {
            h = (char *)stage;
            std::memset(h, 0, img);
        } else {
            hv.assign(img, 0);
            h = hv.data();
        }
        std::memcpy(h + off_inst, inst.data(), inst.size() * sizeof(SieveInst));
        if (!reps.empty()) std::memcpy(h + off_reps, reps.data(), reps.size() * sizeof(int));
        if (!strides.empty()) std::memcpy(h + off_str, strides.data(), strides.size() * sizeof(int64_t));
        std::memcpy(h + off_bin, binoms.data(), binoms.size() * sizeof(double));
        if (!list_off.empty()) std::memcpy(h + off_loff, list_off.data(), list_off.size() * sizeof(int64_t));
        if (!lists.empty()) std::memcpy(h + off_lst, lists.data(), lists.size() * sizeof(uint64_t));
        EGG_CUDA_TRY(cudaMemcpyAsync(base, h, img, cudaMemcpyHostToDevice, st));
    }
    SieveArgs a;
    a.Ax = dAx;
    a.reps = (const int *)(base + off_reps);
    a.binoms = (const double *)(base + off_bin);
    a.binom32 = binom32_device(&rc);
    if (!a.binom32) return rc;
    a.inst = (const SieveInst *)(base + off_inst);
    a.lists = (const uint64_t *)(base + off_lst);
    a.list_off = (const int64_t *)(base + off_loff);
    a.list_stride = list_stride;
    a.fused_out = fused ? dout : nullptr;
    a.done = (unsigned *)(base + off_done);
    a.maxrep = maxrep;
    a.Emax = Ews;
    a.nmax = nmax;
    a.block_warps = 0;
    a.skip_le = skip_le;
    a.terms = terms;
    if (terms) {
        // Terms with no surviving edge are zero (src/hafnian.jl:566-567); every other term is
        // written by the kernel that evaluates it.
        EGG_CUDA_TRY(cudaMemsetAsync(terms, 0, (size_t)inst[0].steps * (cplx ? 16 : 8), st));
    }
    PartialSet ps;
    for (int k = 0; k < kMaxPartials; ++k) {
        ps.p[k] = nullptr;
        ps.w[k] = 0;
    }
    // Side launches go round robin over the library's side streams, the exact kernel first.  With
    // caller-provided scratch (the entry point that allocates nothing) everything stays on the
    // caller's stream: that path uses nothing of the library's context.
    const bool side_ok = fixed == nullptr;
    const bool ex_side = side_ok && run_ex && fast_ok;  // the exact kernel only takes the terms too large for the tiles
    int nside = ex_side ? 1 : 0;
    for (const FastLaunch &L : fl) nside += (side_ok && L.side) ? 1 : 0;
    const int nstreams = nside < Context::kSideStreams ? nside : Context::kSideStreams;
    if (nstreams > 0) {
        EGG_CUDA_TRY(cudaEventRecord(c.fork_ev, st));
        for (int i = 0; i < nstreams; ++i) EGG_CUDA_TRY(cudaStreamWaitEvent(c.side[i], c.fork_ev, 0));
    }
    int next_side = 0;
    if (run_ex) {
        // First, so that on the side stream its long terms start at once.
        SieveArgs ae = a;
        ae.warps_per_inst = ex_bx * ex_wpb;
        ae.partial = (dd *)(base + off_pex);
        const size_t smem = (size_t)ex_wpb * ex_per_warp;
        const dim3 grid((unsigned)ex_bx, (unsigned)B);
        cudaStream_t es = st;
        if (ex_side) es = c.side[next_side++ % Context::kSideStreams];
        rc = smem_limit_at_least(cplx ? (const void *)sieve_exact_kernel<true> : (const void *)sieve_exact_kernel<false>, smem);
        if (rc) return rc;
        if (cplx) sieve_exact_kernel<true><<<grid, ex_wpb * 32, smem, es>>>(ae, ex_wpb);
        else sieve_exact_kernel<false><<<grid, ex_wpb * 32, smem, es>>>(ae, ex_wpb);
        count_launch();
        EGG_CUDA_TRY(cudaGetLastError());
        ps.p[0] = ae.partial;
        ps.w[0] = ae.warps_per_inst;
    }
    {
        a.partial = nullptr;
        int slot = 1;
        dd *part = (dd *)(base + off_pf);
        const int64_t *dstr = (const int64_t *)(base + off_str);
        for (const FastLaunch &L : fl) {
            a.warps_per_inst = L.bx * L.cw;
            a.block_warps = fused ? 0 : L.cw;
            cudaStream_t ls = st;
            if (side_ok && L.side) ls = c.side[next_side++ % Context::kSideStreams];
            if (fused)
                rc = cplx ? level_launch_all_cplx(a, L.level, L.narrow, exact, part, L.bx, ls)
                          : level_launch_all_real(a, L.level, L.narrow, exact, part, L.bx, ls);
            else
                rc = cplx ? level_launch_cplx(a, dstr, (int)B, L.level, L.narrow, exact, part, L.bx, ls)
                          : level_launch_real(a, dstr, (int)B, L.level, L.narrow, exact, part, L.bx, ls);
            if (rc) return rc;
            ps.p[slot] = part;
            ps.w[slot] = L.bx;
            part += (size_t)B * L.bx * 2;
            ++slot;
        }
    }
    for (int i = 0; i < nstreams; ++i) {
        EGG_CUDA_TRY(cudaEventRecord(c.join_ev[i], c.side[i]));
        EGG_CUDA_TRY(cudaStreamWaitEvent(st, c.join_ev[i], 0));
    }
    if (terms || fused) {
        // (The all-levels launch sums its own partials.)
        EGG_CUDA_TRY(cudaGetLastError());
        return EGG_OK;
    }
    if (cplx) sieve_reduce_kernel<true><<<(unsigned)B, kReduceThreads, 0, st>>>(ps, a.inst, dout);
    else sieve_reduce_kernel<false><<<(unsigned)B, kReduceThreads, 0, st>>>(ps, a.inst, dout);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

int sieve_run(int dtype, int prec, const void *dAx, int64_t E, const int64_t *edge_reps, int glynn, void *dout,
              cudaStream_t st, void *stage, size_t stage_cap)
{
    int32_t g = glynn ? 1 : 0;
    int64_t e = E;
    std::vector<int64_t> reps(edge_reps, edge_reps + E);
    if (reps.empty()) reps.push_back(0);
    return sieve_batch_run(dtype, prec, 1, E, dAx, &e, reps.data(), &g, dout, st, nullptr, nullptr, stage, stage_cap);
}

// ---- the reference's summation ------------------------------------------------------------------

// Chunk c of [0, steps) (c = 0..nchunks-1, the reference's div((c-1) steps, nchunks) bounds, 0-based):
// a plain FP64 sum in term order, starting from zero.
template <bool CPLX>
__global__ void sieve_chunk_sum_kernel(const double *__restrict__ terms, int64_t steps, int64_t nchunks, double *__restrict__ part)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const int64_t lo = (c * steps) / nchunks, hi = ((c + 1) * steps) / nchunks;
    double hr = 0.0, hi_ = 0.0;
    for (int64_t j = lo; j < hi; ++j) {
        if (CPLX) {
            hr = __dadd_rn(hr, terms[2 * j]);
            hi_ = __dadd_rn(hi_, terms[2 * j + 1]);
        } else {
            hr = __dadd_rn(hr, terms[j]);
        }
    }
    part[2 * c] = hr;
    part[2 * c + 1] = hi_;
}

// The chunk sums left to right (Julia's sum over a short array), then Glynn's 2^-(n-1).
template <bool CPLX>
__global__ void sieve_chunk_fold_kernel(const double *__restrict__ part, int64_t nchunks, int glynn, int n, double *__restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double hr = part[0], hi_ = part[1];
    for (int64_t c = 1; c < nchunks; ++c) {
        hr = __dadd_rn(hr, part[2 * c]);
        hi_ = __dadd_rn(hi_, part[2 * c + 1]);
    }
    if (glynn) {
        double s = 1.0;  // R(0.5)^(n-1), exact
        for (int i = 0; i < n - 1; ++i) s = __dmul_rn(s, 0.5);
        hr = __dmul_rn(hr, s);
        hi_ = __dmul_rn(hi_, s);
    }
    out[0] = hr;
    if (CPLX) out[1] = hi_;
}

int sieve_reference_sum_run(int dtype, const void *dAx, int64_t E, const int64_t *edge_reps, int glynn, int64_t nchunks,
                            void *dout, cudaStream_t st)
{
    const int cplx = dtype == EGG_C128;
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (nchunks < 1) return fail(EGG_ERR_ARGUMENT, "nchunks must be >= 1");
    std::vector<int64_t> reps(edge_reps, edge_reps + E);
    if (reps.empty()) reps.push_back(0);
    const int64_t steps = term_count(reps.data(), E, glynn);
    if (steps < 0) return fail(EGG_ERR_TOO_LARGE, "the sieve's term count overflows Int64");
    if (steps == 0) {  // no edges: the hafnian of the empty matrix
        const double one[2] = {1.0, 0.0};
        EGG_CUDA_TRY(cudaMemcpyAsync(dout, one, cplx ? 16 : 8, cudaMemcpyHostToDevice, st));
        return EGG_OK;
    }
    if (steps > ((int64_t)1 << 28))
        return fail(EGG_ERR_TOO_LARGE, "the reference-order sum keeps every term; " + std::to_string(steps) +
                                           " terms exceed its limit of 2^28");
    if (nchunks > steps) nchunks = steps;
    int n = 0;
    for (int64_t i = 0; i < E; ++i) n += (int)edge_reps[i];
    Context &c = ctx();
    const size_t tbytes = (size_t)steps * (cplx ? 16 : 8), pbytes = (size_t)nchunks * 16;
    int rc = ensure_buf(c.scratch[8], tbytes + pbytes + 256);
    if (rc) return rc;
    double *terms = (double *)c.scratch[8].ptr;
    double *part = (double *)((char *)c.scratch[8].ptr + ((tbytes + 255) / 256) * 256);
    int32_t g = glynn ? 1 : 0;
    int64_t e = E;
    rc = sieve_batch_run(dtype, EGG_PREC_EXACT, 1, E, dAx, &e, reps.data(), &g, nullptr, st, nullptr, terms);
    if (rc) return rc;
    const unsigned blocks = (unsigned)((nchunks + 255) / 256);
    if (cplx) {
        sieve_chunk_sum_kernel<true><<<blocks, 256, 0, st>>>(terms, steps, nchunks, part);
        sieve_chunk_fold_kernel<true><<<1, 32, 0, st>>>(part, nchunks, glynn, n, (double *)dout);
    } else {
        sieve_chunk_sum_kernel<false><<<blocks, 256, 0, st>>>(terms, steps, nchunks, part);
        sieve_chunk_fold_kernel<false><<<1, 32, 0, st>>>(part, nchunks, glynn, n, (double *)dout);
    }
    count_launch(2);
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

}  // namespace egg
