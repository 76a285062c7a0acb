// egg_sieve_fast.cu -- the size-class kernels of the register-resident sieve (egg_sieve_fast.cuh):
// each evaluates the terms of one range of sizes, for any multiplicities.
#include "egg_sieve_fast.cuh"

namespace egg {

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
    if constexpr (MHI > 32) {
        for (int i = lane; i < (MHI + 1) * (MHI + 1); i += 32) w.C[i] = 0.0;
        __syncwarp();
    }
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
    // One term: the surviving edges are compacted into w.eidx / w.kval (mE of them) by the caller.
    auto eval_term = [&](int mE, double prefac) {
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
    };
    if (in.subset) {
        // All multiplicities 1 under inclusion-exclusion: term j is the edge subset with bits j (edge
        // E-1 least significant; here bit i is edge i, the same set of terms), its sign (-1)^(n-k).
        // This class's terms are the k-subsets with MLO < 2k <= MHI.  Every warp takes an equal
        // share of every popcount level -- one colex unrank, then successors -- so all warps do the
        // same work whatever the class.
        const int klo = MLO / 2 + 1, khi = MHI / 2 < E ? MHI / 2 : E;
        for (int k = klo; k <= khi; ++k) {
            const uint64_t cnt = c_binom[E * 33 + k];
            const uint64_t lo = (uint64_t)wslot * cnt / (uint64_t)W, hi = ((uint64_t)wslot + 1) * cnt / (uint64_t)W;
            if (lo >= hi) continue;
            const double prefac = ((n - k) & 1) ? -1.0 : 1.0;
            uint32_t S = subset_unrank(E, k, (uint32_t)lo);
            for (uint64_t rk = lo; rk < hi; ++rk) {
                if (rk > lo) S = subset_next(S);
                if (lane < E && ((S >> lane) & 1u)) {
                    const int pos = __popc(S & ((1u << lane) - 1u));
                    w.eidx[pos] = lane;
                    w.kval[pos] = 1.0;
                }
                __syncwarp();
                eval_term(k, prefac);
                __syncwarp();
            }
        }
    } else {
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
                eval_term(mE, prefac);
                __syncwarp();
            }
        }
    }
    if (lane == 0) {
        dd *out = partial + ((size_t)b * W + wslot) * 2;
        out[0] = acc_re;
        out[1] = acc_im;
    }
}

size_t fast_ws_bytes(int nmax, int cplx, int mhi) { return fast_ws_doubles(nmax, cplx, mhi) * sizeof(double); }

size_t fast_smem_bytes(int nmax, int cplx, int cls, int warps)
{
    return (size_t)warps * fast_ws_doubles(nmax, cplx, kFastClasses[cls][1]) * sizeof(double);
}

template <bool CPLX, int MLO, int MHI>
static int launch_one(const SieveArgs &a, const int64_t *strides, dim3 grid, int cls, dd *partial, cudaStream_t st)
{
    constexpr int cw = SizeClass<CPLX, MHI>::threads / 32;
    const size_t smem = fast_smem_bytes(a.nmax, CPLX, cls, cw);
    auto k = sieve_fast_kernel<CPLX, MLO, MHI>;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, cw * 32, smem, st>>>(a, strides, cw, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int MLO, int MHI>
static int shape_one(int nmax, int cls, int *warps_per_block, int *blocks_per_sm)
{
    constexpr int cw = SizeClass<CPLX, MHI>::threads / 32;
    const size_t smem = fast_smem_bytes(nmax, CPLX, cls, cw);
    auto k = sieve_fast_kernel<CPLX, MLO, MHI>;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    EGG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, cw * 32, smem));
    *warps_per_block = cw;
    *blocks_per_sm = nb;
    return EGG_OK;
}

const int kFastClasses[][2] = {{0, 8}, {8, 16}, {16, 24}, {24, 32}, {32, 40}, {40, 48}};

int launch_fast(const SieveArgs &a, const int64_t *strides, int B, int cplx, int cls, dd *partial, int blocks_x,
                cudaStream_t st)
{
    int rc = upload_fast_tables_once(st);
    if (rc) return rc;
    dim3 grid((unsigned)blocks_x, (unsigned)B);
    if (cplx) {
        switch (cls) {
        case 0: return launch_one<true, 0, 8>(a, strides, grid, cls, partial, st);
        case 1: return launch_one<true, 8, 16>(a, strides, grid, cls, partial, st);
        case 2: return launch_one<true, 16, 24>(a, strides, grid, cls, partial, st);
        case 3: return launch_one<true, 24, 32>(a, strides, grid, cls, partial, st);
        }
    } else {
        switch (cls) {
        case 0: return launch_one<false, 0, 8>(a, strides, grid, cls, partial, st);
        case 1: return launch_one<false, 8, 16>(a, strides, grid, cls, partial, st);
        case 2: return launch_one<false, 16, 24>(a, strides, grid, cls, partial, st);
        case 3: return launch_one<false, 24, 32>(a, strides, grid, cls, partial, st);
        case 4: return launch_one<false, 32, 40>(a, strides, grid, cls, partial, st);
        case 5: return launch_one<false, 40, 48>(a, strides, grid, cls, partial, st);
        }
    }
    return fail(EGG_ERR_ARGUMENT, "no such sieve size class");
}

int fast_class_shape(int nmax, int cplx, int cls, int *warps_per_block, int *blocks_per_sm)
{
    // Occupancy depends only on the class (its block size, registers and per-warp scratch).
    static int cache[2][kFastClassesReal][2];
    int *c = cache[cplx ? 1 : 0][cls];
    if (c[1] > 0) {
        *warps_per_block = c[0];
        *blocks_per_sm = c[1];
        return EGG_OK;
    }
    int rc = fail(EGG_ERR_ARGUMENT, "no such sieve size class");
    if (cplx) {
        switch (cls) {
        case 0: rc = shape_one<true, 0, 8>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 1: rc = shape_one<true, 8, 16>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 2: rc = shape_one<true, 16, 24>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 3: rc = shape_one<true, 24, 32>(nmax, cls, warps_per_block, blocks_per_sm); break;
        }
    } else {
        switch (cls) {
        case 0: rc = shape_one<false, 0, 8>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 1: rc = shape_one<false, 8, 16>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 2: rc = shape_one<false, 16, 24>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 3: rc = shape_one<false, 24, 32>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 4: rc = shape_one<false, 32, 40>(nmax, cls, warps_per_block, blocks_per_sm); break;
        case 5: rc = shape_one<false, 40, 48>(nmax, cls, warps_per_block, blocks_per_sm); break;
        }
    }
    if (rc) return rc;
    c[0] = *warps_per_block;
    c[1] = *blocks_per_sm;
    return EGG_OK;
}

}  // namespace egg
