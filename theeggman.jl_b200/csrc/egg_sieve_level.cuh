// egg_sieve_level.cuh -- the popcount-level kernels of the register-resident sieve.
//
// With every multiplicity 1 under inclusion-exclusion (distinct rows: hafnian(A; method=:sieve)'s
// default variant, src/hafnian.jl:1139-1146), term j is the subset of edges whose digit is 1 and
// its size is m = 2k for a k-subset.  One kernel per popcount level k evaluates exactly the
// k-subsets, on a register tile of exactly m columns: no slot, step or La Budde order is spent on
// sizes the level does not have.  Every warp takes an equal share of the level (one colex unrank,
// then Gosper successors), so the level runs as one balanced wave.  Each block writes one partial
// (re, im) per instance: its warps' double-double sums added in a fixed order.
#pragma once
#include "egg_sieve_fast.cuh"

namespace egg {

// 128-thread blocks; resident blocks per SM from the tile's register need (65536 / (128 * blocks)
// registers per thread): a real tile holds m doubles per row, a complex one 2m.
template <bool CPLX, int K>
struct LevelShape {
    static constexpr int MW = 2 * K;
    static constexpr int threads = 128;
    static constexpr int min_blocks =
        CPLX ? (MW <= 8 ? 6 : (MW <= 10 ? 5 : (MW <= 16 ? 4 : (MW <= 24 ? 3 : 2))))
             : (MW <= 8 ? 8 : (MW <= 12 ? 7 : (MW <= 18 ? 6 : (MW <= 26 ? 5 : (MW <= 32 ? 4 : 2)))));
};

template <bool CPLX, int K>
__global__ void __launch_bounds__(LevelShape<CPLX, K>::threads, LevelShape<CPLX, K>::min_blocks)
    sieve_level_kernel(SieveArgs a, dd *partial)
{
    constexpr int MW = 2 * K;
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.y;
    const SieveInst in = a.inst[b];
    const int E = in.E, n = in.n;
    const FastWs w = fast_carve(smem + (size_t)wib * fast_ws_doubles(a.nmax, CPLX, MW), a.nmax, CPLX, MW);
    if constexpr (MW > 32) {
        // The La Budde table's entries left of column 0 must read as zero; nothing ever writes them.
        for (int i = lane; i < (MW + 1) * (MW + 1); i += 32) w.C[i] = 0.0;
        __syncwarp();
    }
    const int wslot = blockIdx.x * cw + wib;
    const uint64_t W = (uint64_t)a.warps_per_inst;
    dd acc_re{0.0, 0.0}, acc_im{0.0, 0.0};
    if (in.subset && K <= E) {
        const uint64_t cnt = c_binom[E * 33 + K];
        const uint64_t lo = (uint64_t)wslot * cnt / W, hi = ((uint64_t)wslot + 1) * cnt / W;
        const double prefac = ((n - K) & 1) ? -1.0 : 1.0;  // (-1)^(n - k), every binomial factor 1
        uint32_t S = lo < hi ? subset_unrank(E, K, (uint32_t)lo) : 0u;
        for (uint64_t rk = lo; rk < hi; ++rk) {
            if (rk > lo) S = subset_next(S);
            if (lane < E && ((S >> lane) & 1u)) {
                const int pos = __popc(S & ((1u << lane) - 1u));
                w.eidx[pos] = lane;
                w.kval[pos] = 1.0;
            }
            __syncwarp();
            if constexpr (!CPLX) {
                const double val = term_real<MW, (MW > 32 ? 2 : 1)>((const double *)a.Ax + in.ax_off, in.lda, E, K, n, w,
                                                                    lane);
                if (lane == 0) dd_add(acc_re, prefac * val);
            } else {
                const cd val = term_cplx<MW>((const cd *)a.Ax + in.ax_off, in.lda, E, K, n, w, lane);
                if (lane == 0) {
                    dd_add(acc_re, prefac * val.re);
                    dd_add(acc_im, prefac * val.im);
                }
            }
            __syncwarp();
        }
    }
    // The block's warps summed in a fixed order: one partial per block.
    __shared__ dd red[2 * cw];
    if (lane == 0) {
        red[2 * wib] = acc_re;
        red[2 * wib + 1] = acc_im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dd r = red[0], i = red[1];
#pragma unroll
        for (int q = 1; q < cw; ++q) {
            dd_add(r, red[2 * q]);
            dd_add(i, red[2 * q + 1]);
        }
        dd *out = partial + ((size_t)b * gridDim.x + blockIdx.x) * 2;
        out[0] = r;
        out[1] = i;
    }
}

template <bool CPLX, int K>
static int level_launch_k(const SieveArgs &a, int B, dd *partial, int blocks_x, cudaStream_t st)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * fast_ws_doubles(a.nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K>;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3((unsigned)blocks_x, (unsigned)B), cw * 32, smem, st>>>(a, partial);
    count_launch();
    EGG_CUDA_TRY(cudaGetLastError());
    return EGG_OK;
}

template <bool CPLX, int K>
static int level_shape_k(int nmax, int *warps_per_block, int *blocks_per_sm)
{
    constexpr int cw = LevelShape<CPLX, K>::threads / 32;
    const size_t smem = (size_t)cw * fast_ws_doubles(nmax, CPLX, 2 * K) * sizeof(double);
    auto k = sieve_level_kernel<CPLX, K>;
    EGG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    EGG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, cw * 32, smem));
    *warps_per_block = cw;
    *blocks_per_sm = nb;
    return EGG_OK;
}

}  // namespace egg

// Case K of a switch over levels: launch or shape the level-K kernel of the given variant.
#define EGG_LEVEL_CASES(CPLX, X)                                                                   \
    X(CPLX, 1) X(CPLX, 2) X(CPLX, 3) X(CPLX, 4) X(CPLX, 5) X(CPLX, 6) X(CPLX, 7) X(CPLX, 8) X(CPLX, 9) \
    X(CPLX, 10) X(CPLX, 11) X(CPLX, 12) X(CPLX, 13) X(CPLX, 14) X(CPLX, 15) X(CPLX, 16)
#define EGG_LEVEL_CASES_HI(CPLX, X)                                                                 \
    X(CPLX, 17) X(CPLX, 18) X(CPLX, 19) X(CPLX, 20) X(CPLX, 21) X(CPLX, 22) X(CPLX, 23) X(CPLX, 24)
