// egg_gridbar.cuh -- a grid-wide barrier with a bounded wait, for cooperative launches.
//
// A cooperative launch places every block of the grid at once, so every block reaches every
// barrier and no wait is long.  Each wait is still bounded: a block that has waited longer than
// `wait_ns` (read from the GPU's global nanosecond timer) records the fact in *flag and goes on,
// and once *flag is set every later barrier of the launch returns at once.  The launch therefore
// always ends; its results are then invalid and the host reports EGG_ERR_TIMEOUT.
//
// bar[0] counts arrivals over the whole launch and bar[1] holds the number of the last barrier
// that every block has reached; both start at zero.  `epoch` is the calling block's count of
// barriers passed (kept by thread 0).
#pragma once

#include "egg_internal.cuh"

namespace egg {

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void grid_barrier(unsigned *bar, unsigned nblocks, unsigned &epoch, int *flag,
                                             unsigned long long wait_ns)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        ++epoch;
        __threadfence();  // this block's writes before its arrival
        const unsigned arrived = atomicAdd(&bar[0], 1u) + 1u;
        if (arrived == epoch * nblocks) {
            atomicExch(&bar[1], epoch);
        } else {
            const unsigned long long t0 = global_ns();
            while (*(volatile unsigned *)&bar[1] < epoch) {
                if (*(volatile int *)flag) break;
                if (global_ns() - t0 > wait_ns) {
                    atomicExch(flag, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();  // the other blocks' writes before this block's next reads
    }
    __syncthreads();
}

}  // namespace egg
