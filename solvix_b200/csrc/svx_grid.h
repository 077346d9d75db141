// svx_grid.h - the bounded grid-wide barrier of the cooperative kernels
// (the persistent PCG kernels, the direct path's substitution kernel).
// Device code: included by the .cu units only.
#ifndef SVX_GRID_H
#define SVX_GRID_H
#ifdef __CUDACC__

#include "svx_internal.h"

namespace svx {

// polls of a grid barrier before it gives up (about a second)
constexpr long long BARRIER_SPIN_LIMIT = 1LL << 25;
// back-off between two polls of a grid barrier's arrival count
#ifndef SVX_BARRIER_SLEEP_NS
#define SVX_BARRIER_SLEEP_NS 32
#endif

// Bounded grid-wide barrier (all blocks co-resident: cooperative launch).
// gb->count only grows during a launch (the host zeroes it before each
// launch); every block keeps its own running target, nblocks more per
// barrier.  After bar.sync, thread 0 arrives with a gpu-scope release add
// (cumulative over the block's writes ordered before it by the bar.sync)
// and polls with acquire loads until the count reaches the target; the
// closing bar.sync passes that on to the block.  A block that polls
// spin_limit times raises gb->error and returns false, and so does a block
// that finds the flag raised by another while it waits.
__device__ __forceinline__ void barrier_arrive(unsigned int* p) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}
__device__ __forceinline__ unsigned int barrier_count(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool grid_sync(GridBarrier* gb, unsigned int nblocks,
                                          unsigned int& target,
                                          long long spin_limit = BARRIER_SPIN_LIMIT) {
    __shared__ int ok;
    target += nblocks;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        barrier_arrive(&gb->count);
        long long spins = 0;
        while (barrier_count(&gb->count) < target) {
            if (++spins > spin_limit) {
                atomicExch(&gb->error, 1);
                good = 0;
                break;
            }
            if ((spins & 255) == 0 && *((volatile int*)&gb->error) != 0) {
                good = 0;
                break;
            }
#if SVX_BARRIER_SLEEP_NS > 0
            __nanosleep(SVX_BARRIER_SLEEP_NS);
#endif
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace svx

#endif  // __CUDACC__
#endif  // SVX_GRID_H
