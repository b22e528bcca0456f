// Grid barrier for cooperative launches (every block resident), with a bounded wait.
//
// The counter only grows: a block arrives with one relaxed atomic add after an acquire-release fence at GPU scope
// (which orders the writes that its threads made before the __syncthreads), and waits until the counter reaches
// (its arrival index rounded up to a whole grid).  The last block to arrive therefore releases the others by its
// own add, and nothing has to reset the counter between barriers; the host clears it before a launch (and after a
// launch that timed out, where the blocks left at different barriers).  A waiting block gives up after `pollLimit`
// polls: it records LBM_ERR_DEVICE_TIMEOUT in `status`, and every block leaves at its next barrier (a block also
// looks at the status word every 256 polls).  Thread 0 takes the decision for its block, so all threads of a block
// return the same value.
#pragma once

#include "lbm_b200.h"
#include <cstdint>

namespace lbm {

__device__ __forceinline__ unsigned loadRelaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fenceAcqRel() {
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

__device__ __forceinline__ bool gridSync(unsigned* counter, int* status, long long pollLimit) {
    __shared__ int okShared;
    __syncthreads();
    if (threadIdx.x == 0) {
        bool ok = true;
        fenceAcqRel();
        const unsigned arrival = atomicAdd(counter, 1u);
        const unsigned target = (arrival/gridDim.x + 1)*gridDim.x;
        long long polls = 0;
        while ((int) (loadRelaxed(counter) - target) < 0) {
            if (++polls > pollLimit ||
                    ((polls & 255) == 0 && *((volatile int*) status) == LBM_ERR_DEVICE_TIMEOUT)) {
                atomicExch(status, LBM_ERR_DEVICE_TIMEOUT);
                ok = false;
                break;
            }
        }
        fenceAcqRel();
        okShared = ok && *((volatile int*) status) != LBM_ERR_DEVICE_TIMEOUT;
    }
    __syncthreads();
    return okShared != 0;
}

} // namespace lbm
