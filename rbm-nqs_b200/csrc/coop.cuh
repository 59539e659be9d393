// coop.cuh -- grid-wide barrier with a bounded wait for the cooperative
// persistent solver kernels (cg_mfree.cu, direct.cu).
#pragma once

#include <cstdint>

#include "sr.cuh"

namespace rbmnqs {

constexpr uint32_t kBarrierSpin = 1u << 24;

// Counter + generation barrier over all blocks of a cooperative launch.
// Returns false (on every thread of the block) if this block waited more
// than kBarrierSpin polls or another block already gave up; the kernel then
// records the failure and returns instead of hanging.  sync must be zeroed
// before the launch.
static __device__ bool grid_barrier(MfreeSync* sync, uint32_t nblocks) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* gen = &sync->gen;
        volatile int* bad = &sync->bad;
        const uint32_t g = *gen;
        const uint32_t need = nblocks + sync->extra;
        const uint32_t cap = sync->spin_cap ? sync->spin_cap : kBarrierSpin;
        __threadfence();
        if (atomicAdd(&sync->count, 1u) == need - 1) {
            sync->count = 0;
            __threadfence();
            atomicAdd(&sync->gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g) {
                if (++spins > cap || *bad) {
                    ok = 0;
                    atomicExch(&sync->bad, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (*bad) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace rbmnqs
