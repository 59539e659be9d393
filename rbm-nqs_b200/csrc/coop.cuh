// coop.cuh -- grid-wide barrier with a bounded wait for the cooperative
// persistent solver kernels (cg_mfree.cu, direct.cu).
#pragma once

#include <cstdint>

#include "sr.cuh"

namespace rbmnqs {

constexpr uint32_t kBarrierSpin = 1u << 24;

// Counter barrier over all blocks of a cooperative launch.  The counter only
// grows: the arrival of barrier k returns a value in [k need, (k + 1) need),
// so each block knows the count that ends its barrier, and waiting blocks
// poll the counter itself (acquire loads), with no reset and no second
// atomic on the critical path.  Returns false (on every thread of the block)
// if this block waited more than kBarrierSpin polls or another block already
// gave up (checked every 64 polls); the kernel then records the failure and
// returns instead of hanging.  sync must be zeroed before the launch.
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

static __device__ bool grid_barrier(MfreeSync* sync, uint32_t nblocks) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const uint32_t need = nblocks + sync->extra;
        const uint32_t cap = sync->spin_cap ? sync->spin_cap : kBarrierSpin;
        __threadfence();  // the block's writes before the arrival
        const uint32_t old = atomicAdd(&sync->count, 1u);
        const uint32_t target = (old / need + 1u) * need;
        uint32_t spins = 0;
        while (ld_acquire_gpu(&sync->count) < target) {
            if ((++spins & 63u) == 0u && (spins > cap || *reinterpret_cast<volatile int*>(&sync->bad))) {
                ok = 0;
                atomicExch(&sync->bad, 1);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace rbmnqs
