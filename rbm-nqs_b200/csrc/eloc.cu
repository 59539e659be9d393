// eloc.cu -- host launcher of the FP32 evaluation kernel (eloc.cuh): picks
// the instantiation for the machine's entries per lane, sizes shared memory
// and the persistent grid.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "eloc.cuh"

namespace rbmnqs {
namespace {

using eloc::ElocLayout;

const void* pick_eloc(int kb, int ng, bool sym, int nfm) {
    switch (kb) {
        case 4: return eloc::pick_kb4(ng, sym, nfm);
        case 2: return eloc::pick_kb2(ng, sym, nfm);
        case 1: return eloc::pick_kb1(ng, sym, nfm);
    }
    return nullptr;
}

// resident blocks per SM of a kernel at a dynamic shared-memory size, per
// (device, kernel, size)
int blocks_per_sm(const void* fn, int threads, int smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int>, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple(dev, fn, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess || nb < 1)
        nb = 1;
    cache[key] = nb;
    return nb;
}

}  // namespace

cudaError_t launch_eloc_fast(const EvalArgs& a, cudaStream_t st) {
    const MachineDev& m = a.m;
    if (m.pf.n > 0 || !a.tt.terms || a.ratio || a.tt.nf_max > 6 || m.n > 255) return cudaErrorNotSupported;
    if (a.B == 0) return cudaSuccess;
    const int kb = m.nh % 4 == 0 ? 4 : (m.nh % 2 == 0 ? 2 : 1);
    const int G = m.T / kb;
    int ng = kb == 1 ? 2 : 1;  // entries come in pairs
    while (32 * ng < G) ng *= 2;
    if (kb * ng > 16) return cudaErrorNotSupported;
    const void* fn = pick_eloc(kb, ng, m.symmetric != 0, a.tt.nf_max);
    if (!fn) return cudaErrorNotSupported;
    int dev = 0, budget = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&budget, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int warps = eloc::eloc_warps(kb * ng);
    // small blocks share the SM seven ways: keep their tables to a seventh
    // where they fit (basic machines read W from L2 otherwise)
    if (kb * ng <= 4) budget = std::min(budget, 32 * 1024 - 1024);
    const ElocLayout L = eloc::eloc_layout(m, a.tt, kb, warps, a.O != nullptr, budget);
    if (L.total > budget) return cudaErrorNotSupported;
    if ((e = ensure_dynamic_smem(fn, L.total)) != cudaSuccess) return e;
    const int per_sm = blocks_per_sm(fn, 32 * warps, L.total);
    const int blocks = std::max(1, std::min((a.B + warps - 1) / warps, sms * per_sm));
    EvalArgs aa = a;
    ElocLayout ll = L;
    void* args[] = {&aa, &ll};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(32 * warps), args, (size_t)L.total, st);
}

}  // namespace rbmnqs
