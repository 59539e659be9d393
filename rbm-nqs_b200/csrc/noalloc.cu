// noalloc.cu -- SR solve that allocates no device memory.
//
// rbmnqs_sr_solve allocates its working buffers (partial Gram sums, the Gram
// matrix, the regularised S and the CG status) with cudaMalloc on every call.
// Some callers cannot do that: code embedded in a runtime that owns all device
// memory through its own pool and forbids raw cudaMalloc/cudaFree, and
// latency-critical loops that cannot afford the implicit device-wide
// synchronisation of cudaMalloc/cudaFree.  rbmnqs_sr_solve_noalloc serves them:
// inputs and outputs are the caller's device buffers, and all working memory
// is the fixed array below, which every GPU that loads this library holds
// until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "rbmnqs_b200.h"
#include "sr.cuh"

namespace {

constexpr int kMaxP = RBMNQS_NOALLOC_MAX_PARAMS;
constexpr int kSplits = 2;  // sample-range splits of the Gram accumulation
constexpr size_t kMat = (size_t)kMaxP * kMaxP * sizeof(double2);
// partial Gram sums [kSplits][P][P] | Gram G [P][P] | S_reg [P][P] | CG status
constexpr size_t kScratchBytes = (kSplits + 2) * kMat + 256;

// The scratch array.  In host code this name is only a host-side stand-in:
// the device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_sr_scratch[kScratchBytes];

std::mutex g_mu;
void* g_addr[64] = {};  // device address of g_sr_scratch, per device ordinal

int fail(int code, const std::string& m) {
    rbmnqs::set_last_error(m);
    return code;
}

}  // namespace

extern "C" int rbmnqs_sr_solve_noalloc(const double* O, int32_t N, int32_t P, int32_t n_neural, const double* d,
                                       double norm, const double* F, double* x, double r1, double r2, double rd,
                                       const double* diag, int32_t max_iterations, double rtol, void* stream,
                                       int32_t* iterations, double* residual) {
    if (!O || !d || !F || !x || !diag) return fail(RBMNQS_ERR_ARG, "rbmnqs_sr_solve_noalloc: null buffer");
    if (P < 1 || P > kMaxP)
        return fail(RBMNQS_ERR_ARG, "rbmnqs_sr_solve_noalloc: n_params must be in 1.." + std::to_string(kMaxP) +
                                        " (fixed scratch of " + std::to_string(kScratchBytes) + " bytes), got " +
                                        std::to_string(P));
    if (N < 1 || !(norm > 0) || n_neural < 0 || n_neural > P)
        return fail(RBMNQS_ERR_ARG, "rbmnqs_sr_solve_noalloc: bad N, norm or n_neural");
    if (max_iterations < 0)
        return fail(RBMNQS_ERR_ARG, "rbmnqs_sr_solve_noalloc: max_iterations must be >= 0 (0 = 2 n_params)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(RBMNQS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(RBMNQS_ERR_ARG, "rbmnqs_sr_solve_noalloc: device ordinal >= 64");
    unsigned char* base = nullptr;
    {
        // first call on this device: resolve the array's device address
        // with this device current
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_sr_scratch);
            if (e != cudaSuccess)
                return fail(RBMNQS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_addr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_addr[dev]);
    }
    const size_t mat = (size_t)P * P * sizeof(double2);
    double2* part = reinterpret_cast<double2*>(base);
    double2* G = reinterpret_cast<double2*>(base + kSplits * mat);
    double2* Sreg = reinterpret_cast<double2*>(base + (kSplits + 1) * mat);
    auto* res = reinterpret_cast<rbmnqs::CgResultDev*>(base + (kSplits + 2) * mat);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: the CG status is the only
    // part read before being written
    e = cudaMemsetAsync(res, 0, sizeof(*res), st);
    if (e != cudaSuccess) return fail(RBMNQS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    int splits = kSplits;
    if (N < 16 * splits) splits = 1;
    const auto* O2 = reinterpret_cast<const double2*>(O);
    if ((e = rbmnqs::launch_gram_fp64(O2, 1, nullptr, N, P, splits, part, G, st)) != cudaSuccess ||
        (e = rbmnqs::launch_solve_prep(G, N, norm, reinterpret_cast<const double2*>(d), diag, P, n_neural, r1, r2,
                                       rd, Sreg, st)) != cudaSuccess)
        return fail(RBMNQS_ERR_CUDA, std::string("rbmnqs_sr_solve_noalloc: ") + cudaGetErrorString(e));
    int max_it = max_iterations < 2 * P ? max_iterations : 2 * P;
    if (max_it == 0) max_it = 2 * P;
    if (rtol == 0) rtol = 1e-16;
    e = rbmnqs::launch_cg(Sreg, reinterpret_cast<const double2*>(F), reinterpret_cast<double2*>(x), P, max_it, rtol,
                          res, st);
    if (e != cudaSuccess) return fail(RBMNQS_ERR_CUDA, std::string("rbmnqs_sr_solve_noalloc: ") + cudaGetErrorString(e));
    if (iterations || residual) {
        rbmnqs::CgResultDev h{};
        e = cudaMemcpyAsync(&h, res, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(RBMNQS_ERR_CUDA, std::string("status read: ") + cudaGetErrorString(e));
        if (iterations) *iterations = h.iterations;
        if (residual) *residual = h.residual;
    }
    return RBMNQS_OK;
}
