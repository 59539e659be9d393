// gram_tc.cuh -- tensor-core (tcgen05, TF32 split precision) SR Gram.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace rbmnqs {

// Shapes, planes and TMA descriptors of one Gram problem (N samples x P
// complex parameters).  R = 2P rounded up to 128 (real rows of X^T),
// K = N rounded up to 32; Xh / Xl are the TF32 hi / lo planes [R][K].
struct GramTC {
    int N = 0, P = 0, R = 0, K = 0, ntile = 0, nsplit = 1;
    float* Xh = nullptr;
    float* Xl = nullptr;
    alignas(64) unsigned char map_h[128];
    alignas(64) unsigned char map_l[128];
    // bytes of the FP32 split-K partial tiles
    size_t partial_bytes() const;
    // floats of one plane
    size_t plane_floats() const { return (size_t)R * K; }
};

cudaError_t gram_tc_plan(int N, int P, GramTC* g);
// Planes must be zero-filled once (the padding rows / columns are never
// written); encodes the two tensor maps.
cudaError_t gram_tc_maps(GramTC* g, float* Xh, float* Xl);
// S = <conj(O - d)(O - d)^T> (divided by N, Hermitian, P x P) from
// sample-major O (fp64 != 0: double2, else float2).  err receives a nonzero
// code if a pipeline wait timed out (S is then incomplete).
cudaError_t launch_gram_tc(const GramTC& g, const void* O, int fp64, const double2* d, float* part, int* err,
                           double2* S, cudaStream_t st);

}  // namespace rbmnqs
