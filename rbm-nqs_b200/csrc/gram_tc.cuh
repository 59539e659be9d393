// gram_tc.cuh -- tensor-core (tcgen05, FP16 split precision) SR Gram.
#pragma once

#include <cstddef>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace rbmnqs {

// Shapes, planes and TMA descriptors of one Gram problem (N samples x P
// complex parameters).  R = 2P rounded up to 128 (real rows of X^T),
// K = N rounded up to 64; Xh / Xl are the FP16 hi / lo planes [R][K] of the
// scaled rows, rmax the R row maxima the scales come from.
struct GramTC {
    int N = 0, P = 0, R = 0, K = 0, ntile = 0, nsplit = 1, max_splits = 1;
    __half* Xh = nullptr;
    __half* Xl = nullptr;
    float* rmax = nullptr;
    alignas(64) unsigned char map_h[128];
    alignas(64) unsigned char map_l[128];
    // bytes of the FP32 split-K partial tiles for the largest split count
    size_t partial_bytes() const;
    // elements of one plane
    size_t plane_elems() const { return (size_t)R * K; }
    // bytes of the planes and the row maxima (one buffer, gram_tc_maps)
    size_t buffer_bytes() const { return 2 * plane_elems() * 2 + (size_t)R * 4; }
};

cudaError_t gram_tc_plan(int N, int P, GramTC* g);
// up to max_out split counts (1..max_splits) in order of modelled cost
int gram_tc_split_candidates(const GramTC& g, int* out, int max_out);
cudaError_t gram_tc_set_splits(GramTC* g, int ns);
// buf: buffer_bytes(), zero-filled once (the padding rows / columns of the
// planes are never written); carves the planes and encodes the two tensor
// maps.
cudaError_t gram_tc_maps(GramTC* g, void* buf);
// S = <conj(O - d)(O - d)^T> (divided by N, Hermitian, P x P) from
// sample-major O (fp64 != 0: double2, else float2).  err receives a nonzero
// code if a pipeline wait timed out (S is then incomplete).
cudaError_t launch_gram_tc(const GramTC& g, const void* O, int fp64, const double2* d, float* part, int* err,
                           double2* S, cudaStream_t st);

}  // namespace rbmnqs
