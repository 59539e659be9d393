// ed.cuh -- Lanczos ground state of a model Hamiltonian on the full basis.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sampler.cuh"

namespace rbmnqs {

// Lowest eigenvalue of H (device operator tables of n sites) by Lanczos,
// stopping when it changed by at most tol (relative) over three iterations
// or after max_iter; psi_host (2^n entries, may be null) receives the
// normalised eigenvector.  Allocates 3 (4 with psi) vectors of 2^n double2.
cudaError_t ed_ground_state(const HamDev& H, int n, int max_iter, double tol, uint64_t seed, cudaStream_t st,
                            double* energy, int* iterations, double2* psi_host);

}  // namespace rbmnqs
