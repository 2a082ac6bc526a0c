// Far-field NUFFT for blocks of RHS with precomputed spreading weights.
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// w[t * 3W + d * W + c] = phi of tap c along axis d for sorted target t (t < n)
void launch_es_weights(const NufftArgs& a, int64_t n, double* w, cudaStream_t s);
// grid[c] += spread of q_sorted[c] for c < nrhs (grid zeroed by the caller)
void launch_spread_multi(const NufftArgs& a, const double* esw, int max_jk, int max_ex, int nrhs, cudaStream_t s);
// far[c][t] = interpolation of grid[c] at sorted target t, c < nrhs
void launch_interp_multi(const NufftArgs& a, const double* esw, int64_t n, int nrhs, cudaStream_t s);
// Spreading with single-precision weights and partial sums into the FP64
// grid (mixed-precision path); false: not applicable, use launch_spread_multi.
bool launch_spread_multi_f32(const NufftArgs& a, const float* esw32, int nrhs, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
