// Quasi-periodic (Bloch) evaluate kernels (qp.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace pdmkb {
namespace dev {

// src_q[2 j + c] = q[idx[j]] (cos, sin)_c(bloch.R_j) for every sorted source j
// (the image charges of the reference's build_combined_sources,
// cpp/include/dmk/pbc.hpp:142-256); far_q[c n + t] = q[perm[t]] times
// (cos, -sin)_c(bloch.x_t) for every sorted target (the far field's phased
// charges q e^{-i bloch.x}, cpp/src/dmk/pbc.cpp:280-287).  q: user order.
void launch_qp_charges(double* src_q, const int* idx, const double2* src_phase, int64_t n_all, double* far_q,
                       const int* perm, const double2* trg_phase, int64_t n, const double* q, cudaStream_t s);
// a = spec[i], b = spec[n_spec + i] (spectra of the two real grids):
// spec[i] = s a + i d b, spec[n_spec + i] = s b - i d a (the spectra of the real
// and the imaginary part of the weighted non-Hermitian spectrum).
void launch_qp_combine(cd* spec, const double* qs, const double* qd, int64_t n_spec, cudaStream_t s);
// out[2 u] + i out[2 u + 1], u = perm[t]: tree part (pot[t] + i pot[n + t]) minus
// the self term w_t q_u, plus e^{i bloch.x_t} (far[t] + i far[n + t]).
void launch_qp_finalize(const double* pot, const double* far, const double4* trg, const int* perm, const double* q,
                        const double2* trg_phase, double* out, int64_t n, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
