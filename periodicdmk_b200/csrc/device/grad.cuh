// Gradient of the potential at the targets, plain FP64 path (grad.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// The tree's frame: positions were rotated by Q^T (r = Q^T x); fractional
// coordinates are s = U^-1 r.  Column-major 3x3 each.
struct GradFrame {
    double qmat[9];
    double umatinv[9];
};

// Near field: pot += residual sum (as launch_near) and grad[d n + t] += its gradient.
void launch_near_pg(const NearArgs& a, double* grad, int64_t n, cudaStream_t s);
// Leaf evaluation gradient: grad[d n + t] += d/dx_d of the local expansions.
void launch_eval_grad(const EvalArgs& a, int p, double* grad, int64_t n, cudaStream_t s);
// out = i K_d spec over the half spectrum of an n1 x n2 x n3 real grid.
void launch_grad_multiply(const cd* spec, cd* out, int n1, int n2, int n3, int d, const GradFrame& f,
                          cudaStream_t s);
// grad_user[3 perm[t] + e] = (Q (g + far_g)[., t])_e
void launch_finalize_grad(const double* g, const double* far_g, const int* perm, double* out, int64_t n,
                          const GradFrame& f, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
