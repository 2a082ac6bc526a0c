// Tensor-core (tcgen05, TF32 split into hi + lo parts) kernels of the
// mixed-precision multi-RHS path.  Launchers return false when the shape is
// not covered (the caller then uses its CUDA-core kernel).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// Proxy moments of kb charge vectors as a GEMM per centre box:
//   proxy_up[(slot*kb + c)*p^3 + i + p*j + p^2*l] += sum_s T_i(x_s) T_j(y_s) T_l(z_s) q[s*kb + c]
// rows (l, c) of the product on the MMA M side (128 per CTA), columns (i, j)
// on the N side, sources along K.  err: device int set to 1 if a pipeline
// wait timed out.  Covers p in {9, 18}, 16 <= kb <= 64.
bool launch_c2proxy_tc(const C2ProxyArgs& a, const float* src_q, float* proxy_up, int kb, int p, int* err,
                       cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
