// One step of a separable tensor transform on the tcgen05 tensor cores
// (contract_tc.cu), FP32 data, 3xTF32 products, FP32 accumulation in tensor
// memory:
//   out[e][(r + R a) co + c_o] (op)= sum_{i, c_i} in[e][(i + ni r) ci + c_i] * B[(i, c_i), (a, c_o)]
// with B the real form of the na x ni matrix M (column-major, M[a + na i]):
//   real M, ci = co = 1:          B = M
//   complex M, ci = 1, co = 2:    (re, im) of M x
//   complex M, ci = co = 2:       complex product M x
//   complex M, ci = 2, co = 1:    scale * Re(M x)
// The contracted index is the fastest of the input and the new index the
// slowest of the output, so three steps apply a matrix along each axis of a
// tensor in turn (the convention of the CUDA-core contraction kernels).
// Entry ge = e0 + blockIdx.x is (box eb = ge / rhs, RHS ec = ge % rhs);
// offsets are in units of the input / output element (real or complex).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pdmkb {
namespace dev {

struct ContractTc {
    const float* in;
    const int64_t* in_off;  // per box; null: entry blockIdx.x at in_stride
    int64_t in_stride, in_unit;
    float* out;
    const int64_t* out_off;
    int64_t out_stride, out_unit;
    const float* mat;         // real or complex (interleaved) floats
    const int64_t* mat_off;   // per box, in matrix elements; null: one matrix
    int mat_complex;
    int ni, na, R;
    int ci, co;
    int rhs;
    int64_t e0;
    int n_entries;
    int accumulate;           // 0 store, 1 add
    float scale;              // complex -> real steps: factor on Re
    int* err;                 // set when a pipeline wait runs out
};

// false if the shape is not covered (K = ni ci > 96 or N = na co > 128)
bool contract_tc_supported(int ni, int na, int ci, int co);
void launch_contract_tc(const ContractTc& a, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
