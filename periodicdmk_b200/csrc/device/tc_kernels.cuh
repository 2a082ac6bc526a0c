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

// Residual near field of kb charge vectors as a GEMM per (target leaf, 128-target tile):
//   pot[c*N + t] += sum_s K(t,s) q[s*kb + c],   K(t,s) = P((r - b/2) 2/b) / r for 1e-30 < r^2 < b^2
// over the leaf's list-1 source boxes (b per box).  The kernel values are
// generated from double-float coordinates in FP32 on the CUDA cores, the
// products run on the tensor cores (TF32 hi/lo split) into a tensor-memory
// accumulator per source box, and each box's sum is added to FP64
// accumulators.  Chunks whose bounding box lies farther than b from the
// tile's targets are skipped.  Covers nc in {5, 6, 9, 11, 12}, 1 <= kb <= 64 and
// leaves with at most 128 source boxes and 4096 chunks.
struct NearTc {
    const int* trg_start;
    const int* trg_count;
    const int* pair_start;  // CSR over target leaves
    const int* pair_src_start;
    const int* pair_src_count;
    const double* pair_bsize;
    // bounding boxes of the 32-source chunks of each pair's source range:
    // chunk j of pair pr is entry pair_chunk_base[pr] + j (float, rounded outwards)
    const int* pair_chunk_base;
    const float4* chunk_lo;
    const float4* chunk_hi;
    double coef[32];
    int n_leaves;
    int max_trg;  // largest trg_count (grid extent over 128-target tiles)
    int64_t N;
    int kb;
    // Failure-detection test hook: CTA 0 issues neither the MMAs nor the
    // commits of chunk withhold_chunk (-1: none), so a later bounded wait on
    // that chunk's barrier runs out; wait_cycles bounds the pipeline waits
    // inside the chunk loop (SM clock cycles).
    int withhold_chunk;
    long long wait_cycles;
    // chunks of 32 sources accumulated in tensor memory between two FP64 drains
    // (<= 0: the default, 2)
    int seg_chunks;
};
constexpr int kNearTcMaxPairs = 128;
constexpr int kNearTcChunk = 32;        // sources per chunk
constexpr int kNearTcMaxChunks = 4096;  // chunks of one leaf's pairs (before the bounding-box cull)
bool launch_near_tc(const NearTc& a, int nc, const float4* trg_hi, const float4* trg_lo, const float4* src_hi,
                    const float4* src_lo, const float* src_q, double* pot, int* err, cudaStream_t s);

// Leaf evaluation of kb RHS as a GEMM per (leaf, 128-target tile):
//   pot[c*N + t] += sum_l T_l(z_t) sum_{(i,j)} T_i(x_t) T_j(y_t) C[(slot*kb + c)*p^3 + i + p j + p^2 l]
// with D[t, (l,c)] = A[t, (i,j)] B[(l,c), (i,j)] on the tensor cores (TF32
// hi/lo split) and the z sum in the epilogue.  Covers p in {9, 18}, kb in
// {16, 32, 64}.
struct EvalTc {
    const double4* trg;
    const float* proxy_down;
    double* pot;
    int n_leaves;
    int max_trg;
    const int* slot;
    const int* trg_start;
    const int* trg_count;
    const double4* center_scale;
    int64_t N;
};
bool launch_eval_tc(const EvalTc& a, int p, int kb, int* err, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
