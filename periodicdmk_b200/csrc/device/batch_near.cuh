// Near field + final gather of many independent systems in one persistent
// launch over a device queue of (system, target leaf) items (batch_near.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// One system's device buffers, as its float tree's single-RHS state holds them.
struct NearLeafSys {
    const int* trg_start;       // per near leaf: first sorted target
    const int* trg_count;
    const int* pair_start;      // CSR over near leaves
    const int* pair_src_start;  // per near pair: sorted source range
    const int* pair_src_count;
    const double* pair_bsize;   // per near pair: cutoff b
    const int* pair_chunk_base; // per near pair: index of the first 32-source chunk box of its source box
    const float4* chunk_lo;     // per 32-source chunk: bounding box (rounded outwards)
    const float4* chunk_hi;
    const float4* trg_hi;       // double-float split positions (tree order)
    const float4* trg_lo;
    const float4* src_hi;
    const float4* src_lo;
    const float* src_q;         // source charges (tree order)
    const double* pot;          // tree part of the potential without the near field (tree order)
    const double* far;          // far field (tree order)
    const double4* trg;         // .w = self-interaction weight of the target's leaf
    const int* perm;            // sorted target -> user index
    const double* q_t;          // target charges (tree order)
    double* out;                // potentials, user order
};

struct BatchNearArgs {
    const NearLeafSys* sys;
    const int2* items;  // (system, near leaf), largest estimated work first
    int n_items;
    int* head;          // queue head (reset to 0 by the launcher)
    float coef32[32];   // residual polynomial (same digit count for every system)
};

// One system's leaf-evaluation inputs (float tree, one RHS): the leaves,
// their proxy potentials (FP32, one RHS) and the tree-order potentials the
// evaluation adds to.
struct EvalLeafSys {
    EvalArgs a;              // trg, slot, trg_start, trg_count, center_scale
    const float* proxy_down;
    double* pot;
};
// Leaf evaluation of many systems in one launch: one CTA per (system, leaf)
// item (defined with the single-system kernel in multi.cu).
void launch_batch_eval(const EvalLeafSys* sys, const int2* items, int n_items, int p, cudaStream_t s);

// One system's far-field interpolation inputs (one RHS): its transformed
// grid, its targets' window taps and the far-field output (tree order).
struct InterpSys {
    NufftArgs a;        // grid, far, pt_l0, grid sizes, width, visit order
    const double* esw;  // per target: 3 x W taps
    int64_t n;          // targets
};
// Interpolation of many systems in one launch: one CTA per (system, block of
// 128 targets) item; every system has the kernel width w (defined with the
// single-system kernels in nufft_multi.cu).
void launch_batch_interp(const InterpSys* sys, const int2* items, int n_items, int w, cudaStream_t s);

// CTAs that fill the GPU at full occupancy for tpt targets per thread.
int batch_near_ctas(int nc, int tpt);
// tpt: targets per thread (1, 2 or 4); ctas: persistent grid size.
void launch_batch_near(const BatchNearArgs& a, int nc, int tpt, int ctas, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
