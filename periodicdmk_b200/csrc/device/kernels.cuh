// Kernel argument blocks and launchers for the periodic DMK evaluate path.
// All pointers are device pointers.  Index lists are built once per tree on
// the host (device_tree.cu) and checked there against the buffer sizes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace pdmkb {
namespace dev {

// ---- charge gather: src[i].w = q_user[src_charge_idx[i]]
void launch_gather(double4* src, const int* src_charge_idx, const double* q_user, int n_all, cudaStream_t s);

// ---- proxy moments: for each centre box, M(i,j,k) = sum_s q_s T_i T_j T_k
struct C2ProxyArgs {
    const double4* src;
    double* proxy_up;
    int n_centers;
    const int* slot;              // proxy_up slot of the centre
    const double4* center_scale;  // (cx, cy, cz, 2/boxsize)
    const int* rng_start;         // CSR over centres into (src_start, src_count)
    const int* src_start;
    const int* src_count;
};
void launch_c2proxy(const C2ProxyArgs& a, int p, cudaStream_t s);

// ---- batched separable contraction:
// out[r + R*a] (op)= sum_i M[a + na*i] * in[i + ni*r],  r < R, a < na
// for each entry e with in = in_base + in_off[e] (or e*in_stride),
// out = out_base + out_off[e] (or e*out_stride), M = mat_base + mat_off[e] (or 0).
enum ContractMode { kStore = 0, kAdd = 1, kAddRealScaled = 2 };
enum ContractType { kRRR = 0, kRCC = 1, kCCC = 2, kCCR = 3 };  // (in, mat, out): R real, C complex
// Structure of M the contraction may exploit (the entries it skips are zero up
// to rounding in the tables it is used with):
//   kTriUpper  M[a + na*i] = 0 for i > a   (child -> parent translation)
//   kTriLower  M[a + na*i] = 0 for i < a   (parent -> child translation)
//   kParIn     M real for even i, imaginary for odd i   (polynomial -> plane wave)
//   kParOut    M real for even a, imaginary for odd a   (plane wave -> polynomial)
enum ContractStruct { kDense = 0, kTriUpper = 1, kTriLower = 2, kParIn = 3, kParOut = 4 };
struct ContractArgs {
    const void* in;
    const int64_t* in_off;
    int64_t in_stride;
    void* out;
    const int64_t* out_off;
    int64_t out_stride;
    const void* mat;
    const int64_t* mat_off;
    int ni, na, R, n_entries;
    int mode;
    double scale;
    int structure;  // ContractStruct (0: dense)
};
void launch_contract(const ContractArgs& a, ContractType t, cudaStream_t s);

// ---- plane-wave shift: pw_in[e][m] = sum_terms pw_out[slot][m] * shift[stencil][m]
struct ShiftArgs {
    const cd* pw_out;
    const double* shift;  // 27 x (M re | M im) for the level
    cd* pw_in;
    int M, n_entries;
    const int* term_start;  // CSR (n_entries + 1)
    const int* term_slot;
    const int* term_stencil;
};
void launch_shift(const ShiftArgs& a, cudaStream_t s);

// ---- proxy -> leaf targets
struct EvalArgs {
    const double4* trg;
    const double* proxy_down;
    double* pot;  // sorted targets, accumulated
    int n_leaves;
    const int* slot;
    const int* trg_start;
    const int* trg_count;
    const double4* center_scale;
};
void launch_eval(const EvalArgs& a, int p, cudaStream_t s);

// ---- residual near field
struct NearArgs {
    const double4* trg;
    const double4* src;
    double* pot;  // sorted targets, accumulated
    int n_leaves;
    const int* trg_start;
    const int* trg_count;
    const int* pair_start;        // CSR (n_leaves + 1)
    const int* pair_src_start;
    const int* pair_src_count;
    const double* pair_bsize;
    // bounding boxes (float, rounded outwards) of the 32-source chunks of each
    // pair's source range: chunk j of pair pr is entry pair_chunk_base[pr] + j
    const int* pair_chunk_base;
    const float4* chunk_lo;
    const float4* chunk_hi;
    double coef[32];
    int nc;
};
void launch_near(const NearArgs& a, cudaStream_t s);

// ---- final gather: pot_user[trg_perm[i]] = pot[i] + far[i] - selfw[i] * q_user[trg_perm[i]]
void launch_finalize(const double* pot_sorted, const double* far_sorted, const double4* trg, const int* trg_perm,
                     const double* q_user, double* pot_user, int n, cudaStream_t s);

// ---- out[i] = (float)in[i]
void launch_to_float(const double* in, float* out, int64_t n, cudaStream_t s);

// ---- FMA throughput probe of the current device, TFLOP/s (2 flops per FMA)
double fma_probe_tflops(bool fp64);
// Measured tensor-core throughput (TFLOP/s, 2 flops per multiply-add) of the
// current device: kind 0 tcgen05 TF32 MMA (M 128, N 256, operands in shared
// memory), kind 1 FP64 DMMA (mma.sync m8n8k4).  Defined in peaks.cu.
double tc_probe_tflops(int kind);

// ---- the two parts of the potential in user order (tests / diagnostics)
void launch_desort_parts(const double* pot_sorted, const double* far_sorted, const double4* trg, const int* trg_perm,
                         const double* q_user, double* tree_part, double* far_part, int n, cudaStream_t s);

// ---- NUFFT far field (ES kernel, sigma = 2)
constexpr int kSpreadRunDx = 4;
struct NufftArgs {
    int n_leaves;
    const int* trg_start;
    const int* trg_count;
    const int4* sub_origin;  // per leaf: subgrid origin (x,y,z), w unused
    const int4* sub_extent;  // per leaf: extents
    const double4* pt_t;     // per sorted target: grid coordinate t = s*n per axis, .w = charge slot unused
    const int4* pt_l0;       // per sorted target: first grid index of the window
    const double* q_sorted;  // per sorted target charge (user charge gathered)
    double* grid;            // n1*n2*n3 real
    double* far;             // per sorted target output
    // Order in which the interpolation visits the sorted targets: inside each
    // bin, targets grouped by the grid cell their window starts at, so that
    // neighbouring threads read the same grid values (null: sorted order).
    const int* interp_order = nullptr;
    // Interpolation pairs: consecutive targets of the interpolation order
    // whose windows start at the same cell, interpolated by one thread (y = -1
    // for a target without a partner); bin e owns pairs bin_pair[e] ..
    // bin_pair[e + 1] - 1.  Null: no pair lists.
    const int2* interp_pair = nullptr;
    const int* bin_pair = nullptr;
    int max_pairs = 0;  // most pairs in one bin
    // Spreading by runs: inside each bin, targets whose windows start at the
    // same (y, z) cell form a run (ordered by x; x offsets within a run at
    // most kSpreadRunDx).  run = (first index into spread_order, count,
    // y | z << 16 relative to the bin origin, smallest x relative to it);
    // bin e owns runs bin_run[e] .. bin_run[e + 1] - 1.  Null: no run lists.
    const int4* spread_run = nullptr;
    const int* bin_run = nullptr;
    const int* spread_order = nullptr;
    int max_cells = 0;  // largest bin subgrid (cells)
    int n1, n2, n3;
    int w;
    double es_beta;
    // RHS batching (blockIdx.z = RHS index): element strides between RHS of
    // q_sorted, grid and far; 0 for a single RHS.
    int64_t rhs_q_stride = 0, rhs_grid_stride = 0, rhs_far_stride = 0;
};
void launch_nufft_gather_q(const int* trg_perm, const double* q_user, double* q_sorted, int n, cudaStream_t s);
void launch_spread(const NufftArgs& a, int max_jk, int max_ex, cudaStream_t s, int nrhs = 1);
void launch_interp(const NufftArgs& a, cudaStream_t s, int nrhs = 1);
// spec[c * n + i] *= mult[i] for c < nrhs
void launch_multiply(cd* spec, const double* mult, int64_t n, cudaStream_t s, int nrhs = 1);

}  // namespace dev
}  // namespace pdmkb
