// Far-field NUFFT spreading / interpolation for blocks of RHS (FP64).
//
// The spreading-kernel weights of a target depend only on its position, so
// they are evaluated once per tree (k_es_weights) and shared by every RHS of
// every block and by both the spread and the interpolation.  Spread keeps the
// per-bin subgrid layout of the single-RHS kernel (thread = (y,z) column, x in
// registers) with an inner block of CB RHS per thread; interpolation runs one
// thread per target with CB RHS accumulated in registers.
// Grid layout (cuFFT batched real input): grid[c * rhs_grid_stride + (x*n2 + y)*n3 + z].
#include <stdexcept>

#include "batch_near.cuh"
#include "common.cuh"
#include "kernels.cuh"
#include "nufft_multi.cuh"

namespace pdmkb {
namespace dev {

namespace {

// exponential-of-semicircle kernel phi(z) = exp(beta (sqrt(1 - z^2) - 1)), |z| < 1
__device__ __forceinline__ double es_phi(double z, double beta) {
    const double z2 = z * z;
    return z2 < 1.0 ? exp(beta * (sqrt(1.0 - z2) - 1.0)) : 0.0;
}

__device__ __forceinline__ int wrap_index(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

template <int W>
__global__ void k_es_weights(NufftArgs a, int64_t n, double* __restrict__ w) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double4 tt = a.pt_t[t];
    const int4 l0 = a.pt_l0[t];
    const double hw = 0.5 * W;
    double* o = w + t * 3 * W;
#pragma unroll
    for (int c = 0; c < W; ++c) {
        o[c] = es_phi((tt.x - (double)(l0.x + c)) / hw, a.es_beta);
        o[W + c] = es_phi((tt.y - (double)(l0.y + c)) / hw, a.es_beta);
        o[2 * W + c] = es_phi((tt.z - (double)(l0.z + c)) / hw, a.es_beta);
    }
}

template <int W, int NX, int CB>
__global__ void __launch_bounds__(128) k_spread_m(NufftArgs a, const double* __restrict__ esw) {
    constexpr int TS = 32;
    __shared__ double sBx[TS][NX];
    __shared__ double sKy[TS][W], sKz[TS][W];
    __shared__ int sOy[TS], sOz[TS];
    __shared__ double sQ[CB][TS];
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const int4 org = a.sub_origin[e], ext = a.sub_extent[e];
    const int c0 = blockIdx.z * CB;
    const int jk = blockIdx.y * blockDim.x + threadIdx.x;
    const bool active = jk < ext.y * ext.z;
    const int ez = max(ext.z, 1);
    const int kk = jk % ez, jj = jk / ez;
    double acc[NX][CB];
#pragma unroll
    for (int i = 0; i < NX; ++i)
#pragma unroll
        for (int c = 0; c < CB; ++c) acc[i][c] = 0.0;
    for (int base = 0; base < nt; base += TS) {
        const int m = min(TS, nt - base);
        __syncthreads();
        for (int idx = threadIdx.x; idx < TS * NX; idx += blockDim.x) {
            const int s = idx / NX, i = idx - s * NX;
            double v = 0.0;
            if (s < m) {
                const int o = i - (a.pt_l0[t0 + base + s].x - org.x);
                if (o >= 0 && o < W) v = esw[(int64_t)(t0 + base + s) * 3 * W + o];
            }
            sBx[s][i] = v;
        }
        for (int idx = threadIdx.x; idx < TS * 2 * W; idx += blockDim.x) {
            const int s = idx / (2 * W), r = idx - s * 2 * W;
            const double v = s < m ? esw[(int64_t)(t0 + base + s) * 3 * W + W + r] : 0.0;
            if (r < W)
                sKy[s][r] = v;
            else
                sKz[s][r - W] = v;
        }
        for (int idx = threadIdx.x; idx < CB * TS; idx += blockDim.x) {
            const int c = idx / TS, s = idx - c * TS;
            sQ[c][s] = s < m ? a.q_sorted[(int64_t)(c0 + c) * a.rhs_q_stride + t0 + base + s] : 0.0;
        }
        if (threadIdx.x < TS) {
            const int s = threadIdx.x;
            if (s < m) {
                const int4 l0 = a.pt_l0[t0 + base + s];
                sOy[s] = l0.y - org.y;
                sOz[s] = l0.z - org.z;
            } else {
                sOy[s] = sOz[s] = -(1 << 20);
            }
        }
        __syncthreads();
        if (active) {
            for (int s = 0; s < m; ++s) {
                const int dj = jj - sOy[s], dk = kk - sOz[s];
                if (dj < 0 || dj >= W || dk < 0 || dk >= W) continue;
                const double kyz = sKy[s][dj] * sKz[s][dk];
                double f[CB];
#pragma unroll
                for (int c = 0; c < CB; ++c) f[c] = kyz * sQ[c][s];
#pragma unroll
                for (int i = 0; i < NX; ++i) {
                    const double bx = sBx[s][i];
#pragma unroll
                    for (int c = 0; c < CB; ++c) acc[i][c] = fma(f[c], bx, acc[i][c]);
                }
            }
        }
    }
    if (!active) return;
    const int gy = wrap_index(org.y + jj, a.n2), gz = wrap_index(org.z + kk, a.n3);
#pragma unroll
    for (int i = 0; i < NX; ++i) {
        if (i >= ext.x) continue;
        const int gx = wrap_index(org.x + i, a.n1);
        const int64_t cell = ((int64_t)gx * a.n2 + gy) * a.n3 + gz;
#pragma unroll
        for (int c = 0; c < CB; ++c)
            if (acc[i][c] != 0.0) atomicAdd(a.grid + (int64_t)(c0 + c) * a.rhs_grid_stride + cell, acc[i][c]);
    }
}

// Spreading by runs.  One CTA = one bin x CB RHS; thread (dy, dz) of the W x W
// window columns.  For each run (targets sharing the window's (y, z) start,
// ordered by x) the thread accumulates its column's W + kSpreadRunDx x-values
// for CB RHS in registers (each target's x offset selects a compile-time
// register window), then adds them to the bin subgrid in shared memory; at
// the end the subgrid is added to the global grid.  Every multiply-add
// belongs to a (target, tap) pair.
template <int W, int CB, int XO, typename TW>
__device__ __forceinline__ void spread_run_add(TW (&acc)[W + kSpreadRunDx][CB], const TW* __restrict__ wx,
                                               const TW (&f)[CB]) {
#pragma unroll
    for (int ia = 0; ia < W; ++ia) {
        const TW w = wx[ia];
#pragma unroll
        for (int c = 0; c < CB; ++c) acc[XO + ia][c] = fma(f[c], w, acc[XO + ia][c]);
    }
}

// TW: type of the weights, the run accumulators and the bin subgrid (double,
// or float in the mixed-precision path); the global grid stays FP64.
template <int W, int CB, typename TW>
__global__ void __launch_bounds__((W * W + 31) / 32 * 32) k_spread_r(NufftArgs a, const TW* __restrict__ esw) {
    constexpr int NXR = W + kSpreadRunDx;
    constexpr int TS = 32;                  // targets staged at a time
    constexpr int NT = (W * W + 31) / 32 * 32;
    __shared__ TW sW[TS][3 * W];            // weights of the staged targets
    __shared__ TW sQ[TS][CB];               // their charges
    __shared__ int sXo[TS];                 // their x offset in the run
    extern __shared__ __align__(16) unsigned char sub_raw[];
    TW* sub = reinterpret_cast<TW*>(sub_raw);  // [c][x][y][z] over the bin's extents
    const int e = blockIdx.x;
    const int c0 = blockIdx.y * CB;
    const int4 org = a.sub_origin[e], ext = a.sub_extent[e];
    const int ncell = ext.x * ext.y * ext.z;
    for (int i = threadIdx.x; i < ncell * CB; i += NT) sub[i] = TW(0);
    const bool active = threadIdx.x < W * W;
    const int dy = threadIdx.x / W, dz = threadIdx.x % W;
    for (int r = a.bin_run[e]; r < a.bin_run[e + 1]; ++r) {
        const int4 R = a.spread_run[r];
        TW acc[NXR][CB];
#pragma unroll
        for (int i = 0; i < NXR; ++i)
#pragma unroll
            for (int c = 0; c < CB; ++c) acc[i][c] = TW(0);
        for (int base = 0; base < R.y; base += TS) {
            const int m = min(TS, R.y - base);
            __syncthreads();  // previous chunk (or subgrid flush) done
            for (int i = threadIdx.x; i < m * 3 * W; i += NT) {
                const int k = i / (3 * W), j = i - k * 3 * W;
                const int t = a.spread_order[R.x + base + k];
                sW[k][j] = esw[(int64_t)t * 3 * W + j];
            }
            for (int i = threadIdx.x; i < m * CB; i += NT) {
                const int k = i / CB, c = i - k * CB;
                const int t = a.spread_order[R.x + base + k];
                sQ[k][c] = (TW)a.q_sorted[(int64_t)(c0 + c) * a.rhs_q_stride + t];
            }
            for (int k = threadIdx.x; k < m; k += NT) sXo[k] = a.pt_l0[a.spread_order[R.x + base + k]].x - org.x - R.w;
            __syncthreads();
            if (active) {
                for (int k = 0; k < m; ++k) {
                    const TW wyz = sW[k][W + dy] * sW[k][2 * W + dz];
                    TW f[CB];
#pragma unroll
                    for (int c = 0; c < CB; ++c) f[c] = wyz * sQ[k][c];
                    switch (sXo[k]) {
                        case 0: spread_run_add<W, CB, 0, TW>(acc, sW[k], f); break;
                        case 1: spread_run_add<W, CB, 1, TW>(acc, sW[k], f); break;
                        case 2: spread_run_add<W, CB, 2, TW>(acc, sW[k], f); break;
                        case 3: spread_run_add<W, CB, 3, TW>(acc, sW[k], f); break;
                        default: spread_run_add<W, CB, 4, TW>(acc, sW[k], f); break;
                    }
                }
            }
        }
        __syncthreads();  // every thread of the previous run has flushed
        if (active) {
            const int y = (R.z & 0xFFFF) + dy, z = (R.z >> 16) + dz;
#pragma unroll
            for (int i = 0; i < NXR; ++i) {
                const int x = R.w + i;
                if (x >= ext.x) break;
#pragma unroll
                for (int c = 0; c < CB; ++c) sub[((c * ext.x + x) * ext.y + y) * ext.z + z] += acc[i][c];
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ncell * CB; i += NT) {
        const double v = (double)sub[i];
        if (v == 0.0) continue;
        const int c = i / ncell, cell = i - c * ncell;
        const int x = cell / (ext.y * ext.z), yz = cell - x * (ext.y * ext.z);
        const int y = yz / ext.z, z = yz - y * ext.z;
        const int64_t g = ((int64_t)wrap_index(org.x + x, a.n1) * a.n2 + wrap_index(org.y + y, a.n2)) * a.n3 +
                          wrap_index(org.z + z, a.n3);
        atomicAdd(a.grid + (int64_t)(c0 + c) * a.rhs_grid_stride + g, v);
    }
}

// interpolation of the it-th target of the visit order, RHS c0 .. c0 + CB - 1
template <int W, int CB>
__device__ __forceinline__ void interp_target(const NufftArgs& a, const double* __restrict__ esw, int64_t it, int c0) {
    const int64_t t = a.interp_order ? a.interp_order[it] : it;
    const int4 l0 = a.pt_l0[t];
    const double* wt = esw + t * 3 * W;
    double wy[W], wz[W];
    int iy[W], iz[W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
        wy[c] = wt[W + c];
        wz[c] = wt[2 * W + c];
        iy[c] = wrap_index(l0.y + c, a.n2);
        iz[c] = wrap_index(l0.z + c, a.n3);
    }
    const double* g0 = a.grid + (int64_t)c0 * a.rhs_grid_stride;
    double u[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) u[c] = 0.0;
    // x taps stay rolled (weights re-read from L1) so that the y/z tap arrays stay in registers
#pragma unroll 1
    for (int ia = 0; ia < W; ++ia) {
        const double wxa = wt[ia];
        const int64_t gx = (int64_t)wrap_index(l0.x + ia, a.n1) * a.n2;
#pragma unroll
        for (int ib = 0; ib < W; ++ib) {
            const double wxy = wxa * wy[ib];
            const double* row = g0 + (gx + iy[ib]) * a.n3;
#pragma unroll
            for (int ic = 0; ic < W; ++ic) {
                const double w = wxy * wz[ic];
                const double* p = row + iz[ic];
#pragma unroll
                for (int c = 0; c < CB; ++c) u[c] = fma(w, __ldg(p + (int64_t)c * a.rhs_grid_stride), u[c]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < CB; ++c) a.far[(int64_t)(c0 + c) * a.rhs_far_stride + t] = u[c];
}

template <int W, int CB>
__global__ void __launch_bounds__(128) k_interp_m(NufftArgs a, const double* __restrict__ esw, int64_t n) {
    const int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    interp_target<W, CB>(a, esw, it, blockIdx.y * CB);
}

// many systems' interpolations in one grid (one RHS): item = (system, block of 128 targets)
template <int W>
__global__ void __launch_bounds__(128) k_interp_batch(const InterpSys* __restrict__ sys, const int2* __restrict__ items) {
    const int2 w = items[blockIdx.x];
    const InterpSys& S = sys[w.x];
    const int64_t it = (int64_t)w.y * 128 + threadIdx.x;
    if (it >= S.n) return;
    interp_target<W, 1>(S.a, S.esw, it, 0);
}

// Interpolation from each bin's subgrid in shared memory: one CTA per bin,
// looping over the RHS in blocks of CB.  The CTA copies the ext.x x ext.y x
// ext.z cells of a block's CB RHS planes into shared memory as [RHS pair]
// [cell][2] with asynchronous 8-byte copies, the next block's copies in flight
// while the current block is interpolated (two buffers).  Each thread owns one
// pair of targets whose windows start at the same cell and keeps their y/z
// weights in registers across the blocks: every 16-byte load (two RHS) feeds
// four FMAs, half the bytes per FMA of one target per thread (shared-memory
// and L1 delivery, 128 B per clock, bound the one-target kernel).  Taps and
// FMA order per target are those of k_interp_m, so the results agree bit for
// bit.  Bins with more cells than cap_cells are left to k_interp_big, which
// reads the grid directly.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int W, int CB>
__device__ __forceinline__ void interp_direct(const NufftArgs& a, const double* esw, const double* g0, int t,
                                              double (&u)[CB]) {
    const int4 l0 = a.pt_l0[t];
    const double* wt = esw + (int64_t)t * 3 * W;
    double wy[W], wz[W];
    int iy[W], iz[W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
        wy[c] = wt[W + c];
        wz[c] = wt[2 * W + c];
        iy[c] = wrap_index(l0.y + c, a.n2);
        iz[c] = wrap_index(l0.z + c, a.n3);
    }
#pragma unroll
    for (int c = 0; c < CB; ++c) u[c] = 0.0;
#pragma unroll 1
    for (int ia = 0; ia < W; ++ia) {
        const double wxa = wt[ia];
        const int64_t gx = (int64_t)wrap_index(l0.x + ia, a.n1) * a.n2;
#pragma unroll
        for (int ib = 0; ib < W; ++ib) {
            const double wxy = wxa * wy[ib];
            const double* row = g0 + (gx + iy[ib]) * a.n3;
#pragma unroll
            for (int ic = 0; ic < W; ++ic) {
                const double w = wxy * wz[ic];
                const double* p = row + iz[ic];
#pragma unroll
                for (int c = 0; c < CB; ++c) u[c] = fma(w, __ldg(p + (int64_t)c * a.rhs_grid_stride), u[c]);
            }
        }
    }
}

template <int W, int CB>
__global__ void __launch_bounds__(256, 2)
    k_interp_s(NufftArgs a, const double* __restrict__ esw, int cap_cells, int nblocks) {
    static_assert(CB % 2 == 0, "RHS pairs");
    extern __shared__ __align__(16) double sub[];  // [2 buffers][CB / 2][cap_cells][2]
    const int e = blockIdx.x;
    const int4 org = a.sub_origin[e], ext = a.sub_extent[e];
    const int eyz = ext.y * ext.z, ncell = ext.x * eyz;
    if (ncell > cap_cells) return;
    const int bufsz = CB * cap_cells;
    // asynchronous copies of RHS block b into buffer b & 1 (one commit group)
    auto stage = [&](int b) {
        const double* gb = a.grid + (int64_t)b * CB * a.rhs_grid_stride;
        double* dst = sub + (b & 1) * bufsz;
        for (int i = threadIdx.x; i < CB * ncell; i += blockDim.x) {
            const int h = i & 1, r = i >> 1;
            const int j = r / ncell, cell = r - j * ncell;
            const int x = cell / eyz, yz = cell - x * eyz;
            const int y = yz / ext.z, z = yz - y * ext.z;
            const int64_t g = ((int64_t)wrap_index(org.x + x, a.n1) * a.n2 + wrap_index(org.y + y, a.n2)) * a.n3 +
                              wrap_index(org.z + z, a.n3);
            cp_async8(dst + i, gb + (int64_t)(2 * j + h) * a.rhs_grid_stride + g);
        }
        cp_async_commit_group();
    };
    const int p0 = a.bin_pair[e], p1 = a.bin_pair[e + 1];
    for (int base = p0; base < p1; base += blockDim.x) {  // the same trip count for all threads
        const int ip = base + (int)threadIdx.x;
        const bool act = ip < p1;
        const int2 tp = act ? a.interp_pair[ip] : make_int2(0, -1);
        const bool two = tp.y >= 0;
        int lx = 0, ly = 0, lz = 0;
        const double* wa = esw;
        const double* wb = esw;
        double wya[W], wza[W], wyb[W], wzb[W];
#pragma unroll
        for (int c = 0; c < W; ++c) wya[c] = wza[c] = wyb[c] = wzb[c] = 0.0;
        if (act) {
            const int4 l0 = a.pt_l0[tp.x];
            lx = l0.x - org.x;
            ly = l0.y - org.y;
            lz = l0.z - org.z;
            wa = esw + (int64_t)tp.x * 3 * W;
            wb = esw + (int64_t)(two ? tp.y : tp.x) * 3 * W;
#pragma unroll
            for (int c = 0; c < W; ++c) {
                wya[c] = wa[W + c];
                wza[c] = wa[2 * W + c];
                wyb[c] = two ? wb[W + c] : 0.0;
                wzb[c] = wb[2 * W + c];
            }
        }
        stage(0);
        for (int b = 0; b < nblocks; ++b) {
            if (b + 1 < nblocks) {
                stage(b + 1);
                cp_async_wait_group<1>();
            } else {
                cp_async_wait_group<0>();
            }
            __syncthreads();
            if (act) {
                const double2* s2 = reinterpret_cast<const double2*>(sub + (b & 1) * bufsz);
                double ua[CB], ub[CB];
#pragma unroll
                for (int c = 0; c < CB; ++c) ua[c] = ub[c] = 0.0;
#pragma unroll 1
                for (int ia = 0; ia < W; ++ia) {
                    const double wxa = wa[ia], wxb = wb[ia];
                    const int rx = (lx + ia) * ext.y + ly;
#pragma unroll
                    for (int ib = 0; ib < W; ++ib) {
                        const double wxya = wxa * wya[ib], wxyb = wxb * wyb[ib];
                        const int row = (rx + ib) * ext.z + lz;
#pragma unroll
                        for (int ic = 0; ic < W; ++ic) {
                            const double w0 = wxya * wza[ic], w1 = wxyb * wzb[ic];
#pragma unroll
                            for (int j = 0; j < CB / 2; ++j) {
                                const double2 v = s2[j * ncell + row + ic];
                                ua[2 * j] = fma(w0, v.x, ua[2 * j]);
                                ua[2 * j + 1] = fma(w0, v.y, ua[2 * j + 1]);
                                ub[2 * j] = fma(w1, v.x, ub[2 * j]);
                                ub[2 * j + 1] = fma(w1, v.y, ub[2 * j + 1]);
                            }
                        }
                    }
                }
                const int c0 = b * CB;
#pragma unroll
                for (int c = 0; c < CB; ++c) a.far[(int64_t)(c0 + c) * a.rhs_far_stride + tp.x] = ua[c];
                if (two)
#pragma unroll
                    for (int c = 0; c < CB; ++c) a.far[(int64_t)(c0 + c) * a.rhs_far_stride + tp.y] = ub[c];
            }
            __syncthreads();
        }
    }
}

// The bins that k_interp_s leaves (more cells than cap_cells): each thread
// interpolates its pair's targets from the grid in global memory.
template <int W, int CB>
__global__ void __launch_bounds__(256) k_interp_big(NufftArgs a, const double* __restrict__ esw, int cap_cells) {
    const int e = blockIdx.x, c0 = blockIdx.y * CB;
    const int4 ext = a.sub_extent[e];
    if (ext.x * ext.y * ext.z <= cap_cells) return;
    const double* g0 = a.grid + (int64_t)c0 * a.rhs_grid_stride;
    for (int ip = a.bin_pair[e] + (int)threadIdx.x; ip < a.bin_pair[e + 1]; ip += blockDim.x) {
        const int2 tp = a.interp_pair[ip];
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
            const int t = k == 0 ? tp.x : tp.y;
            if (t < 0) break;
            double u[CB];
            interp_direct<W, CB>(a, esw, g0, t, u);
#pragma unroll
            for (int c = 0; c < CB; ++c) a.far[(int64_t)(c0 + c) * a.rhs_far_stride + t] = u[c];
        }
    }
}

constexpr int kInterpCB = 4;                     // RHS per shared-memory interpolation CTA
constexpr size_t kInterpSmemMax = 96 * 1024;     // subgrid bytes per CTA

constexpr size_t kSpreadRunSmem = 100 * 1024;

template <int W, typename TW>
bool spread_run_w(const NufftArgs& a, const TW* esw, int nrhs, cudaStream_t s) {
    if (!(a.spread_run && nrhs % 4 == 0 && (size_t)a.max_cells * 4 * sizeof(TW) <= kSpreadRunSmem)) return false;
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_spread_r<W, 4, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSpreadRunSmem));
        configured[dev] = true;
    }
    const size_t smem = (size_t)a.max_cells * 4 * sizeof(TW);
    k_spread_r<W, 4, TW><<<dim3(a.n_leaves, nrhs / 4), (W * W + 31) / 32 * 32, smem, s>>>(a, esw);
    return true;
}

template <int W>
void spread_w(const NufftArgs& a, const double* esw, int max_jk, int max_ex, int nrhs, cudaStream_t s) {
    if (spread_run_w<W, double>(a, esw, nrhs, s)) return;
    const int yb = (max_jk + 127) / 128;
    if (max_ex <= 12) {
        if (nrhs % 4 == 0) {
            k_spread_m<W, 12, 4><<<dim3(a.n_leaves, yb, nrhs / 4), 128, 0, s>>>(a, esw);
            return;
        }
        k_spread_m<W, 12, 1><<<dim3(a.n_leaves, yb, nrhs), 128, 0, s>>>(a, esw);
    } else if (max_ex <= 16) {
        if (nrhs % 4 == 0) {
            k_spread_m<W, 16, 4><<<dim3(a.n_leaves, yb, nrhs / 4), 128, 0, s>>>(a, esw);
            return;
        }
        k_spread_m<W, 16, 1><<<dim3(a.n_leaves, yb, nrhs), 128, 0, s>>>(a, esw);
    } else if (max_ex <= 32) {
        if (nrhs % 2 == 0) {
            k_spread_m<W, 32, 2><<<dim3(a.n_leaves, yb, nrhs / 2), 128, 0, s>>>(a, esw);
            return;
        }
        k_spread_m<W, 32, 1><<<dim3(a.n_leaves, yb, nrhs), 128, 0, s>>>(a, esw);
    } else if (max_ex <= 48) {
        k_spread_m<W, 48, 1><<<dim3(a.n_leaves, yb, nrhs), 128, 0, s>>>(a, esw);
    } else {
        throw std::runtime_error("NUFFT leaf subgrid too large");
    }
}

template <int W>
void interp_w(const NufftArgs& a, const double* esw, int64_t n, int nrhs, cudaStream_t s) {
    // windows up to 9 taps keep the staged kernel within 128 registers (two CTAs per SM)
    if constexpr (W <= 9) if (nrhs % kInterpCB == 0 && a.interp_pair && a.bin_pair && a.n_leaves > 0 && a.max_cells > 0) {
        const int cap = (int)std::min<int64_t>(a.max_cells, kInterpSmemMax / (2 * kInterpCB * sizeof(double)));
        static bool configured[64] = {};
        int dev = 0;
        PDMK_CUDA_CHECK(cudaGetDevice(&dev));
        if (dev >= 0 && dev < 64 && !configured[dev]) {
            PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_interp_s<W, kInterpCB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)kInterpSmemMax));
            configured[dev] = true;
        }
        const size_t smem = 2 * (size_t)cap * kInterpCB * sizeof(double);
        // one pass over a bin's pairs: threads = its pair count, whole warps, at most 256
        const int nt = std::min(256, std::max(64, (a.max_pairs + 31) / 32 * 32));
        k_interp_s<W, kInterpCB><<<a.n_leaves, nt, smem, s>>>(a, esw, cap, nrhs / kInterpCB);
        if (a.max_cells > cap) k_interp_big<W, kInterpCB><<<dim3(a.n_leaves, nrhs / kInterpCB), nt, 0, s>>>(a, esw, cap);
        return;
    }
    const unsigned bx = (unsigned)((n + 127) / 128);
    if (nrhs % 8 == 0)
        k_interp_m<W, 8><<<dim3(bx, nrhs / 8), 128, 0, s>>>(a, esw, n);
    else
        k_interp_m<W, 1><<<dim3(bx, nrhs), 128, 0, s>>>(a, esw, n);
}

}  // namespace

#define PDMK_NUFFT_W_SWITCH(W_, CALL)                                                                   \
    switch (W_) {                                                                                       \
        case 4: CALL(4); break;                                                                         \
        case 5: CALL(5); break;                                                                         \
        case 6: CALL(6); break;                                                                         \
        case 7: CALL(7); break;                                                                         \
        case 8: CALL(8); break;                                                                         \
        case 9: CALL(9); break;                                                                         \
        case 10: CALL(10); break;                                                                       \
        case 11: CALL(11); break;                                                                       \
        case 12: CALL(12); break;                                                                       \
        case 13: CALL(13); break;                                                                       \
        case 14: CALL(14); break;                                                                       \
        default: throw std::runtime_error("unsupported NUFFT kernel width");                            \
    }

void launch_es_weights(const NufftArgs& a, int64_t n, double* w, cudaStream_t s) {
    if (n <= 0) return;
    const unsigned blocks = (unsigned)((n + 255) / 256);
#define PDMK_ESW(W) k_es_weights<W><<<blocks, 256, 0, s>>>(a, n, w)
    PDMK_NUFFT_W_SWITCH(a.w, PDMK_ESW)
#undef PDMK_ESW
}

void launch_spread_multi(const NufftArgs& a, const double* esw, int max_jk, int max_ex, int nrhs, cudaStream_t s) {
    if (a.n_leaves <= 0 || nrhs <= 0) return;
#define PDMK_SPW(W) spread_w<W>(a, esw, max_jk, max_ex, nrhs, s)
    PDMK_NUFFT_W_SWITCH(a.w, PDMK_SPW)
#undef PDMK_SPW
}

void launch_interp_multi(const NufftArgs& a, const double* esw, int64_t n, int nrhs, cudaStream_t s) {
    if (n <= 0 || nrhs <= 0) return;
#define PDMK_INW(W) interp_w<W>(a, esw, n, nrhs, s)
    PDMK_NUFFT_W_SWITCH(a.w, PDMK_INW)
#undef PDMK_INW
}

void launch_batch_interp(const InterpSys* sys, const int2* items, int n_items, int w, cudaStream_t s) {
    if (n_items <= 0) return;
#define PDMK_IB(W) k_interp_batch<W><<<n_items, 128, 0, s>>>(sys, items)
    PDMK_NUFFT_W_SWITCH(w, PDMK_IB)
#undef PDMK_IB
    PDMK_CUDA_CHECK(cudaGetLastError());
}

bool launch_spread_multi_f32(const NufftArgs& a, const float* esw32, int nrhs, cudaStream_t s) {
    if (a.n_leaves <= 0 || nrhs <= 0) return true;
    bool done = false;
#define PDMK_SPF(W) done = spread_run_w<W, float>(a, esw32, nrhs, s)
    PDMK_NUFFT_W_SWITCH(a.w, PDMK_SPF)
#undef PDMK_SPF
    return done;
}

#undef PDMK_NUFFT_W_SWITCH

}  // namespace dev
}  // namespace pdmkb
