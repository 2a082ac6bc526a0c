// Near field of many independent systems in one persistent launch.
//
// The batch of independent periodic systems (float trees, one charge vector
// each) runs every system's upward pass, plane-wave levels, leaf evaluation
// and far field on the system's own stream; then this kernel sums the residual
// near field (cpp/src/dmk/pbc_tree.cpp:1442-1681, the pair kernel of
// cpp/include/dmk/vector_kernels.hpp:354-421) of every (system, target leaf)
// work item and, since a leaf's near sum is complete inside its item, writes
// the leaf's final potentials at once: tree part + near sum + far field - self
// term, scattered to user order (cpp/src/dmk/pbc_tree.cpp:1759-1805).
//
// Work distribution: a device queue.  The items are sorted by estimated work
// (targets x sources of the leaf's near pairs, largest first); every CTA of a
// grid sized to fill the GPU takes the next item with one atomicAdd on the
// queue head until the queue is empty (no waits: a CTA that finds the queue
// empty exits).  Pair arithmetic as the float path's near field: double-float
// coordinate differences, FP32 kernel values and per-pair partial sums, FP64
// accumulation per target.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>

#include "batch_near.cuh"
#include "common.cuh"

namespace pdmkb {
namespace dev {

namespace {

// squared gap between a chunk's box and a target box (0 when they overlap)
__device__ __forceinline__ float box_gap2(const float4& lo, const float4& hi, const volatile float* b) {
    const float gx = fmaxf(0.0f, fmaxf(lo.x - b[3], b[0] - hi.x));
    const float gy = fmaxf(0.0f, fmaxf(lo.y - b[4], b[1] - hi.y));
    const float gz = fmaxf(0.0f, fmaxf(lo.z - b[5], b[2] - hi.z));
    return fmaf(gx, gx, fmaf(gy, gy, gz * gz));
}

template <int NC, int TPT>
__global__ void __launch_bounds__(128) k_batch_near(BatchNearArgs a) {
    __shared__ float4 sh[128], sl[128];
    __shared__ float sq[128];
    __shared__ int s_item;
    __shared__ float s_wbox[4][6];  // per warp: bounding box of its targets of the pass
    __shared__ float s_cbox[4][6];  // per warp: its copy of the pass's bounding box
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        __syncthreads();  // the previous item's shared-memory reads are done
        if (threadIdx.x == 0) s_item = atomicAdd(a.head, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const int2 w = a.items[it];
        const NearLeafSys& S = a.sys[w.x];
        const int e = w.y;
        const int t0 = S.trg_start[e], nt = S.trg_count[e];
        const int p0 = S.pair_start[e], p1 = S.pair_start[e + 1];
        for (int base = 0; base < nt; base += TPT * 128) {
            float4 th[TPT], tl[TPT];
            double acc[TPT];
            float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                const int t = base + threadIdx.x + u * 128;
                th[u] = t < nt ? S.trg_hi[t0 + t] : make_float4(1e30f, 1e30f, 1e30f, 0.f);
                tl[u] = t < nt ? S.trg_lo[t0 + t] : make_float4(0.f, 0.f, 0.f, 0.f);
                acc[u] = 0.0;
                if (t < nt) {
                    lo[0] = fminf(lo[0], th[u].x); hi[0] = fmaxf(hi[0], th[u].x);
                    lo[1] = fminf(lo[1], th[u].y); hi[1] = fmaxf(hi[1], th[u].y);
                    lo[2] = fminf(lo[2], th[u].z); hi[2] = fmaxf(hi[2], th[u].z);
                }
            }
            // target boxes of the warps and of the pass, widened by the FP32
            // rounding of the hi-part coordinates (relative 2^-23)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                    hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
                }
            if (lane == 0)
                for (int d = 0; d < 3; ++d) {
                    const float pad = 2.5e-7f * fmaxf(fabsf(lo[d]), fabsf(hi[d])) + 1e-30f;
                    s_wbox[warp][d] = lo[d] - pad;
                    s_wbox[warp][3 + d] = hi[d] + pad;
                }
            __syncthreads();
            if (lane == 0)
                for (int d = 0; d < 3; ++d) {
                    s_cbox[warp][d] = fminf(fminf(s_wbox[0][d], s_wbox[1][d]), fminf(s_wbox[2][d], s_wbox[3][d]));
                    s_cbox[warp][3 + d] =
                        fmaxf(fmaxf(s_wbox[0][3 + d], s_wbox[1][3 + d]), fmaxf(s_wbox[2][3 + d], s_wbox[3][3 + d]));
                }
            __syncwarp();
            // the boxes stay in shared memory (read once per chunk test) rather
            // than in 12 registers through the pair loop: 64 registers instead
            // of 80 at two targets per thread, 8 CTAs per SM instead of 6
            const volatile float* wbox = s_wbox[warp];
            const volatile float* cbox = s_cbox[warp];
            for (int pr = p0; pr < p1; ++pr) {
                const int s0 = S.pair_src_start[pr], ns = S.pair_src_count[pr];
                const double bd = S.pair_bsize[pr];
                const float d2max = (float)(bd * bd), rsc = (float)(2.0 / bd), cen = (float)(-0.5 * bd);
                const float keep2 = d2max * 1.00001f;
                const int cb = S.pair_chunk_base[pr];
                float part[TPT];
#pragma unroll
                for (int u = 0; u < TPT; ++u) part[u] = 0.f;
                for (int sb = 0; sb < ns; sb += 128) {
                    // 32-source chunks of this block that come within b of the pass's
                    // targets (the same answer in every thread: the skip is uniform)
                    const int nchk = min(4, (ns - sb + 31) / 32);
                    unsigned need = 0;
                    for (int k = 0; k < nchk; ++k) {
                        const int c = cb + (sb >> 5) + k;
                        if (box_gap2(__ldg(S.chunk_lo + c), __ldg(S.chunk_hi + c), cbox) <= keep2) need |= 1u << k;
                    }
                    if (!need) continue;
                    __syncthreads();
                    const int js = sb + threadIdx.x;
                    if (js < ns && ((need >> (threadIdx.x >> 5)) & 1u)) {
                        sh[threadIdx.x] = S.src_hi[s0 + js];
                        sl[threadIdx.x] = S.src_lo[s0 + js];
                        sq[threadIdx.x] = S.src_q[s0 + js];
                    }
                    __syncthreads();
                    const int m = min(128, ns - sb);
                    for (int k = 0; k < nchk; ++k) {
                        if (!((need >> k) & 1u)) continue;
                        const int c = cb + (sb >> 5) + k;
                        // this warp's targets against the chunk (warp-uniform)
                        if (box_gap2(__ldg(S.chunk_lo + c), __ldg(S.chunk_hi + c), wbox) > keep2) continue;
                        const int je = min(m, 32 * k + 32);
                        for (int j = 32 * k; j < je; ++j) {
                            const float4 yh = sh[j], yl = sl[j];
                            const float qj = sq[j];
#pragma unroll
                            for (int u = 0; u < TPT; ++u) {
                                const float dx = (th[u].x - yh.x) + (tl[u].x - yl.x);
                                const float dy = (th[u].y - yh.y) + (tl[u].y - yl.y);
                                const float dz = (th[u].z - yh.z) + (tl[u].z - yl.z);
                                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                                if (r2 > 1e-30f && r2 < d2max) {
                                    const float rinv = rsqrtf(r2);
                                    const float x = fmaf(r2, rinv, cen) * rsc;
                                    float pv = a.coef32[NC - 1];
#pragma unroll
                                    for (int i = NC - 2; i >= 0; --i) pv = fmaf(pv, x, a.coef32[i]);
                                    part[u] = fmaf(pv * rinv, qj, part[u]);
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < TPT; ++u) acc[u] += (double)part[u];
            }
            // final gather of this leaf's targets: tree part + near + far - self
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                const int t = base + threadIdx.x + u * 128;
                if (t < nt) {
                    const int i = t0 + t;
                    S.out[S.perm[i]] = S.pot[i] + acc[u] + S.far[i] - S.trg[i].w * S.q_t[i];
                }
            }
            __syncthreads();  // s_wbox is rewritten by the next pass
        }
    }
}

template <int TPT>
void launch_tpt(const BatchNearArgs& a, int nc, int ctas, cudaStream_t s) {
    switch (nc) {
#define PDMK_BN(NC) \
    case NC: k_batch_near<NC, TPT><<<ctas, 128, 0, s>>>(a); break;
        PDMK_BN(5) PDMK_BN(6) PDMK_BN(9) PDMK_BN(11) PDMK_BN(12) PDMK_BN(15) PDMK_BN(17) PDMK_BN(18) PDMK_BN(22)
        PDMK_BN(23) PDMK_BN(25)
#undef PDMK_BN
        default: throw std::runtime_error("unsupported residual polynomial length");
    }
}

template <int TPT>
int occupancy_tpt(int nc) {
    int blocks = 0;
    switch (nc) {
#define PDMK_BO(NC)                                                                                          \
    case NC:                                                                                                 \
        PDMK_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_batch_near<NC, TPT>, 128, 0)); \
        break;
        PDMK_BO(5) PDMK_BO(6) PDMK_BO(9) PDMK_BO(11) PDMK_BO(12) PDMK_BO(15) PDMK_BO(17) PDMK_BO(18) PDMK_BO(22)
        PDMK_BO(23) PDMK_BO(25)
#undef PDMK_BO
        default: throw std::runtime_error("unsupported residual polynomial length");
    }
    return std::max(1, blocks);
}

}  // namespace

int batch_near_ctas(int nc, int tpt) {
    int dev = 0, sms = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    PDMK_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int occ = tpt == 1 ? occupancy_tpt<1>(nc) : tpt == 2 ? occupancy_tpt<2>(nc) : occupancy_tpt<4>(nc);
    return sms * occ;
}

void launch_batch_near(const BatchNearArgs& a, int nc, int tpt, int ctas, cudaStream_t s) {
    if (a.n_items <= 0) return;
    PDMK_CUDA_CHECK(cudaMemsetAsync(a.head, 0, sizeof(int), s));
    switch (tpt) {
        case 1: launch_tpt<1>(a, nc, ctas, s); break;
        case 2: launch_tpt<2>(a, nc, ctas, s); break;
        case 4: launch_tpt<4>(a, nc, ctas, s); break;
        default: throw std::invalid_argument("targets per thread must be 1, 2 or 4");
    }
}

}  // namespace dev
}  // namespace pdmkb
