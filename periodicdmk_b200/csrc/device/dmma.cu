// FP64 child <-> parent translation steps on the FP64 tensor cores (DMMA,
// mma.sync.aligned.m8n8k4.f64; tcgen05 has no f64 kind).  One separable step
// of cpp/src/dmk/tensorprod.cpp:39-75 in the convention of the CUDA-core
// contraction (ContractArgs): out[e][r + R a] (+)= sum_i M[a + na i] in[e][i + ni r].
//
// A CTA of 8 warps owns 128 rows r of one entry (16 per warp: two 8-row MMA
// tiles) and every output column a (8-column MMA tiles); the rows' inputs and
// the matrix sit in shared memory with strides that spread the fragment loads
// over the banks.  The parent/child matrices are triangular (entries outside
// the triangle are rounding-level zeros, as the CUDA-core kernel uses too), so
// each 8-column tile runs only the 4-wide steps of the contracted index that
// meet its triangle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>

#include "common.cuh"
#include "dmma.cuh"

namespace pdmkb {
namespace dev {

namespace {

constexpr int kDRows = 128;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// S: 0 dense, 1 upper (M(a,i) = 0 for i > a), 2 lower (M(a,i) = 0 for i < a); NT: column tiles
template <int S, int NT, bool ACC>
__global__ void __launch_bounds__(256) k_translate_dmma(ContractArgs a, int RS, int BS) {
    extern __shared__ __align__(16) double smd[];
    const int K = a.ni, N = a.na, R = a.R;
    const int KS = (K + 3) / 4;
    double* sA = smd;                       // [kDRows][RS]: row r, contracted index i
    double* sB = smd + (size_t)kDRows * RS;  // [4 KS][BS]: contracted index i, column a
    const int e = blockIdx.x, r0 = blockIdx.y * kDRows;
    const int nr = min(kDRows, R - r0);
    const double* in = static_cast<const double*>(a.in) + (a.in_off ? a.in_off[e] : (int64_t)e * a.in_stride);
    double* out = static_cast<double*>(a.out) + (a.out_off ? a.out_off[e] : (int64_t)e * a.out_stride);
    const double* mat = static_cast<const double*>(a.mat) + (a.mat_off ? a.mat_off[e] : 0);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // The tile's input rows are contiguous in global memory: asynchronous
    // 16-byte copies when K is even and the block is 16-byte aligned (the
    // translation tensors are), element loads otherwise; zero padding after.
    const bool vec = (K % 2 == 0) && ((reinterpret_cast<uintptr_t>(in + (int64_t)r0 * K) & 15) == 0) && (RS % 2 == 0);
    if (vec) {
        const int hk = K / 2, nchunk = nr * hk;
        const double* src0 = in + (int64_t)r0 * K;
        for (int c = tid; c < nchunk; c += blockDim.x) {
            const int r = c / hk, k = 2 * (c - r * hk);
            const unsigned dst = (unsigned)__cvta_generic_to_shared(sA + r * RS + k);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src0 + (int64_t)r * K + k) : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        for (int r = warp; r < kDRows; r += 8)
            for (int k = lane; k < 4 * KS; k += 32)
                if (r >= nr || k >= K) sA[r * RS + k] = 0.0;
    } else {
        for (int r = warp; r < kDRows; r += 8) {
            const double* row = in + (int64_t)(r0 + r) * K;
            for (int k = lane; k < 4 * KS; k += 32) sA[r * RS + k] = (r < nr && k < K) ? row[k] : 0.0;
        }
    }
    for (int i = warp; i < 4 * KS; i += 8)
        for (int c = lane; c < 8 * NT; c += 32) sB[i * BS + c] = (i < K && c < N) ? mat[c + (int64_t)N * i] : 0.0;
    if (vec) asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    double acc[2][NT][2];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int t = 0; t < NT; ++t) acc[m][t][0] = acc[m][t][1] = 0.0;
    const int rq = lane >> 2, kq = lane & 3;
    const double* pa0 = sA + (warp * 16 + rq) * RS + kq;
    const double* pa1 = pa0 + 8 * RS;
    const double* pb = sB + kq * BS + rq;
    for (int ks = 0; ks < KS; ++ks) {
        const double x0 = pa0[4 * ks], x1 = pa1[4 * ks];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            if (S == 1 && ks > 2 * t + 1) continue;  // i >= 4 ks > 8 t + 7 >= a
            if (S == 2 && ks < 2 * t) continue;      // i <= 4 ks + 3 < 8 t <= a
            const double b = pb[4 * ks * BS + 8 * t];
            dmma(acc[0][t][0], acc[0][t][1], x0, b);
            dmma(acc[1][t][0], acc[1][t][1], x1, b);
        }
    }
    // D fragment: row rq, columns 2 kq and 2 kq + 1 of each tile
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int r = warp * 16 + m * 8 + rq;
        if (r >= nr) continue;
#pragma unroll
        for (int t = 0; t < NT; ++t)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = 8 * t + 2 * kq + h;
                if (c >= N) continue;
                double* p = out + (int64_t)(r0 + r) + (int64_t)R * c;
                if (ACC) *p += acc[m][t][h];
                else *p = acc[m][t][h];
            }
    }
}

template <int S, int NT>
void launch_s(const ContractArgs& a, cudaStream_t s) {
    const int KS = (a.ni + 3) / 4;
    // strides (in doubles) that spread the fragment loads over the 16 64-bit banks:
    // A rows r = lane/4 at stride RS = 4 (mod 16), B rows i = lane%4 at BS = 8 (mod 16)
    int RS = 4 * KS;
    while (RS % 16 != 4) ++RS;
    int BS = 8 * NT;
    while (BS % 16 != 8) ++BS;
    const size_t smem = sizeof(double) * ((size_t)kDRows * RS + (size_t)4 * KS * BS);
    static bool configured_dev[64] = {};
    int cur_dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&cur_dev));
    bool& configured = configured_dev[cur_dev & 63];
    if (!configured) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_translate_dmma<S, NT, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_translate_dmma<S, NT, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        configured = true;
    }
    if (smem > 200 * 1024) throw std::runtime_error("translation tile exceeds shared memory");
    const dim3 grid(a.n_entries, (a.R + kDRows - 1) / kDRows);
    if (a.mode == kStore)
        k_translate_dmma<S, NT, false><<<grid, 256, smem, s>>>(a, RS, BS);
    else
        k_translate_dmma<S, NT, true><<<grid, 256, smem, s>>>(a, RS, BS);
}

template <int NT>
void launch_nt(const ContractArgs& a, cudaStream_t s) {
    if (a.structure == kTriUpper && a.ni == a.na) return launch_s<1, NT>(a, s);
    if (a.structure == kTriLower && a.ni == a.na) return launch_s<2, NT>(a, s);
    launch_s<0, NT>(a, s);
}

// Proxy moments of the FP64 path for the high orders on the FP64 tensor cores:
// per centre box O[(i,j), k] = sum_s X_i(s) Y_j(s) (q_s Z_k(s)) with X, Y, Z the
// Chebyshev values at the source's scaled coordinates (cpp/src/dmk/proxy.cpp,
// charge-to-proxy), a GEMM with M = P^2 rows r = i + P j, N = P columns k and
// K = the box's sources.  A CTA of 8 warps takes 256 rows (4 row tiles of 8 per
// warp) and all columns (NT tiles of 8); sources are staged 32 at a time as
// their three Chebyshev tables (the charge folded into Z); per 4 sources a
// thread forms its A element X_i Y_j (one product) and NT B elements and the
// warp issues 4 x NT mma.m8n8k4.f64.  Every coefficient is written once (the
// children's translations are added afterwards), as the CUDA-core kernel does.
template <int P>
__global__ void __launch_bounds__(256) k_c2proxy_dmma(C2ProxyArgs a) {
    constexpr int TS = 32, NT = (P + 7) / 8, PN = NT * 8, RT = 4, ROWS = 8 * 8 * RT;
    constexpr int LX = P + 1, LZ = PN + 1;
    __shared__ double sx[TS][LX], sy[TS][LX], sz[TS][LZ];
    const int e = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rq = lane >> 2, kq = lane & 3;
    const int r0 = blockIdx.y * ROWS + warp * 8 * RT;
    int ai[RT], aj[RT];
    bool av[RT];
#pragma unroll
    for (int t = 0; t < RT; ++t) {
        const int r = r0 + 8 * t + rq;
        av[t] = r < P * P;
        ai[t] = av[t] ? r % P : 0;
        aj[t] = av[t] ? r / P : 0;
    }
    double acc[RT][NT][2];
#pragma unroll
    for (int t = 0; t < RT; ++t)
#pragma unroll
        for (int c = 0; c < NT; ++c) acc[t][c][0] = acc[t][c][1] = 0.0;
    const double4 cs = a.center_scale[e];
    for (int rg = a.rng_start[e]; rg < a.rng_start[e + 1]; ++rg) {
        const int s0 = a.src_start[rg], ns = a.src_count[rg];
        for (int base = 0; base < ns; base += TS) {
            const int nt = min(TS, ns - base);
            __syncthreads();
            for (int task = threadIdx.x; task < 3 * TS; task += blockDim.x) {
                const int si = task % TS, d = task / TS;
                double* dst = d == 0 ? sx[si] : (d == 1 ? sy[si] : sz[si]);
                const int len = d == 2 ? PN : P;
                if (si < nt) {
                    const double4 pt = a.src[s0 + base + si];
                    const double x = (d == 0 ? pt.x - cs.x : (d == 1 ? pt.y - cs.y : pt.z - cs.z)) * cs.w;
                    const double mult = d == 2 ? pt.w : 1.0;  // the charge folded into the z factor
                    double t0 = 1.0, t1 = x;
                    dst[0] = mult;
                    dst[1] = mult * x;
                    for (int n = 2; n < P; ++n) {
                        const double t2 = 2.0 * x * t1 - t0;
                        dst[n] = mult * t2;
                        t0 = t1;
                        t1 = t2;
                    }
                    for (int n = P; n < len; ++n) dst[n] = 0.0;
                } else {
                    for (int n = 0; n < len; ++n) dst[n] = 0.0;
                }
            }
            __syncthreads();
            const int nks = (nt + 3) / 4;
            for (int ks = 0; ks < nks; ++ks) {
                const int s = 4 * ks + kq;
                double b[NT];
#pragma unroll
                for (int c = 0; c < NT; ++c) b[c] = sz[s][8 * c + rq];
#pragma unroll
                for (int t = 0; t < RT; ++t) {
                    const double x = sx[s][ai[t]] * sy[s][aj[t]];
                    const double av_t = av[t] ? x : 0.0;
#pragma unroll
                    for (int c = 0; c < NT; ++c) dmma(acc[t][c][0], acc[t][c][1], av_t, b[c]);
                }
            }
        }
    }
    double* out = a.proxy_up + (int64_t)a.slot[e] * (P * P * P);
#pragma unroll
    for (int t = 0; t < RT; ++t) {
        const int r = r0 + 8 * t + rq;
        if (r >= P * P) continue;
#pragma unroll
        for (int c = 0; c < NT; ++c)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = 8 * c + 2 * kq + h;
                if (k < P) out[r + (int64_t)P * P * k] = acc[t][c][h];
            }
    }
}

}  // namespace

bool c2proxy_dmma_supported(int p) { return p == 28 || p == 38; }

void launch_c2proxy_dmma(const C2ProxyArgs& a, int p, cudaStream_t s) {
    if (a.n_centers <= 0) return;
    switch (p) {
        case 28: k_c2proxy_dmma<28><<<dim3(a.n_centers, (28 * 28 + 255) / 256), 256, 0, s>>>(a); break;
        case 38: k_c2proxy_dmma<38><<<dim3(a.n_centers, (38 * 38 + 255) / 256), 256, 0, s>>>(a); break;
        default: throw std::runtime_error("moments order not covered");
    }
}

bool translate_dmma_supported(int ni, int na) { return ni > 0 && na > 0 && ni <= 64 && na <= 40; }

void launch_translate_dmma(const ContractArgs& a, cudaStream_t s) {
    if (a.n_entries <= 0) return;
    if (a.mode != kStore && a.mode != kAdd) throw std::invalid_argument("translation: store or add only");
    if (!translate_dmma_supported(a.ni, a.na)) throw std::runtime_error("translation shape not covered");
    switch ((a.na + 7) / 8) {
        case 1: launch_nt<1>(a, s); break;
        case 2: launch_nt<2>(a, s); break;
        case 3: launch_nt<3>(a, s); break;
        case 4: launch_nt<4>(a, s); break;
        default: launch_nt<5>(a, s); break;
    }
}

}  // namespace dev
}  // namespace pdmkb
