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
    for (int r = warp; r < kDRows; r += 8) {
        const double* row = in + (int64_t)(r0 + r) * K;
        for (int k = lane; k < 4 * KS; k += 32) sA[r * RS + k] = (r < nr && k < K) ? row[k] : 0.0;
    }
    for (int i = warp; i < 4 * KS; i += 8)
        for (int c = lane; c < 8 * NT; c += 32) sB[i * BS + c] = (i < K && c < N) ? mat[c + (int64_t)N * i] : 0.0;
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

}  // namespace

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
