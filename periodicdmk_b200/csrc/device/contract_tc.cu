// One step of a separable tensor transform on the tcgen05 tensor cores; the
// contract is in contract_tc.cuh.  These are the c2p / p2c translations
// (cpp/src/dmk/tensorprod.cpp:39-75), the proxy -> outgoing plane-wave steps
// (cpp/src/dmk/proxy.cpp:42-90) and the incoming plane-wave -> proxy steps
// (cpp/src/dmk/planewave.cpp:49-105) of the mixed-precision path.
//
// One CTA of 128 threads per (box, RHS) entry: it builds the real form of the
// entry's matrix once as the B operand (TF32 hi / lo parts, K-major, no
// swizzle), then for each 128-row tile of the entry loads the rows (each row's
// K values are contiguous in the input), splits them into TF32 hi / lo in the
// canonical K-major layout, issues hi*hi + hi*lo + lo*hi MMAs (M = 128, N =
// padded na*co, K = 8 per step) into an FP32 tensor-memory accumulator, and
// drains it: thread t owns row t (tensor-memory lane t) and writes its N
// values to the output (store or add).  At most 12 K-steps (K <= 96) run into
// one accumulator, short enough that the tensor-core accumulation error stays
// below the FP32 rounding of the CUDA-core kernels it replaces.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>

#include "common.cuh"
#include "contract_tc.cuh"
#include "tc_util.cuh"

namespace pdmkb {
namespace dev {

namespace {

constexpr int kCMaxK = 96, kCMaxN = 128;

__device__ __forceinline__ float embed(const ContractTc& a, const float* mat, int n, int k, int N, int K) {
    if (n >= N || k >= K) return 0.0f;
    const int ci = a.ci, co = a.co;
    const int ai = n / co, cn = n - ai * co;
    const int i = k / ci, ck = k - i * ci;
    const int64_t m = (int64_t)ai + (int64_t)a.na * i;
    if (!a.mat_complex) return mat[m];
    const float ur = mat[2 * m], ui = mat[2 * m + 1];
    if (ci == 1) return cn == 0 ? ur : ui;                             // real x complex
    if (co == 2) return ck == 0 ? (cn == 0 ? ur : ui) : (cn == 0 ? -ui : ur);  // complex x complex
    return a.scale * (ck == 0 ? ur : -ui);                              // scale * Re(complex x complex)
}

__global__ void __launch_bounds__(128) k_contract_tc(ContractTc a, int KP, int NP, int ncols) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int K = a.ni * a.ci, N = a.na * a.co;
    const int kch = KP / 4;
    const int a_bytes = 128 * KP * 4, b_bytes = NP * KP * 4;
    unsigned char* ahi = sm;
    unsigned char* alo = sm + a_bytes;
    unsigned char* bhi = sm + 2 * a_bytes;
    unsigned char* blo = bhi + b_bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(blo + b_bytes);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(blo + b_bytes + 8);
    volatile int* s_abort = reinterpret_cast<volatile int*>(blo + b_bytes + 12);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t ge = a.e0 + blockIdx.x;
    const int rhs = a.rhs > 0 ? a.rhs : 1;
    const int64_t eb = ge / rhs, ec = ge - eb * rhs;
    const float* in = a.in + (a.in_off ? a.in_off[eb] * rhs + ec * a.in_unit : (int64_t)blockIdx.x * a.in_stride) * a.ci;
    float* out = a.out + (a.out_off ? a.out_off[eb] * rhs + ec * a.out_unit : (int64_t)blockIdx.x * a.out_stride) * a.co;
    const float* mat = a.mat + (a.mat_off ? a.mat_off[eb] : 0) * (a.mat_complex ? 2 : 1);

    if (warp == 0) {
        tc::tmem_alloc(s_tmem, ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        *s_abort = 0;
        tc::fence_mbar_init();
    }
    // B operand: rows n = (a, c_o), K = (i, c_i)
    for (int n = warp; n < NP; n += 4)
        for (int k = lane; k < KP; k += 32) {
            uint32_t h, l;
            tc::split_tf32(embed(a, mat, n, k, N, K), h, l);
            const uint32_t off = tc::kmajor_offset(n, k, kch);
            *reinterpret_cast<uint32_t*>(bhi + off) = h;
            *reinterpret_cast<uint32_t*>(blo + off) = l;
        }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;
    const uint32_t idesc = tc::idesc_tf32(128, NP);
    const uint32_t sbo = (uint32_t)kch * 128;

    const int ntile = (a.R + 127) / 128;
    for (int tile = 0; tile < ntile; ++tile) {
        const int r0 = tile * 128;
        const int nr = min(128, a.R - r0);
        // A operand: row r = input row r0 + r, its K values contiguous
        for (int r = warp; r < 128; r += 4) {
            const float* row = in + (int64_t)(r0 + r) * K;
            for (int k = lane; k < KP; k += 32) {
                const float v = (r < nr && k < K) ? row[k] : 0.0f;
                uint32_t h, l;
                tc::split_tf32(v, h, l);
                const uint32_t off = tc::kmajor_offset(r, k, kch);
                *reinterpret_cast<uint32_t*>(ahi + off) = h;
                *reinterpret_cast<uint32_t*>(alo + off) = l;
            }
        }
        tc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t ab = tc::smem_u32(ahi), al = tc::smem_u32(alo);
            const uint32_t bb = tc::smem_u32(bhi), bl = tc::smem_u32(blo);
            for (int ks = 0; ks < KP / 8; ++ks) {
                const uint32_t ko = ks * 256;
                const uint64_t dah = tc::smem_desc_k_noswizzle(ab + ko, 128, sbo);
                const uint64_t dal = tc::smem_desc_k_noswizzle(al + ko, 128, sbo);
                const uint64_t dbh = tc::smem_desc_k_noswizzle(bb + ko, 128, sbo);
                const uint64_t dbl = tc::smem_desc_k_noswizzle(bl + ko, 128, sbo);
                tc::mma_tf32(tmem, dah, dbh, idesc, ks > 0 ? 1u : 0u);
                tc::mma_tf32(tmem, dah, dbl, idesc, 1u);
                tc::mma_tf32(tmem, dal, dbh, idesc, 1u);
            }
            tc::commit(bar);
        }
        // every thread waits for the tile's MMAs (the A buffer is rewritten next)
        const bool done = tc::mbar_wait(bar, tile & 1);
        if (!done) *s_abort = 1;
        if (!__all_sync(0xffffffffu, done)) {
            // leave the tile loop; the MMAs of this tile are waited for below
        } else {
            tc::fence_after_sync();
            // drain: warp w owns tensor-memory lanes 32 w .. 32 w + 31 = rows
            const int r = warp * 32 + lane;
            const uint32_t base = tmem + ((uint32_t)(warp * 32) << 16);
            for (int n0 = 0; n0 < N; n0 += 8) {
                float v[8];
                tc::tmem_ld_x8(base + (uint32_t)n0, v);
                tc::tmem_wait_ld();
                if (r < nr) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int n = n0 + j;
                        if (n >= N) break;
                        const int ai = n / a.co, c = n - ai * a.co;
                        float* p = out + ((int64_t)(r0 + r) + (int64_t)a.R * ai) * a.co + c;
                        if (a.accumulate) *p += v[j];
                        else *p = v[j];
                    }
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        if (*s_abort) {
            // the bounded wait ran out: wait again (bounded) so that no MMA is in
            // flight when the tensor memory is freed, then report
            tc::mbar_wait(bar, tile & 1);
            break;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, ncols);
    }
    if (*s_abort && tid == 0 && a.err) atomicExch(a.err, 1);
}

}  // namespace

bool contract_tc_supported(int ni, int na, int ci, int co) {
    return ni * ci <= kCMaxK && na * co <= kCMaxN && ni > 0 && na > 0;
}

void launch_contract_tc(const ContractTc& a, cudaStream_t s) {
    if (a.n_entries <= 0 || a.R <= 0) return;
    const int K = a.ni * a.ci, N = a.na * a.co;
    if (!contract_tc_supported(a.ni, a.na, a.ci, a.co)) throw std::runtime_error("contraction shape not covered");
    const int KP = (K + 7) / 8 * 8;
    const int NP = std::max(16, (N + 15) / 16 * 16);
    const int ncols = NP <= 32 ? 32 : NP <= 64 ? 64 : 128;
    const size_t smem = (size_t)2 * 128 * KP * 4 + (size_t)2 * NP * KP * 4 + 64;
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    if (!configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_contract_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             2 * 128 * kCMaxK * 4 + 2 * kCMaxN * kCMaxK * 4 + 64));
        configured[dev] = true;
    }
    k_contract_tc<<<a.n_entries, 128, smem, s>>>(a, KP, NP, ncols);
}

}  // namespace dev
}  // namespace pdmkb
