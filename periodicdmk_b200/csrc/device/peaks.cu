// Throughput probes of the tensor-core paths the roofline figures divide by:
//   * tcgen05 TF32 MMA (kind::tf32, M = 128, N = 256, K = 8, operands in shared
//     memory, FP32 accumulator in tensor memory), one CTA per SM with one
//     issuing thread, as the near-field, moment and leaf-evaluation kernels use
//     it (their 3xTF32 split issues three of these per product);
//   * FP64 DMMA, mma.sync.aligned.m8n8k4 f64 (the only FP64 tensor-core form on
//     sm_100a; tcgen05 has no f64 kind), eight independent accumulators per warp.
// Operand values do not matter for the rate; shared memory is zero-filled.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_util.cuh"

namespace pdmkb {
namespace dev {

namespace {

constexpr int kPK = 32;                        // K elements staged per operand row
constexpr int kPA = 128 * kPK * 4;             // A bytes
constexpr int kPB = 256 * kPK * 4;             // B bytes
constexpr int kPSmem = kPA + kPB + 64;

__global__ void __launch_bounds__(128, 1) k_tf32_probe(int iters, int* err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kPA + kPB);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + kPA + kPB + 16);
    for (int i = threadIdx.x; i < (kPA + kPB) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(sm)[i] = make_uint4(0, 0, 0, 0);
    if (threadIdx.x < 32) {
        tc::tmem_alloc(s_tmem, 256);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;
    bool ok = true;
    if (threadIdx.x == 0) {
        const uint32_t base = tc::smem_u32(sm);
        const uint32_t idesc = tc::idesc_tf32(128, 256);
        const uint32_t sbo = (kPK / 4) * 128;
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int ks = 0; ks < kPK / 8; ++ks) {
                const uint64_t ad = tc::smem_desc_k_noswizzle(base + ks * 256, 128, sbo);
                const uint64_t bd = tc::smem_desc_k_noswizzle(base + kPA + ks * 256, 128, sbo);
                tc::mma_tf32(tmem, ad, bd, idesc, (it | ks) ? 1u : 0u);
            }
        }
        tc::commit(bar);
        // the probe's MMAs take well under a millisecond; the bound only
        // guards against a wait that never completes
        ok = tc::mbar_wait(bar, 0);
        if (!ok) ok = tc::mbar_wait(bar, 0);
        if (!ok) atomicExch(err, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 256);
    }
}

__global__ void __launch_bounds__(256) k_dmma_probe(int iters, double* sink) {
    double acc[8][2];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 0.999;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile(
                "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                : "+d"(acc[i][0]), "+d"(acc[i][1])
                : "d"(a), "d"(b));
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1];
    if (s == -12345.678) sink[threadIdx.x] = s;
}

}  // namespace

double tc_probe_tflops(int kind) {
    int dev = 0, sms = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    PDMK_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    void* buf = nullptr;
    PDMK_CUDA_CHECK(cudaMalloc(&buf, 256 * sizeof(double)));
    PDMK_CUDA_CHECK(cudaMemset(buf, 0, 256 * sizeof(double)));
    cudaEvent_t e0, e1;
    PDMK_CUDA_CHECK(cudaEventCreate(&e0));
    PDMK_CUDA_CHECK(cudaEventCreate(&e1));
    double flops = 0;
    float best = 1e30f;
    if (kind == 0) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_tf32_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, kPSmem));
        const int iters = 4000;
        for (int rep = 0; rep < 4; ++rep) {
            PDMK_CUDA_CHECK(cudaEventRecord(e0));
            k_tf32_probe<<<sms, 128, kPSmem>>>(iters, static_cast<int*>(buf));
            PDMK_CUDA_CHECK(cudaEventRecord(e1));
            PDMK_CUDA_CHECK(cudaEventSynchronize(e1));
            float ms = 0;
            PDMK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) best = std::min(best, ms);
        }
        int flag = 0;
        PDMK_CUDA_CHECK(cudaMemcpy(&flag, buf, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) throw std::runtime_error("CUDA error: tensor-core probe wait timed out");
        flops = 2.0 * 128 * 256 * kPK * (double)iters * sms;
    } else if (kind == 1) {
        const int blocks = sms * 8, threads = 256, iters = 1000;
        for (int rep = 0; rep < 4; ++rep) {
            PDMK_CUDA_CHECK(cudaEventRecord(e0));
            k_dmma_probe<<<blocks, threads>>>(iters, static_cast<double*>(buf));
            PDMK_CUDA_CHECK(cudaEventRecord(e1));
            PDMK_CUDA_CHECK(cudaEventSynchronize(e1));
            float ms = 0;
            PDMK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) best = std::min(best, ms);
        }
        flops = 2.0 * 8 * 8 * 4 * 8 * (double)iters * blocks * (threads / 32);
    } else {
        cudaFree(buf);
        throw std::invalid_argument("unknown probe kind");
    }
    PDMK_CUDA_CHECK(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace dev
}  // namespace pdmkb
