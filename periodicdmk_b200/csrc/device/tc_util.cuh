// Thin inline-PTX wrappers for the sm_100a 5th-generation tensor cores
// (tcgen05: MMA from shared-memory descriptors into tensor memory, TMEM
// allocation and loads) and mbarriers, used by the generated-operand GEMM
// kernels.  Forms follow the PTX ISA; descriptor bit layouts follow the
// UMMA shared-memory / instruction descriptors.
#pragma once
#include <cstdint>

namespace pdmkb {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- shared-memory matrix descriptor, K-major, no swizzle.
// Canonical layout (16-byte units): ((8 rows, n groups), 2 K-chunks) :
// ((1, SBO), LBO).  lbo / sbo in bytes (multiples of 16).
__device__ __forceinline__ uint64_t smem_desc_k_noswizzle(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    // base offset 0, leading-byte-offset mode 0, layout type 0 (no swizzle)
    return d;
}

// ---- instruction descriptor: kind::tf32, D = F32, A = B = TF32, both K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4)                      // D format F32
           | (2u << 7)                    // A format TF32
           | (2u << 10)                   // B format TF32
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// D[tmem] (+)= A(smem desc) * B(smem desc)^T, issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z));
}

// Arrive on an mbarrier when all previously issued tcgen05 ops of this thread complete.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make generic-proxy shared-memory writes visible to the tensor cores
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- TMEM allocation (one full warp executes these)
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 32-bit, 8 consecutive columns per thread (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld_x8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// 32 lanes x 32-bit, 4 consecutive columns per thread
__device__ __forceinline__ void tmem_ld_x4(uint32_t taddr, float* v) {
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- mbarriers
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false if the phase did not complete within max_cycles SM
// clock cycles (about 2 s at the default budget and B200 clocks).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, long long max_cycles = 4000000000LL) {
    if (mbar_try_wait(mbar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(mbar, parity))
        if (clock64() - t0 > max_cycles) return false;
    return true;
}
// make mbarrier initialisation visible to the async proxy (tensor-core commits)
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// ---- asynchronous global -> shared copies (completion per thread, by group)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- 3xTF32 split: x ~ hi + lo with hi, lo representable in TF32.
// Rounding to the 10-bit TF32 mantissa is done on the bit pattern: adding half
// a TF32 unit (0x1000) and clearing the 13 low bits rounds the magnitude to
// nearest (ties away from zero); a mantissa carry moves into the exponent.
__device__ __forceinline__ uint32_t round_tf32_bits(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = round_tf32_bits(__float_as_uint(x));
    lo = round_tf32_bits(__float_as_uint(x - __uint_as_float(hi)));
}

// Byte offset of element (row, k) of a K-major, no-swizzle operand tile with
// 32-bit elements: 8-row groups of 16-byte K-chunks, LBO = 128 B between the
// K-chunks of one group, SBO = kchunks * 128 B between row groups.
__host__ __device__ constexpr uint32_t kmajor_offset(int row, int k, int kchunks) {
    return (uint32_t)((row >> 3) * (kchunks * 128) + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

}  // namespace tc
}  // namespace pdmkb
