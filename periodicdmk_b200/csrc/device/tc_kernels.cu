// Tensor-core kernels of the mixed-precision multi-RHS path (sm_100a).
//
// Proxy moments (the "charge -> proxy" step of the upward pass, done in the
// reference by a per-box tensor-product sum over sources) for a block of kb
// charge vectors is, per centre box, the product
//     D[(l,c), (i,j)] = sum_s A[(l,c), s] B[(i,j), s]
//     A = T_l(z_s) q_sc,   B = T_i(x_s) T_j(y_s)
// with the source coordinates scaled to the box, T the Chebyshev polynomials.
// Both operands are generated on the fly into shared memory in the UMMA
// K-major no-swizzle layout; the accumulator lives in tensor memory.  Each
// FP32 operand is split into TF32 hi + lo parts and the product is formed as
// hi*hi + hi*lo + lo*hi (three MMAs into one accumulator), which keeps FP32
// accuracy.  Two shared-memory stages alternate: while the tensor core works
// on chunk q, the CTA generates chunk q+1.  Charges and coordinates of the
// next chunk are prefetched into registers; the Chebyshev values of chunk q+1
// are evaluated while chunk q's operands are generated, so one CTA barrier
// per chunk suffices.
#include <stdexcept>

#include "tc_kernels.cuh"
#include "tc_util.cuh"

namespace pdmkb {
namespace dev {

namespace {

constexpr int kKC = 16;       // sources per pipeline stage (two MMA k-steps of 8)
constexpr int kKCH = kKC / 4; // 16-byte K chunks per operand row
constexpr int kThreads = 256;
constexpr int kMaxKb = 64;
constexpr int kMinKb = 16;

template <int P>
struct C2PShape {
    static constexpr int P2 = P * P;
    static constexpr int NB = (P2 + 15) / 16 * 16;  // B rows (i,j), padded to the MMA N granule
    static constexpr int TMEM_COLS = NB <= 32 ? 32 : NB <= 64 ? 64 : NB <= 128 ? 128 : NB <= 256 ? 256 : 512;
    static constexpr int SBO = kKCH * 128;  // bytes between 8-row groups
    static constexpr int A_BYTES = 128 * kKC * 4;
    static constexpr int B_BYTES = NB * kKC * 4;
    static constexpr int OFF_AH = 0, OFF_AL = A_BYTES, OFF_BH = 2 * A_BYTES, OFF_BL = 2 * A_BYTES + B_BYTES;
    static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
    // Chebyshev values of one chunk: [dim][k group][degree][4 sources], two buffers
    static constexpr int T_FLOATS = 3 * kKCH * P * 4;
    static constexpr int OFF_T = 2 * STAGE;
    static constexpr int OFF_BAR = OFF_T + 2 * T_FLOATS * 4;
    static constexpr int SMEM = OFF_BAR + 64;
    static constexpr int A_ITEMS = 128 * kKCH / kThreads;  // (row, k group) items of A per thread
    static constexpr int B_ITEMS = (NB * kKCH + kThreads - 1) / kThreads;
    static_assert(NB <= 512, "accumulator exceeds tensor memory");
    static_assert((128 * kKCH) % kThreads == 0, "A items per thread");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

// (global start, valid count) of chunk q of centre e (chunks do not straddle ranges)
__device__ __forceinline__ void chunk_at(const C2ProxyArgs& a, int r0, int r1, int q, int& g0, int& nt) {
    for (int r = r0; r < r1; ++r) {
        const int ns = a.src_count[r];
        const int nc = (ns + kKC - 1) / kKC;
        if (q < nc) {
            g0 = a.src_start[r] + q * kKC;
            nt = min(kKC, ns - q * kKC);
            return;
        }
        q -= nc;
    }
    g0 = 0;
    nt = 0;
}

__device__ __forceinline__ void split_store(const float4 v, unsigned char* hi_p, unsigned char* lo_p) {
    uint4 hi, lo;
    tc::split_tf32(v.x, hi.x, lo.x);
    tc::split_tf32(v.y, hi.y, lo.y);
    tc::split_tf32(v.z, hi.z, lo.z);
    tc::split_tf32(v.w, hi.w, lo.w);
    *reinterpret_cast<uint4*>(hi_p) = hi;
    *reinterpret_cast<uint4*>(lo_p) = lo;
}

template <int P>
__global__ void __launch_bounds__(kThreads, 1)
    k_c2proxy_tc(C2ProxyArgs a, const float* __restrict__ src_q, float* __restrict__ proxy_up, int kb,
                 int* __restrict__ err) {
    using S = C2PShape<P>;
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);  // MMA completion, one per stage
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + S::OFF_BAR + 16);
    volatile int* s_abort = reinterpret_cast<volatile int*>(sm + S::OFF_BAR + 20);  // [3], sticky
    float* sT = reinterpret_cast<float*>(sm + S::OFF_T);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int e = blockIdx.x;
    const int rows = P * kb;
    const int row0 = blockIdx.y * 128;
    const int r0 = a.rng_start[e], r1 = a.rng_start[e + 1];
    int nchunks = 0;
    for (int r = r0; r < r1; ++r) nchunks += (a.src_count[r] + kKC - 1) / kKC;
    const double4 cs = a.center_scale[e];

    if (warp == 0) {
        tc::tmem_alloc(s_tmem, S::TMEM_COLS);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        s_abort[0] = s_abort[1] = s_abort[2] = 0;
        tc::fence_mbar_init();
    }

    // A rows of this thread: row m = tid % 128, k groups kg0 + 2u (u < A_ITEMS)
    const int am = tid & 127, akg0 = tid >> 7;
    const int aR = row0 + am;
    const bool arow = aR < rows;
    const int al = arow ? aR / kb : 0, ac = arow ? aR - al * kb : 0;
    // Chebyshev role: threads < 3*kKC evaluate one (source, dim) of the next chunk
    const bool cheb = tid < 3 * kKC;
    const int cs_s = tid % kKC, cs_d = tid / kKC;
    const double cs_c = cs_d == 0 ? cs.x : (cs_d == 1 ? cs.y : cs.z);

    auto load_q = [&](int g0, int nt, float (&qv)[S::A_ITEMS][4]) {
#pragma unroll
        for (int u = 0; u < S::A_ITEMS; ++u)
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int s = (akg0 + 2 * u) * 4 + w;
                qv[u][w] = (arow && s < nt) ? __ldg(src_q + (int64_t)(g0 + s) * kb + ac) : 0.0f;
            }
    };
    auto load_x = [&](int g0, int nt) -> double {
        if (!cheb || cs_s >= nt) return 0.0;
        const double* pt = reinterpret_cast<const double*>(a.src + g0 + cs_s);
        return __ldg(pt + cs_d);
    };
    auto cheb_store = [&](int buf, double xv, int nt) {
        if (!cheb) return;
        float* dst = sT + buf * S::T_FLOATS + ((cs_d * kKCH + (cs_s >> 2)) * P) * 4 + (cs_s & 3);
        if (cs_s < nt) {
            const float x = (float)((xv - cs_c) * cs.w);
            float t0 = 1.0f, t1 = x;
            dst[0] = 1.0f;
            dst[4] = x;
#pragma unroll
            for (int n = 2; n < P; ++n) {
                const float t2 = 2.0f * x * t1 - t0;
                dst[4 * n] = t2;
                t0 = t1;
                t1 = t2;
            }
        } else {
#pragma unroll
            for (int n = 0; n < P; ++n) dst[4 * n] = 0.0f;
        }
    };

    float qcur[S::A_ITEMS][4], qnext[S::A_ITEMS][4];
    double xnext = 0.0;
    if (nchunks > 0) {
        int g0, nt;
        chunk_at(a, r0, r1, 0, g0, nt);
        load_q(g0, nt, qcur);
        cheb_store(0, load_x(g0, nt), nt);
        if (nchunks > 1) {
            chunk_at(a, r0, r1, 1, g0, nt);
            xnext = load_x(g0, nt);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;

    int issued = 0;  // chunks whose MMAs were issued and committed
    for (int q = 0; q < nchunks; ++q) {
        const int st = q & 1;
        int g1 = 0, nt1 = 0, g2 = 0, nt2 = 0;
        if (q + 1 < nchunks) {
            chunk_at(a, r0, r1, q + 1, g1, nt1);
            load_q(g1, nt1, qnext);
        }
        if (q + 2 < nchunks) chunk_at(a, r0, r1, q + 2, g2, nt2);
        // stage st was last read by the MMAs of chunk q-2
        if (q >= 2 && !tc::mbar_wait(&bar[st], ((q - 2) >> 1) & 1)) s_abort[st] = 1;
        unsigned char* stage = sm + st * S::STAGE;
        const float* T = sT + st * S::T_FLOATS;
        // A = T_l(z_s) q_sc
#pragma unroll
        for (int u = 0; u < S::A_ITEMS; ++u) {
            const int kg = akg0 + 2 * u;
            const float4 tz = *reinterpret_cast<const float4*>(T + ((2 * kKCH + kg) * P + al) * 4);
            const float4 v = make_float4(tz.x * qcur[u][0], tz.y * qcur[u][1], tz.z * qcur[u][2], tz.w * qcur[u][3]);
            const uint32_t off = tc::kmajor_offset(am, kg * 4, kKCH);
            split_store(v, stage + S::OFF_AH + off, stage + S::OFF_AL + off);
        }
        // B = T_i(x_s) T_j(y_s), rows n = i + P j
#pragma unroll
        for (int u = 0; u < S::B_ITEMS; ++u) {
            const int it = tid + u * kThreads;
            if (it < S::NB * kKCH) {
                const int n = it % S::NB, kg = it / S::NB;
                float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (n < S::P2) {
                    const int i = n % P, j = n / P;
                    const float4 tx = *reinterpret_cast<const float4*>(T + ((0 * kKCH + kg) * P + i) * 4);
                    const float4 ty = *reinterpret_cast<const float4*>(T + ((1 * kKCH + kg) * P + j) * 4);
                    v = make_float4(tx.x * ty.x, tx.y * ty.y, tx.z * ty.z, tx.w * ty.w);
                }
                const uint32_t off = tc::kmajor_offset(n, kg * 4, kKCH);
                split_store(v, stage + S::OFF_BH + off, stage + S::OFF_BL + off);
            }
        }
        // Chebyshev values of chunk q+1 (other buffer), prefetch of chunk q+2's coordinate
        if (q + 1 < nchunks) {
            cheb_store(st ^ 1, xnext, nt1);
            if (q + 2 < nchunks) xnext = load_x(g2, nt2);
        }
        tc::fence_proxy_async();
        __syncthreads();
        if (s_abort[st]) break;
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t base = tc::smem_u32(stage);
#pragma unroll
            for (int ks = 0; ks < kKC / 8; ++ks) {
                const uint32_t kofs = ks * 256;  // 8 K elements = two 16-byte chunks of 128 B each
                const uint64_t ah = tc::smem_desc_k_noswizzle(base + S::OFF_AH + kofs, 128, S::SBO);
                const uint64_t alo = tc::smem_desc_k_noswizzle(base + S::OFF_AL + kofs, 128, S::SBO);
#pragma unroll
                for (int n0 = 0; n0 < S::NB; n0 += 256) {
                    const int N = S::NB - n0 < 256 ? S::NB - n0 : 256;
                    const uint32_t idesc = tc::idesc_tf32(128, N);
                    const uint32_t boff = (uint32_t)(n0 / 8) * S::SBO + kofs;
                    const uint64_t bh = tc::smem_desc_k_noswizzle(base + S::OFF_BH + boff, 128, S::SBO);
                    const uint64_t blo = tc::smem_desc_k_noswizzle(base + S::OFF_BL + boff, 128, S::SBO);
                    const uint32_t d = tmem + (uint32_t)n0;
                    tc::mma_tf32(d, ah, bh, idesc, (q > 0 || ks > 0) ? 1u : 0u);
                    tc::mma_tf32(d, ah, blo, idesc, 1u);
                    tc::mma_tf32(d, alo, bh, idesc, 1u);
                }
            }
            tc::commit(&bar[st]);
        }
        issued = q + 1;
#pragma unroll
        for (int u = 0; u < S::A_ITEMS; ++u)
#pragma unroll
            for (int w = 0; w < 4; ++w) qcur[u][w] = qnext[u][w];
    }
    if (issued > 0) {
        const int ql = issued - 1;
        if (!tc::mbar_wait(&bar[ql & 1], (ql >> 1) & 1)) s_abort[2] = 1;
    }
    __syncthreads();
    const bool ok = s_abort[0] == 0 && s_abort[1] == 0 && s_abort[2] == 0;
    if (ok && issued > 0) {
        tc::fence_after_sync();
        const int quarter = warp & 3, half = warp >> 2;
        const int m = quarter * 32 + lane;
        const int R = row0 + m;
        const bool valid = R < rows;
        float* out = nullptr;
        if (valid) {
            const int l = R / kb, c = R - l * kb;
            out = proxy_up + ((int64_t)a.slot[e] * kb + c) * (P * P * P) + (int64_t)S::P2 * l;
        }
        constexpr int HALF = S::NB / 2;
        static_assert(HALF % 8 == 0, "epilogue column split");
        const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
        for (int c0 = half * HALF; c0 < half * HALF + HALF; c0 += 8) {
            float v[8];
            tc::tmem_ld_x8(lane_addr + (uint32_t)c0, v);
            tc::tmem_wait_ld();
            if (!valid) continue;
            if constexpr (S::P2 % 4 == 0) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int n = c0 + 4 * h;
                    if (n < S::P2) {
                        float4* o = reinterpret_cast<float4*>(out + n);
                        float4 w = *o;
                        w.x += v[4 * h];
                        w.y += v[4 * h + 1];
                        w.z += v[4 * h + 2];
                        w.w += v[4 * h + 3];
                        *o = w;
                    }
                }
            } else {
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (c0 + u < S::P2) out[c0 + u] += v[u];
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, S::TMEM_COLS);
    }
    if (!ok && tid == 0) atomicExch(err, 1);
}

template <int P>
void launch_c2proxy_tc_p(const C2ProxyArgs& a, const float* src_q, float* up, int kb, int* err, cudaStream_t s) {
    using S = C2PShape<P>;
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    if (!configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_c2proxy_tc<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
        configured[dev] = true;
    }
    const dim3 grid(a.n_centers, (P * kb + 127) / 128);
    k_c2proxy_tc<P><<<grid, kThreads, S::SMEM, s>>>(a, src_q, up, kb, err);
}

}  // namespace

bool launch_c2proxy_tc(const C2ProxyArgs& a, const float* src_q, float* proxy_up, int kb, int p, int* err,
                       cudaStream_t s) {
    if (kb < kMinKb || kb > kMaxKb || a.n_centers <= 0) return false;
    switch (p) {
        case 9: launch_c2proxy_tc_p<9>(a, src_q, proxy_up, kb, err, s); return true;
        case 18: launch_c2proxy_tc_p<18>(a, src_q, proxy_up, kb, err, s); return true;
        default: return false;
    }
}

}  // namespace dev
}  // namespace pdmkb
