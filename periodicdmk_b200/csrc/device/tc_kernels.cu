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

constexpr int kKC = 32;        // sources per pipeline stage (four MMA k-steps of 8)
constexpr int kKCH = kKC / 4;  // 16-byte K chunks per operand row
constexpr int kSeg = 2;        // chunks accumulated in tensor memory before a drain
constexpr int kThreads = 512;
constexpr int kMaxKb = 64;
constexpr int kMinKb = 16;

// Columns (i, j) < P^2 are split into NSPLIT ranges so that two accumulators
// (one being filled, one being drained) fit in the 512 tensor-memory columns.
template <int P>
struct C2PShape {
    static constexpr int P2 = P * P;
    static constexpr int NSPLIT = 2 * ((P2 + 15) / 16 * 16) <= 512 ? 1 : 2;
    static constexpr int CW = (P2 + NSPLIT - 1) / NSPLIT;  // columns of one CTA
    static constexpr int NB = (CW + 15) / 16 * 16;         // B rows, padded to the MMA N granule
    static constexpr int BUF = NB <= 128 ? 128 : 256;      // column offset of the second accumulator
    static constexpr int TMEM_COLS = 2 * BUF <= 256 ? 256 : 512;
    static constexpr int QCOL = NB / 4;                    // drain columns per thread (four warps per lane quarter)
    static constexpr int SBO = kKCH * 128;
    static constexpr int A_BYTES = 128 * kKC * 4;
    static constexpr int B_BYTES = NB * kKC * 4;
    static constexpr int OFF_AH = 0, OFF_AL = A_BYTES, OFF_BH = 2 * A_BYTES, OFF_BL = 2 * A_BYTES + B_BYTES;
    static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int T_FLOATS = 3 * kKCH * P * 4;  // [dim][k group][degree][4 sources]
    static constexpr int OFF_T = 2 * STAGE;
    static constexpr int OFF_BAR = OFF_T + 2 * T_FLOATS * 4;
    // at least 120 KB so that two CTAs never share an SM's tensor memory when TMEM_COLS is 512
    static constexpr int SMEM_USED = OFF_BAR + 64;
    static constexpr int SMEM = TMEM_COLS == 512 && SMEM_USED < 120 * 1024 ? 120 * 1024 : SMEM_USED;
    static constexpr int A_ITEMS = 128 * kKCH / kThreads;
    // B items: two rounds over all threads, further rounds over the threads
    // that do not evaluate Chebyshev values (tid >= 3 * kKC)
    static constexpr int B_TOTAL = NB * kKCH;
    static constexpr int B_LATE = kThreads - 3 * kKC;
    static constexpr int B_ITEMS =
        B_TOTAL <= 2 * kThreads ? (B_TOTAL + kThreads - 1) / kThreads : 2 + (B_TOTAL - 2 * kThreads + B_LATE - 1) / B_LATE;
    static_assert(2 * BUF <= TMEM_COLS && NB <= BUF, "accumulators exceed tensor memory");
    static_assert(QCOL % 4 == 0, "drain column split");
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

// hi = TF32 rounding of x, lo = x - hi left unrounded (the tensor core reads
// its leading TF32 bits, i.e. truncates it): relative error <= 2^-21 per operand.
__device__ __forceinline__ void split_store_lo_trunc(const float4 v, unsigned char* hi_p, unsigned char* lo_p) {
    uint4 hi, lo;
    hi.x = tc::round_tf32_bits(__float_as_uint(v.x));
    hi.y = tc::round_tf32_bits(__float_as_uint(v.y));
    hi.z = tc::round_tf32_bits(__float_as_uint(v.z));
    hi.w = tc::round_tf32_bits(__float_as_uint(v.w));
    lo.x = __float_as_uint(v.x - __uint_as_float(hi.x));
    lo.y = __float_as_uint(v.y - __uint_as_float(hi.y));
    lo.z = __float_as_uint(v.z - __uint_as_float(hi.z));
    lo.w = __float_as_uint(v.w - __uint_as_float(hi.w));
    *reinterpret_cast<uint4*>(hi_p) = hi;
    *reinterpret_cast<uint4*>(lo_p) = lo;
}

template <int P>
__global__ void __launch_bounds__(kThreads, 1)
    k_c2proxy_tc(C2ProxyArgs a, const float* __restrict__ src_q, float* __restrict__ proxy_up, int kb,
                 int* __restrict__ err) {
    using S = C2PShape<P>;
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);  // [0,1] stage free, [2,3] segment done
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + S::OFF_BAR + 32);
    volatile int* s_abort = reinterpret_cast<volatile int*>(sm + S::OFF_BAR + 36);  // [3], sticky
    float* sT = reinterpret_cast<float*>(sm + S::OFF_T);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // flat grid, centre-major: the row tiles and column splits of one centre
    // run next to each other and share its sources in L2
    const int ntile = (P * kb + 127) / 128;
    const int e = blockIdx.x / (ntile * S::NSPLIT);
    const int tsel = blockIdx.x % (ntile * S::NSPLIT);
    const int rows = P * kb;
    const int row0 = (tsel % ntile) * 128;
    const int col0 = (tsel / ntile) * S::CW;             // first (i, j) column of this CTA
    const int ncol = min(S::CW, S::P2 - col0);
    const int r0 = a.rng_start[e], r1 = a.rng_start[e + 1];
    int nchunks = 0;
    for (int r = r0; r < r1; ++r) nchunks += (a.src_count[r] + kKC - 1) / kKC;
    const double4 cs = a.center_scale[e];

    if (warp == 0) {
        tc::tmem_alloc(s_tmem, S::TMEM_COLS);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < 4; ++i) tc::mbar_init(&bar[i], 1);
        s_abort[0] = s_abort[1] = s_abort[2] = 0;
        tc::fence_mbar_init();
    }

    // A items (row am, k group akg0 + 4u): Chebyshev-table offset of T_l and operand offset, fixed per thread
    const int am = tid & 127, akg0 = tid >> 7;
    const int aR = row0 + am;
    const bool arow = aR < rows;
    const int al = arow ? aR / kb : 0, ac = arow ? aR - al * kb : 0;
    int a_t[S::A_ITEMS], a_o[S::A_ITEMS];
#pragma unroll
    for (int u = 0; u < S::A_ITEMS; ++u) {
        const int kg = akg0 + 4 * u;
        a_t[u] = ((2 * kKCH + kg) * P + al) * 16;  // byte offset of a 4-source float4
        a_o[u] = (int)tc::kmajor_offset(am, kg * 4, kKCH);
    }
    // B items (row nl, k group): offsets of T_i and T_j (-1: zero row) and operand offset
    int b_x[S::B_ITEMS], b_y[S::B_ITEMS], b_o[S::B_ITEMS];
#pragma unroll
    for (int u = 0; u < S::B_ITEMS; ++u) {
        const int it = u < 2 ? tid + u * kThreads
                             : (tid >= 3 * kKC ? 2 * kThreads + (u - 2) * S::B_LATE + tid - 3 * kKC : S::B_TOTAL);
        const int nl = it % S::NB, kg = it / S::NB;
        const int n = col0 + nl;
        const bool valid = it < S::B_TOTAL && nl < ncol;
        b_x[u] = valid ? ((0 * kKCH + kg) * P + n % P) * 16 : -1;  // byte offsets
        b_y[u] = valid ? ((1 * kKCH + kg) * P + n / P) * 16 : -1;
        b_o[u] = it < S::B_TOTAL ? (int)tc::kmajor_offset(nl, kg * 4, kKCH) : -1;
    }
    // Chebyshev role: threads < 3*kKC evaluate one (source, dim) of the next chunk
    const bool cheb = tid < 3 * kKC;
    const int cs_s = tid % kKC, cs_d = tid / kKC;
    const double cs_c = cs_d == 0 ? cs.x : (cs_d == 1 ? cs.y : cs.z);

    auto load_q = [&](int g0, int nt, float (&qv)[S::A_ITEMS][4]) {
#pragma unroll
        for (int u = 0; u < S::A_ITEMS; ++u)
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int s = (akg0 + 4 * u) * 4 + w;
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
    int g1 = 0, nt1 = 0;  // chunk q + 1
    if (nchunks > 0) {
        int g0, nt;
        chunk_at(a, r0, r1, 0, g0, nt);
        load_q(g0, nt, qcur);
        cheb_store(0, load_x(g0, nt), nt);
        if (nchunks > 1) {
            chunk_at(a, r0, r1, 1, g1, nt1);
            xnext = load_x(g1, nt1);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;

    // FP32 sums of the drained segments: lane quarter warp % 4 (rows), column quarter warp / 4
    const int dq = warp & 3, dc = warp >> 2;
    float accd[S::QCOL];
#pragma unroll
    for (int i = 0; i < S::QCOL; ++i) accd[i] = 0.0f;
    auto drain = [&](int gg) -> bool {
        const bool waited = tc::mbar_wait(&bar[2 + (gg & 1)], (gg >> 1) & 1);
        if (!__all_sync(0xffffffffu, waited)) return false;
        tc::fence_after_sync();
        const uint32_t base =
            tmem + ((uint32_t)(dq * 32) << 16) + (uint32_t)((gg & 1) * S::BUF + dc * S::QCOL);
#pragma unroll
        for (int c0 = 0; c0 < S::QCOL; c0 += 16) {
            float v[16];
#pragma unroll
            for (int b4 = 0; b4 < 4; ++b4)
                if (c0 + 4 * b4 < S::QCOL) tc::tmem_ld_x4(base + (uint32_t)(c0 + 4 * b4), v + 4 * b4);
            tc::tmem_wait_ld();
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (c0 + u < S::QCOL) accd[c0 + u] += v[u];
        }
        tc::fence_before_sync();
        return true;
    };

    int issued = 0;  // chunks whose MMAs were issued and committed
    for (int q = 0; q < nchunks; ++q) {
        const int st = q & 1;
        const int seg = q / kSeg;
        const bool first = q % kSeg == 0, last = q % kSeg == kSeg - 1 || q == nchunks - 1;
        int g2 = 0, nt2 = 0;
        if (q + 1 < nchunks) load_q(g1, nt1, qnext);
        if (q + 2 < nchunks) chunk_at(a, r0, r1, q + 2, g2, nt2);
        // stage st was last read by the MMAs of chunk q-2
        if (q >= 2 && !tc::mbar_wait(&bar[st], ((q - 2) >> 1) & 1)) s_abort[st] = 1;
        unsigned char* stage = sm + st * S::STAGE;
        const unsigned char* T = reinterpret_cast<const unsigned char*>(sT + st * S::T_FLOATS);
        // A = T_l(z_s) q_sc
#pragma unroll
        for (int u = 0; u < S::A_ITEMS; ++u) {
            const float4 tz = *reinterpret_cast<const float4*>(T + a_t[u]);
            const float4 v = make_float4(tz.x * qcur[u][0], tz.y * qcur[u][1], tz.z * qcur[u][2], tz.w * qcur[u][3]);
            split_store_lo_trunc(v, stage + S::OFF_AH + a_o[u], stage + S::OFF_AL + a_o[u]);
        }
        // B = T_i(x_s) T_j(y_s) for the columns n = i + P j of this CTA
#pragma unroll
        for (int u = 0; u < S::B_ITEMS; ++u) {
            if (b_o[u] >= 0) {
                float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (b_x[u] >= 0) {
                    const float4 tx = *reinterpret_cast<const float4*>(T + b_x[u]);
                    const float4 ty = *reinterpret_cast<const float4*>(T + b_y[u]);
                    v = make_float4(tx.x * ty.x, tx.y * ty.y, tx.z * ty.z, tx.w * ty.w);
                }
                split_store_lo_trunc(v, stage + S::OFF_BH + b_o[u], stage + S::OFF_BL + b_o[u]);
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
            static_assert(S::NB <= 256, "one MMA per k-step");
            const uint32_t base = tc::smem_u32(stage);
            const uint32_t d = tmem + (uint32_t)((seg & 1) * S::BUF);
            constexpr uint32_t idesc = tc::idesc_tf32(128, S::NB);
            // descriptors of k-step 0; each k-step advances the start address by 256 B (16 units)
            const uint64_t ah = tc::smem_desc_k_noswizzle(base + S::OFF_AH, 128, S::SBO);
            const uint64_t alo = tc::smem_desc_k_noswizzle(base + S::OFF_AL, 128, S::SBO);
            const uint64_t bh = tc::smem_desc_k_noswizzle(base + S::OFF_BH, 128, S::SBO);
            const uint64_t blo = tc::smem_desc_k_noswizzle(base + S::OFF_BL, 128, S::SBO);
#pragma unroll
            for (int ks = 0; ks < kKC / 8; ++ks) {
                const uint64_t dk = (uint64_t)(16 * ks);
                tc::mma_tf32(d, ah + dk, bh + dk, idesc, (first && ks == 0) ? 0u : 1u);
                tc::mma_tf32(d, ah + dk, blo + dk, idesc, 1u);
                tc::mma_tf32(d, alo + dk, bh + dk, idesc, 1u);
            }
            tc::commit(&bar[st]);
            if (last) tc::commit(&bar[2 + (seg & 1)]);
        }
        issued = q + 1;
        // the previous segment is complete: fold it into the FP32 sums while the
        // tensor core works on this segment (the other accumulator buffer).  A
        // failure is flagged for the next iteration's check.
        if (first && seg > 0) {
            if (!drain(seg - 1)) s_abort[st ^ 1] = 1;
        }
#pragma unroll
        for (int u = 0; u < S::A_ITEMS; ++u)
#pragma unroll
            for (int w = 0; w < 4; ++w) qcur[u][w] = qnext[u][w];
        g1 = g2;
        nt1 = nt2;
    }
    bool ok = s_abort[0] == 0 && s_abort[1] == 0;
    if (ok && issued > 0) {
        if (!drain((issued - 1) / kSeg)) s_abort[2] = 1;
    } else if (!ok && issued > 0) {
        const int ql = issued - 1;
        tc::mbar_wait(&bar[ql & 1], (ql >> 1) & 1);
    }
    __syncthreads();
    ok = s_abort[0] == 0 && s_abort[1] == 0 && s_abort[2] == 0;
    if (ok && issued > 0) {
        const int m = dq * 32 + lane;
        const int R = row0 + m;
        if (R < rows) {
            const int l = R / kb, c = R - l * kb;
            float* out = proxy_up + ((int64_t)a.slot[e] * kb + c) * (P * P * P) + (int64_t)S::P2 * l + col0;
#pragma unroll
            for (int i = 0; i < S::QCOL; ++i) {
                const int nl = dc * S::QCOL + i;
                if (nl < ncol) out[nl] += accd[i];
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
    const int64_t nblocks = (int64_t)a.n_centers * ((P * kb + 127) / 128) * S::NSPLIT;
    if (nblocks > INT32_MAX) throw std::runtime_error("too many proxy-moment tiles for one launch");
    k_c2proxy_tc<P><<<(unsigned)nblocks, kThreads, S::SMEM, s>>>(a, src_q, up, kb, err);
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

// ===========================================================================
// Residual near field on the tensor cores.
//   D[t, c] = sum_s K(t, s) Q[c, s]  per source box, A = K (targets x sources),
//   B = Q (RHS x sources), both K-major in shared memory, 32 sources per chunk.
// Per chunk: warps generate A (kernel values) and B (charges) into one of two
// stages; one thread issues 4 k-steps x 3 TF32 MMAs into the accumulator of
// the current source box (two TMEM buffers of 64 columns alternate by box).
// When a box ends, warps 0-3 (TMEM lanes = targets) add its accumulator to
// FP64 sums in shared memory while the next box proceeds.
// ===========================================================================
namespace {

constexpr int kNKC = 32;            // sources per chunk
constexpr int kNSeg = 2;            // default chunks accumulated in tensor memory before a drain
constexpr int kNKCH = kNKC / 4;     // 16-byte K chunks per operand row
constexpr int kNThreads = 512;
constexpr int kNSBO = kNKCH * 128;  // bytes between 8-row groups
constexpr int kNA = 128 * kNKC * 4; // bytes of one A part
constexpr int kNB = 64 * kNKC * 4;  // bytes of one B part (64 RHS rows)
constexpr int kN_OFF_AH = 0, kN_OFF_AL = kNA, kN_OFF_BH = 2 * kNA, kN_OFF_BL = 2 * kNA + kNB;
constexpr int kNStage = 2 * kNA + 2 * kNB;
constexpr int kN_OFF_SRC = 2 * kNStage;          // [2][hi 32 float4 | lo 32 float4]
constexpr int kNSrc = kNKC * 32;
constexpr int kN_OFF_ACC = kN_OFF_SRC + 2 * kNSrc;  // double [64][128]
constexpr int kN_OFF_PAIR = kN_OFF_ACC + 64 * 128 * 8;
constexpr int kNPairBytes = kNearTcMaxPairs * 28;   // int start, count, nch, cb; float d2max, rsc, cen
constexpr int kN_OFF_PREF = kN_OFF_PAIR + kNPairBytes;  // int [kNearTcMaxPairs + 1] chunk prefix
constexpr int kN_OFF_LIST = kN_OFF_PREF + (kNearTcMaxPairs + 1) * 4 + 60;  // int [kNearTcMaxChunks] kept chunks
constexpr int kN_OFF_BAR = kN_OFF_LIST + kNearTcMaxChunks * 4;
constexpr int kNSmem = kN_OFF_BAR + 256;
static_assert(kNSmem <= 227 * 1024, "near smem");
static_assert(kNKC == kNearTcChunk, "chunk size");

struct NearPair {
    int start, count, nch, cb;
    float d2max, rsc, cen;
};

template <int NC>
__global__ void __launch_bounds__(kNThreads, 1)
    k_near_tc(NearTc a, const float4* __restrict__ trg_hi, const float4* __restrict__ trg_lo,
              const float4* __restrict__ src_hi, const float4* __restrict__ src_lo, const float* __restrict__ src_q,
              double* __restrict__ pot, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    // flat grid, leaf-major: the target tiles of one leaf run next to each
    // other and share its neighbours' sources in L2
    const int ntile = (a.max_trg + 127) / 128;
    const int e = blockIdx.x / ntile;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const int m0 = (blockIdx.x % ntile) * 128;
    if (m0 >= nt) return;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kN_OFF_BAR);  // [0,1] stage free, [2,3] segment accumulated
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + kN_OFF_BAR + 32);
    volatile int* s_abort = reinterpret_cast<volatile int*>(sm + kN_OFF_BAR + 36);  // [3]
    int* s_np = reinterpret_cast<int*>(sm + kN_OFF_BAR + 48);
    int* s_nch = reinterpret_cast<int*>(sm + kN_OFF_BAR + 52);   // candidate chunks
    int* s_kept = reinterpret_cast<int*>(sm + kN_OFF_BAR + 56);  // chunks kept after the cull
    float* s_tbox = reinterpret_cast<float*>(sm + kN_OFF_BAR + 64);   // [4 warps][6], then tile box [6]
    int* s_wcnt = reinterpret_cast<int*>(sm + kN_OFF_BAR + 192);      // [16] kept per warp
    int* s_last_commit = reinterpret_cast<int*>(sm + kN_OFF_BAR + 60);  // last chunk whose MMAs were committed
    NearPair* pairs = reinterpret_cast<NearPair*>(sm + kN_OFF_PAIR);
    int* pref = reinterpret_cast<int*>(sm + kN_OFF_PREF);
    int* list = reinterpret_cast<int*>(sm + kN_OFF_LIST);
    double* acc64 = reinterpret_cast<double*>(sm + kN_OFF_ACC);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kb = a.kb;
    const int NBp = (kb + 15) & ~15;

    if (warp == 0) {
        tc::tmem_alloc(s_tmem, 128);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::mbar_init(&bar[2], 1);
        tc::mbar_init(&bar[3], 1);
        s_abort[0] = s_abort[1] = s_abort[2] = 0;
        *s_last_commit = -1;
        int np = 0, nch = 0;
        pref[0] = 0;
        for (int pr = a.pair_start[e]; pr < a.pair_start[e + 1]; ++pr) {
            const int cnt = a.pair_src_count[pr];
            if (cnt <= 0 || np >= kNearTcMaxPairs) continue;
            const double b = a.pair_bsize[pr];
            NearPair q;
            q.start = a.pair_src_start[pr];
            q.count = cnt;
            q.nch = (cnt + kNKC - 1) / kNKC;
            q.cb = a.pair_chunk_base[pr];
            q.d2max = (float)(b * b);
            q.rsc = (float)(2.0 / b);
            q.cen = (float)(-0.5 * b);
            pairs[np++] = q;
            nch += q.nch;
            pref[np] = nch;
        }
        *s_np = np;
        *s_nch = min(nch, kNearTcMaxChunks);
        tc::fence_mbar_init();
    }
    for (int i = tid; i < 64 * 128; i += kNThreads) acc64[i] = 0.0;

    // A role: target row am, source groups ag0 and ag0 + 4
    const int am = tid & 127, ag0 = tid >> 7;
    const bool tval = m0 + am < nt;
    const float4 th = tval ? trg_hi[t0 + m0 + am] : make_float4(1e30f, 1e30f, 1e30f, 0.0f);
    const float4 tl = tval ? trg_lo[t0 + m0 + am] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // bounding box of the tile's targets (warps 0-3 hold all 128 rows)
    if (warp < 4) {
        float lo[3] = {tval ? th.x : 3e38f, tval ? th.y : 3e38f, tval ? th.z : 3e38f};
        float hi[3] = {tval ? th.x : -3e38f, tval ? th.y : -3e38f, tval ? th.z : -3e38f};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
        if (lane == 0)
            for (int d = 0; d < 3; ++d) {
                s_tbox[warp * 6 + d] = lo[d];
                s_tbox[warp * 6 + 3 + d] = hi[d];
            }
    }
    float cf[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) cf[i] = (float)a.coef[i];
    // B role (all threads): RHS row bc, source group bsg (4 sources)
    const int bc = tid & 63, bsg = tid >> 6;
    // position prefetch role (warps 8-9): source tid-256 (hi) or tid-288 (lo)
    const bool prole = tid >= 256 && tid < 256 + 2 * kNKC;
    const int ps_ = (tid - 256) & (kNKC - 1);
    const bool plo = tid >= 256 + kNKC;

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;
    const int np = *s_np, ncand = *s_nch;
    if (tid == 0) {
        for (int d = 0; d < 3; ++d) {
            float lo = s_tbox[d], hi = s_tbox[3 + d];
            for (int w = 1; w < 4; ++w) {
                lo = fminf(lo, s_tbox[w * 6 + d]);
                hi = fmaxf(hi, s_tbox[w * 6 + 3 + d]);
            }
            // widen by the FP32 rounding of hi-part coordinates (relative 2^-23)
            const float pad = 2.5e-7f * fmaxf(fabsf(lo), fabsf(hi)) + 1e-30f;
            s_tbox[24 + d] = lo - pad;
            s_tbox[27 + d] = hi + pad;
        }
        *s_kept = 0;
    }
    __syncthreads();
    // keep the chunks whose bounding box comes within b of the tile (order preserved)
    {
        const float tlo[3] = {s_tbox[24], s_tbox[25], s_tbox[26]};
        const float thi[3] = {s_tbox[27], s_tbox[28], s_tbox[29]};
        for (int base = 0; base < ncand; base += kNThreads) {
            const int c = base + tid;
            bool keep = false;
            int code = 0;
            if (c < ncand) {
                int lo = 0, hi = np - 1;  // pair p with pref[p] <= c < pref[p + 1]
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (pref[mid] <= c) lo = mid; else hi = mid - 1;
                }
                const int j = c - pref[lo];
                const NearPair& q = pairs[lo];
                const float4 clo = __ldg(a.chunk_lo + q.cb + j), chi = __ldg(a.chunk_hi + q.cb + j);
                const float gx = fmaxf(0.0f, fmaxf(clo.x - thi[0], tlo[0] - chi.x));
                const float gy = fmaxf(0.0f, fmaxf(clo.y - thi[1], tlo[1] - chi.y));
                const float gz = fmaxf(0.0f, fmaxf(clo.z - thi[2], tlo[2] - chi.z));
                keep = fmaf(gx, gx, fmaf(gy, gy, gz * gz)) <= q.d2max * 1.00001f;
                code = (lo << 16) | j;
            }
            const unsigned ball = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) s_wcnt[warp] = __popc(ball);
            __syncthreads();
            int off = *s_kept;
            for (int w = 0; w < warp; ++w) off += s_wcnt[w];
            if (keep) list[off + __popc(ball & ((1u << lane) - 1u))] = code;
            __syncthreads();
            if (tid == 0) {
                int tot = 0;
                for (int w = 0; w < kNThreads / 32; ++w) tot += s_wcnt[w];
                *s_kept += tot;
            }
            __syncthreads();
        }
    }
    const int nchunks = *s_kept;

    auto chunk_src = [&](int q, int& p, int& g0, int& n) {
        const int v = list[q];
        p = v >> 16;
        const int j = v & 0xFFFF;
        g0 = pairs[p].start + j * kNKC;
        n = min(kNKC, pairs[p].count - j * kNKC);
    };
    auto load_q = [&](int q, float (&qv)[4]) {
        int p, g0, n;
        chunk_src(q, p, g0, n);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int s = bsg * 4 + u;
            qv[u] = (s < n && bc < kb) ? __ldg(src_q + (int64_t)(g0 + s) * kb + bc) : 0.0f;
        }
    };
    auto load_pos = [&](int q) -> float4 {
        int p, g0, n;
        chunk_src(q, p, g0, n);
        if (ps_ >= n) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return plo ? __ldg(src_lo + g0 + ps_) : __ldg(src_hi + g0 + ps_);
    };
    auto store_pos = [&](int buf, float4 v) {
        float4* dst = reinterpret_cast<float4*>(sm + kN_OFF_SRC + buf * kNSrc);
        dst[(plo ? kNKC : 0) + ps_] = v;
    };
    // Add segment gg's accumulator (TMEM buffer gg & 1) to the FP64 sums.  Warp w
    // reads TMEM lanes 32 (w % 4) .. +31 (targets) and columns 16 (w / 4) .. +15 (RHS).
    auto drain = [&](int gg) -> bool {
        const bool waited = tc::mbar_wait(&bar[2 + (gg & 1)], (gg >> 1) & 1, a.wait_cycles);
        if (!__all_sync(0xffffffffu, waited)) return false;  // keep the warp-collective loads uniform
        tc::fence_after_sync();
        const int lq = warp & 3, cg = warp >> 2;
        if (16 * cg < NBp) {
            const uint32_t base = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)((gg & 1) * 64 + 16 * cg);
            float v[16];
            tc::tmem_ld_x8(base, v);
            tc::tmem_ld_x8(base + 8, v + 8);
            tc::tmem_wait_ld();
            const int m = lq * 32 + lane;
#pragma unroll
            for (int i = 0; i < 16; ++i) acc64[(16 * cg + i) * 128 + m] += (double)v[i];
        }
        tc::fence_before_sync();
        return true;
    };

    float qcur[4], qnext[4];
    float4 pnext = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (nchunks > 0) {
        load_q(0, qcur);
        if (prole) store_pos(0, load_pos(0));
        if (nchunks > 1 && prole) pnext = load_pos(1);
    }
    __syncthreads();

    // The accumulator is drained every nseg chunks: the tensor-core FP32
    // accumulation loses low bits on every MMA step, so each segment stays
    // short and the sums continue in FP64 on the CUDA cores.
    const int nseg = a.seg_chunks > 0 ? a.seg_chunks : kNSeg;
    int issued = 0;
    for (int q = 0; q < nchunks; ++q) {
        const int st = q & 1;
        const int seg = q / nseg;
        const bool first = q % nseg == 0, last = q % nseg == nseg - 1 || q == nchunks - 1;
        int pidx, g0c, nv;
        chunk_src(q, pidx, g0c, nv);
        const NearPair pr = pairs[pidx];
        if (q + 1 < nchunks) {
            load_q(q + 1, qnext);
            if (prole) {
                store_pos(st ^ 1, pnext);
                if (q + 2 < nchunks) pnext = load_pos(q + 2);
            }
        }
        if (q >= 2 && !tc::mbar_wait(&bar[st], ((q - 2) >> 1) & 1, a.wait_cycles)) s_abort[st] = 1;
        unsigned char* stage = sm + st * kNStage;
        const float4* sh = reinterpret_cast<const float4*>(sm + kN_OFF_SRC + st * kNSrc);
        const float4* sl = sh + kNKC;
        // A: kernel values for target am, sources 4g..4g+3
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int g = ag0 + 4 * u;
            float r2v[4];
            bool anyin = false;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int s = 4 * g + k;
                const float4 yh = sh[s], yl = sl[s];
                const float dx = (th.x - yh.x) + (tl.x - yl.x);
                const float dy = (th.y - yh.y) + (tl.y - yl.y);
                const float dz = (th.z - yh.z) + (tl.z - yl.z);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool in = s < nv && r2 > 1e-30f && r2 < pr.d2max;
                r2v[k] = in ? r2 : -1.0f;
                anyin |= in;
            }
            float w[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (__any_sync(0xffffffffu, anyin)) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float r2 = r2v[k] > 0.0f ? r2v[k] : 1.0f;
                    const float rinv = rsqrtf(r2);
                    const float x = fmaf(r2, rinv, pr.cen) * pr.rsc;
                    float pv = cf[NC - 1];
#pragma unroll
                    for (int i = NC - 2; i >= 0; --i) pv = fmaf(pv, x, cf[i]);
                    w[k] = r2v[k] > 0.0f ? pv * rinv : 0.0f;
                }
            }
            const uint32_t off = tc::kmajor_offset(am, 4 * g, kNKCH);
            split_store(make_float4(w[0], w[1], w[2], w[3]), stage + kN_OFF_AH + off, stage + kN_OFF_AL + off);
        }
        // B: charges, rows = RHS, K = sources
        {
            const uint32_t off = tc::kmajor_offset(bc, 4 * bsg, kNKCH);
            split_store(make_float4(qcur[0], qcur[1], qcur[2], qcur[3]), stage + kN_OFF_BH + off,
                        stage + kN_OFF_BL + off);
        }
        // the previous box is complete: fold its accumulator into the FP64 sums
        tc::fence_proxy_async();
        __syncthreads();
        if (s_abort[st]) break;
        if (tid == 0 && !(blockIdx.x == 0 && q == a.withhold_chunk)) {
            tc::fence_after_sync();
            const uint32_t base = tc::smem_u32(stage);
            const uint32_t idesc = tc::idesc_tf32(128, NBp);
            const uint32_t d = tmem + (uint32_t)((seg & 1) * 64);
#pragma unroll
            for (int ks = 0; ks < kNKC / 8; ++ks) {
                const uint32_t kofs = ks * 256;
                const uint64_t ah = tc::smem_desc_k_noswizzle(base + kN_OFF_AH + kofs, 128, kNSBO);
                const uint64_t alo = tc::smem_desc_k_noswizzle(base + kN_OFF_AL + kofs, 128, kNSBO);
                const uint64_t bh = tc::smem_desc_k_noswizzle(base + kN_OFF_BH + kofs, 128, kNSBO);
                const uint64_t blo = tc::smem_desc_k_noswizzle(base + kN_OFF_BL + kofs, 128, kNSBO);
                tc::mma_tf32(d, ah, bh, idesc, (first && ks == 0) ? 0u : 1u);
                tc::mma_tf32(d, ah, blo, idesc, 1u);
                tc::mma_tf32(d, alo, bh, idesc, 1u);
            }
            tc::commit(&bar[st]);
            if (last) tc::commit(&bar[2 + (seg & 1)]);
            *s_last_commit = q;
        }
        issued = q + 1;
        // fold the previous segment while this one runs on the tensor core
        if (first && seg > 0) {
            if (!drain(seg - 1)) s_abort[st ^ 1] = 1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) qcur[u] = qnext[u];
    }
    bool ok = s_abort[0] == 0 && s_abort[1] == 0;
    if (ok && issued > 0) {
        if (!drain((issued - 1) / nseg)) s_abort[2] = 1;
    }
    __syncthreads();
    ok = s_abort[0] == 0 && s_abort[1] == 0 && s_abort[2] == 0;
    if (!ok) {
        // wait (bounded) until this CTA's MMAs in flight are done before the
        // tensor memory is freed: tensor-core ops complete in issue order, so
        // the last committed chunk's barrier covers all of them
        const int lc = *s_last_commit;
        if (lc >= 0) tc::mbar_wait(&bar[lc & 1], (lc >> 1) & 1);
    }
    if (ok) {
        for (int i = tid; i < kb * 128; i += kNThreads) {
            const int c = i >> 7, mm = i & 127;
            if (m0 + mm < nt) pot[(int64_t)c * a.N + t0 + m0 + mm] += acc64[c * 128 + mm];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 128);
    }
    if (!ok && tid == 0) atomicExch(err, 1);
}

template <int NC>
void launch_near_tc_nc(const NearTc& a, const float4* th, const float4* tl, const float4* sh, const float4* sl,
                       const float* q, double* pot, int* err, cudaStream_t s) {
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    if (!configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_near_tc<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNSmem));
        configured[dev] = true;
    }
    const int64_t nblocks = (int64_t)a.n_leaves * ((a.max_trg + 127) / 128);
    if (nblocks > INT32_MAX) throw std::runtime_error("too many near-field tiles for one launch");
    k_near_tc<NC><<<(unsigned)nblocks, kNThreads, kNSmem, s>>>(a, th, tl, sh, sl, q, pot, err);
}


}  // namespace

bool launch_near_tc(const NearTc& a, int nc, const float4* trg_hi, const float4* trg_lo, const float4* src_hi,
                    const float4* src_lo, const float* src_q, double* pot, int* err, cudaStream_t s) {
    if (a.kb < 1 || a.kb > 64 || a.n_leaves <= 0 || a.max_trg <= 0) return false;
    switch (nc) {
#define PDMK_NTC(NC)                                                                  \
    case NC: launch_near_tc_nc<NC>(a, trg_hi, trg_lo, src_hi, src_lo, src_q, pot, err, s); \
        return true;
        PDMK_NTC(5) PDMK_NTC(6) PDMK_NTC(9) PDMK_NTC(11) PDMK_NTC(12)
#undef PDMK_NTC
        default: return false;
    }
}

// ===========================================================================
// Leaf evaluation on the tensor cores.  Rows (l, c) of the proxy coefficients
// are processed in passes of up to kEN = 128 (whole l values); K = (i, j) in
// chunks of 16.  The A operand (T_i(x) T_j(y) of the tile's targets) is
// regenerated per pass from tables in shared memory; B is loaded from the
// coefficients and split.  Every kESeg chunks the accumulator (two alternating
// 128-column buffers) is folded with T_l(z) into per-target FP32 sums of the kb
// RHS by all eight warps (lane quarter = targets, half = l range), so no
// tensor-memory accumulation runs over more than a few MMA steps.  A CTA takes
// 256 tensor-memory columns and under 100 KB of shared memory, so two CTAs share
// an SM (16 warps: the operand generation is latency-bound with 8).
// ===========================================================================
namespace {

constexpr int kEKC = 16;
constexpr int kEKCH = kEKC / 4;
constexpr int kEN = 128;  // accumulator columns of one buffer (MMA N)
constexpr int kESeg = 4;
constexpr int kEThreads = 256;
constexpr int kESBO = kEKCH * 128;
constexpr int kEA = 128 * kEKC * 4;
constexpr int kEB = kEN * kEKC * 4;
constexpr int kE_OFF_AH = 0, kE_OFF_AL = kEA, kE_OFF_BH = 2 * kEA, kE_OFF_BL = 2 * kEA + kEB;
constexpr int kEStage = 2 * kEA + 2 * kEB;

template <int P, int KB>
struct EvShape {
    static constexpr int P2 = P * P;
    static constexpr int P3 = P * P * P;
    static constexpr int NKC = (P2 + kEKC - 1) / kEKC;
    static constexpr int LP = (kEN / KB) < P ? (kEN / KB) : P;  // l values per pass
    static constexpr int NPASS = (P + LP - 1) / LP;
    static constexpr int NSEGP = (NKC + kESeg - 1) / kESeg;     // segments per pass
    static constexpr int TSTR = P | 1;  // odd row stride of the T tables (bank spread)
    static constexpr int OFF_T = 2 * kEStage;
    static constexpr int T_BYTES = 3 * 128 * TSTR * 4;
    static constexpr int OFF_BAR = (OFF_T + T_BYTES + 15) / 16 * 16;
    static constexpr int SMEM_USED = OFF_BAR + 64;
    static constexpr int SMEM = SMEM_USED;  // two CTAs per SM (2 x 256 TMEM columns)
    static constexpr int B_ITEMS = kEN * kEKCH / kEThreads;
    static_assert(SMEM <= 227 * 1024, "eval smem");
    static_assert(KB % 16 == 0 && KB <= 64, "RHS block");
    static_assert(128 * KB * 4 <= kEStage, "half-sum exchange buffer");
};

template <int P, int KB>
__global__ void __launch_bounds__(kEThreads, 2) k_eval_tc(EvalTc a, int* __restrict__ err) {
    using S = EvShape<P, KB>;
    extern __shared__ __align__(1024) unsigned char sm[];
    // flat grid, leaf-major: the target tiles of one leaf run next to each
    // other and share its downward coefficients in L2
    const int ntile = (a.max_trg + 127) / 128;
    const int e = blockIdx.x / ntile;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const int m0 = (blockIdx.x % ntile) * 128;
    if (m0 >= nt) return;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);  // [0,1] stage free, [2,3] segment done
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + S::OFF_BAR + 32);
    volatile int* s_abort = reinterpret_cast<volatile int*>(sm + S::OFF_BAR + 36);  // [3]
    float* sT = reinterpret_cast<float*>(sm + S::OFF_T);  // [3][128][TSTR]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        tc::tmem_alloc(s_tmem, 2 * kEN);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < 4; ++i) tc::mbar_init(&bar[i], 1);
        s_abort[0] = s_abort[1] = s_abort[2] = 0;
        tc::fence_mbar_init();
    }
    const double4 cs = a.center_scale[e];
    if (tid < 128) {
        const bool valid = m0 + tid < nt;
        double4 pt = make_double4(0.0, 0.0, 0.0, 0.0);
        if (valid) pt = a.trg[t0 + m0 + tid];
        const float xs[3] = {(float)((pt.x - cs.x) * cs.w), (float)((pt.y - cs.y) * cs.w),
                             (float)((pt.z - cs.z) * cs.w)};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            float* dst = sT + (d * 128 + tid) * S::TSTR;
            const float x = xs[d];
            float t0v = 1.0f, t1v = x;
            dst[0] = valid ? 1.0f : 0.0f;
            dst[1] = valid ? x : 0.0f;
#pragma unroll
            for (int n = 2; n < P; ++n) {
                const float t2 = 2.0f * x * t1v - t0v;
                dst[n] = valid ? t2 : 0.0f;
                t0v = t1v;
                t1v = t2;
            }
        }
    }
    const float* C0 = a.proxy_down + (int64_t)a.slot[e] * KB * S::P3;

    // B items of this thread: (row group, k group, row in group) -> coalesced loads, conflict-free stores
    auto load_b = [&](int q, float4 (&bv)[S::B_ITEMS]) {
        const int pass = q / S::NKC, kc = q - pass * S::NKC;
        const int l0 = pass * S::LP;
        const int nrows = min(S::LP, P - l0) * KB;
        const int k0 = kc * kEKC;
#pragma unroll
        for (int u = 0; u < S::B_ITEMS; ++u) {
            const int idx = tid + u * kEThreads;
            const int r = (idx >> 5) * 8 + (idx & 7), g = (idx >> 3) & 3;
            const int k = k0 + 4 * g;
            float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (r < nrows) {
                const int l = l0 + r / KB, c = r % KB;
                const float* src = C0 + (int64_t)c * S::P3 + S::P2 * l + k;
                if constexpr (P % 2 == 0) {
                    if (k + 3 < S::P2) {
                        v = __ldg(reinterpret_cast<const float4*>(src));
                    } else {
                        if (k < S::P2) v.x = __ldg(src);
                        if (k + 1 < S::P2) v.y = __ldg(src + 1);
                        if (k + 2 < S::P2) v.z = __ldg(src + 2);
                    }
                } else {
                    if (k < S::P2) v.x = __ldg(src);
                    if (k + 1 < S::P2) v.y = __ldg(src + 1);
                    if (k + 2 < S::P2) v.z = __ldg(src + 2);
                    if (k + 3 < S::P2) v.w = __ldg(src + 3);
                }
            }
            bv[u] = v;
        }
    };

    float acc[KB];
#pragma unroll
    for (int c = 0; c < KB; ++c) acc[c] = 0.0f;
    const int nchunks = S::NPASS * S::NKC;
    float4 bcur[S::B_ITEMS], bnext[S::B_ITEMS];
    load_b(0, bcur);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;

    // fold segment gg (TMEM buffer gg & 1) into acc: lane quarter warp % 4, l half warp / 4
    const int dq = warp & 3, dh = warp >> 2;
    auto drain = [&](int gg) -> bool {
        const bool waited = tc::mbar_wait(&bar[2 + (gg & 1)], (gg >> 1) & 1);
        if (!__all_sync(0xffffffffu, waited)) return false;
        tc::fence_after_sync();
        const int pass = gg / S::NSEGP;
        const int l0 = pass * S::LP;
        const int nl = min(S::LP, P - l0);
        const int hl = (nl + 1) / 2;
        const int lb = dh * hl, le = min(nl, lb + hl);
        const float* Tz = sT + (2 * 128 + dq * 32 + lane) * S::TSTR;
        const uint32_t lane_base = tmem + ((uint32_t)(dq * 32) << 16) + (uint32_t)((gg & 1) * kEN);
        for (int li = lb; li < le; ++li) {
            const float tz = Tz[l0 + li];
#pragma unroll
            for (int c0 = 0; c0 < KB; c0 += 32) {
                float v[32];
#pragma unroll
                for (int b8 = 0; b8 < 4; ++b8)
                    if (c0 + 8 * b8 < KB) tc::tmem_ld_x8(lane_base + (uint32_t)(li * KB + c0 + 8 * b8), v + 8 * b8);
                tc::tmem_wait_ld();
#pragma unroll
                for (int u = 0; u < 32; ++u)
                    if (c0 + u < KB) acc[c0 + u] = fmaf(tz, v[u], acc[c0 + u]);
            }
        }
        tc::fence_before_sync();
        return true;
    };

    int issued = 0;
    for (int q = 0; q < nchunks; ++q) {
        const int st = q & 1;
        const int pass = q / S::NKC, kc = q - pass * S::NKC;
        const int seg = pass * S::NSEGP + kc / kESeg;
        const bool first = kc % kESeg == 0, last = kc % kESeg == kESeg - 1 || kc == S::NKC - 1;
        if (q + 1 < nchunks) load_b(q + 1, bnext);
        if (q >= 2 && !tc::mbar_wait(&bar[st], ((q - 2) >> 1) & 1)) s_abort[st] = 1;
        unsigned char* stage = sm + st * kEStage;
        const int k0 = kc * kEKC;
        // A = T_i(x_t) T_j(y_t), K index k = i + P j
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int idx = tid + u * kEThreads;
            const int m = idx & 127, g = idx >> 7;
            const float* Tx = sT + (0 * 128 + m) * S::TSTR;
            const float* Ty = sT + (1 * 128 + m) * S::TSTR;
            float v[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int k = k0 + 4 * g + w;
                const int i = k % P, j = k / P;
                v[w] = k < S::P2 ? Tx[i] * Ty[j] : 0.0f;
            }
            const uint32_t off = tc::kmajor_offset(m, 4 * g, kEKCH);
            split_store(make_float4(v[0], v[1], v[2], v[3]), stage + kE_OFF_AH + off, stage + kE_OFF_AL + off);
        }
#pragma unroll
        for (int u = 0; u < S::B_ITEMS; ++u) {
            const int idx = tid + u * kEThreads;
            const int r = (idx >> 5) * 8 + (idx & 7), g = (idx >> 3) & 3;
            const uint32_t off = tc::kmajor_offset(r, 4 * g, kEKCH);
            split_store(bcur[u], stage + kE_OFF_BH + off, stage + kE_OFF_BL + off);
        }
        tc::fence_proxy_async();
        __syncthreads();
        if (s_abort[st]) break;
        if (tid == 0) {
            tc::fence_after_sync();
            const int nrows = min(S::LP, P - pass * S::LP) * KB;
            const uint32_t base = tc::smem_u32(stage);
            const uint32_t idesc = tc::idesc_tf32(128, nrows);
            const uint32_t d = tmem + (uint32_t)((seg & 1) * kEN);
#pragma unroll
            for (int ks = 0; ks < kEKC / 8; ++ks) {
                const uint32_t kofs = ks * 256;
                const uint64_t ah = tc::smem_desc_k_noswizzle(base + kE_OFF_AH + kofs, 128, kESBO);
                const uint64_t alo = tc::smem_desc_k_noswizzle(base + kE_OFF_AL + kofs, 128, kESBO);
                const uint64_t bh = tc::smem_desc_k_noswizzle(base + kE_OFF_BH + kofs, 128, kESBO);
                const uint64_t blo = tc::smem_desc_k_noswizzle(base + kE_OFF_BL + kofs, 128, kESBO);
                tc::mma_tf32(d, ah, bh, idesc, (first && ks == 0) ? 0u : 1u);
                tc::mma_tf32(d, ah, blo, idesc, 1u);
                tc::mma_tf32(d, alo, bh, idesc, 1u);
            }
            tc::commit(&bar[st]);
            if (last) tc::commit(&bar[2 + (seg & 1)]);
        }
        issued = q + 1;
        // fold the previous segment while this one runs on the tensor core
        if (first && seg > 0) {
            if (!drain(seg - 1)) s_abort[st ^ 1] = 1;
        }
#pragma unroll
        for (int u = 0; u < S::B_ITEMS; ++u) bcur[u] = bnext[u];
    }
    bool ok = s_abort[0] == 0 && s_abort[1] == 0;
    if (ok && issued == nchunks) {
        if (!drain(S::NPASS * S::NSEGP - 1)) s_abort[2] = 1;
    } else if (issued > 0) {
        const int ql = issued - 1;
        tc::mbar_wait(&bar[ql & 1], (ql >> 1) & 1);
    }
    __syncthreads();
    ok = s_abort[0] == 0 && s_abort[1] == 0 && s_abort[2] == 0;
    // combine the two l halves: half 1 publishes its sums, half 0 adds and writes
    float* xch = reinterpret_cast<float*>(sm);  // stage 0, idle now
    const int m = dq * 32 + lane;
    if (dh == 1) {
#pragma unroll
        for (int c = 0; c < KB; ++c) xch[c * 128 + m] = acc[c];
    }
    __syncthreads();
    if (ok && dh == 0 && m0 + m < nt) {
        double* pt = a.pot + t0 + m0 + m;
#pragma unroll
        for (int c = 0; c < KB; ++c) pt[(int64_t)c * a.N] += (double)(acc[c] + xch[c * 128 + m]);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 2 * kEN);
    }
    if (!ok && tid == 0) atomicExch(err, 1);
}

template <int P, int KB>
void launch_eval_tc_pk(const EvalTc& a, int* err, cudaStream_t s) {
    using S = EvShape<P, KB>;
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    if (!configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_eval_tc<P, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
        configured[dev] = true;
    }
    const int64_t nblocks = (int64_t)a.n_leaves * ((a.max_trg + 127) / 128);
    if (nblocks > INT32_MAX) throw std::runtime_error("too many leaf-evaluation tiles for one launch");
    k_eval_tc<P, KB><<<(unsigned)nblocks, kEThreads, S::SMEM, s>>>(a, err);
}

}  // namespace

bool launch_eval_tc(const EvalTc& a, int p, int kb, int* err, cudaStream_t s) {
    if (a.n_leaves <= 0 || a.max_trg <= 0) return false;
    if (p != 9 && p != 18) return false;
    if (kb != 16 && kb != 32 && kb != 64) return false;
    if (p == 9) {
        if (kb == 16) launch_eval_tc_pk<9, 16>(a, err, s);
        else if (kb == 32) launch_eval_tc_pk<9, 32>(a, err, s);
        else launch_eval_tc_pk<9, 64>(a, err, s);
    } else {
        if (kb == 16) launch_eval_tc_pk<18, 16>(a, err, s);
        else if (kb == 32) launch_eval_tc_pk<18, 32>(a, err, s);
        else launch_eval_tc_pk<18, 64>(a, err, s);
    }
    return true;
}

}  // namespace dev
}  // namespace pdmkb
