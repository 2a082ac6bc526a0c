// Multi-RHS evaluate: k charge vectors on one tree, in RHS blocks of kb.
//
// Same stages as the single-RHS path (kernels.cu), with an RHS dimension:
//   charges    T[n_all * kb]            source-major, RHS fastest (near field reads a source's kb charges)
//   proxy      T[slots * kb * p^3]      (slot, rhs) tensors contiguous -> transforms batch over (box, rhs)
//   plane wave complex<T>[slots * kb * M]
//   potentials double[kb * N]           RHS-major (coalesced per RHS)
// T = double: plain FP64.  T = float: mixed precision -- FP32 Chebyshev moments,
// transforms, shifts and leaf evaluation; FP32 near field on double-float
// coordinate differences with per-box FP32 partial sums merged in FP64; FP64
// far field (NUFFT), self term and final accumulation.
#include <cuda_runtime.h>

#include <cstdint>

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "device_tree.hpp"
#include "qp.cuh"
#include "nufft_multi.cuh"
#include "pw_fused.cuh"
#include "sep3.cuh"
#include "contract_tc.cuh"
#include "tc_kernels.cuh"

namespace pdmkb {
namespace dev {

struct cf {  // complex float
    float x, y;
};

template <>
__device__ __forceinline__ float zero<float>() { return 0.0f; }
template <>
__device__ __forceinline__ cf zero<cf>() { return {0.0f, 0.0f}; }
__device__ __forceinline__ float mac(float m, float x, float acc) { return fmaf(m, x, acc); }
__device__ __forceinline__ cf mac(cf m, float x, cf acc) { return {fmaf(m.x, x, acc.x), fmaf(m.y, x, acc.y)}; }
__device__ __forceinline__ cf mac(cf m, cf x, cf acc) {
    return {fmaf(m.x, x.x, fmaf(-m.y, x.y, acc.x)), fmaf(m.x, x.y, fmaf(m.y, x.x, acc.y))};
}

template <typename T>
struct Cplx;
template <>
struct Cplx<double> {
    using type = cd;
};
template <>
struct Cplx<float> {
    using type = cf;
};

// ---------------------------------------------------------------------------
// conversions and gathers
// ---------------------------------------------------------------------------
__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

// double-float split of positions: hi = fl(x), lo = fl(x - hi); .w of hi keeps the
// point's fourth field (self weight for targets) rounded to float.
__global__ void k_split_positions(const double4* __restrict__ in, float4* __restrict__ hi, float4* __restrict__ lo,
                                  int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = in[i];
    const float hx = (float)p.x, hy = (float)p.y, hz = (float)p.z;
    hi[i] = make_float4(hx, hy, hz, (float)p.w);
    lo[i] = make_float4((float)(p.x - (double)hx), (float)(p.y - (double)hy), (float)(p.z - (double)hz), 0.0f);
}

// Q (N x kb column-major, user order; RHS c >= kvalid read as zero) ->
// Qr (N x kb row-major): 32 x 32 tiles through shared memory, coalesced on
// both sides.  Gathering rows of Qr reads one contiguous kb-vector per source.
__global__ void k_transpose_q(const double* __restrict__ Q, double* __restrict__ Qr, int64_t N, int kb, int kvalid) {
    __shared__ double tile[32][33];
    const int64_t r0 = (int64_t)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = c0 + j;
        const int64_t r = r0 + threadIdx.x;
        tile[j][threadIdx.x] = (c < kvalid && r < N) ? Q[(int64_t)c * N + r] : 0.0;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t r = r0 + j;
        const int c = c0 + threadIdx.x;
        if (r < N && c < kb) Qr[r * kb + c] = tile[threadIdx.x][j];
    }
}

template <typename T>
__global__ void k_gather_src_rows(T* __restrict__ src_q, const int* __restrict__ idx, const double* __restrict__ Qr,
                                  int64_t n_all, int kb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_all * kb) return;
    const int64_t s = i / kb;
    const int c = (int)(i - s * kb);
    src_q[i] = (T)Qr[(int64_t)idx[s] * kb + c];
}

__global__ void k_gather_trg_m(double* __restrict__ q_t, const int* __restrict__ perm, const double* __restrict__ Q,
                               int64_t N, int kb, int kvalid) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * kb) return;
    const int c = (int)(i / N);
    const int64_t t = i % N;
    q_t[i] = c < kvalid ? Q[(int64_t)c * N + perm[t]] : 0.0;
}

__global__ void k_finalize_m(const double* __restrict__ pot, const double* __restrict__ far,
                             const double4* __restrict__ trg, const int* __restrict__ perm,
                             const double* __restrict__ q_t, double* __restrict__ out, int64_t N, int kvalid) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * kvalid) return;
    const int64_t c = i / N, t = i % N;
    out[c * N + perm[t]] = pot[i] + far[i] - trg[t].w * q_t[i];
}

// ---------------------------------------------------------------------------
// proxy moments: grid (centres, jk chunks, rhs)
// ---------------------------------------------------------------------------
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_c2proxy_m(C2ProxyArgs a, const T* __restrict__ src_q, T* __restrict__ proxy_up, int kb) {
    constexpr int TS = 32;
    __shared__ T sx[TS][P], sy[TS][P], sz[TS][P];
    const int e = blockIdx.x, c = blockIdx.z;
    const int jk = blockIdx.y * blockDim.x + threadIdx.x;
    const bool active = jk < P * P;
    const int j = jk % P, k = jk / P;
    T acc[P];
#pragma unroll
    for (int i = 0; i < P; ++i) acc[i] = T(0);
    const double4 cs = a.center_scale[e];
    for (int r = a.rng_start[e]; r < a.rng_start[e + 1]; ++r) {
        const int s0 = a.src_start[r], ns = a.src_count[r];
        for (int base = 0; base < ns; base += TS) {
            const int nt = min(TS, ns - base);
            __syncthreads();
            for (int task = threadIdx.x; task < 3 * TS; task += blockDim.x) {
                const int si = task % TS, d = task / TS;
                T* dst = d == 0 ? sx[si] : (d == 1 ? sy[si] : sz[si]);
                if (si < nt) {
                    const double4 pt = a.src[s0 + base + si];
                    const T x = (T)((d == 0 ? pt.x - cs.x : (d == 1 ? pt.y - cs.y : pt.z - cs.z)) * cs.w);
                    const T mult = d == 2 ? src_q[(int64_t)(s0 + base + si) * kb + c] : T(1);
                    T t0 = T(1), t1 = x;
                    dst[0] = mult;
                    if (P > 1) dst[1] = mult * x;
                    for (int n = 2; n < P; ++n) {
                        const T t2 = T(2) * x * t1 - t0;
                        dst[n] = mult * t2;
                        t0 = t1;
                        t1 = t2;
                    }
                } else {
                    for (int n = 0; n < P; ++n) dst[n] = T(0);
                }
            }
            __syncthreads();
            if (active) {
                for (int s = 0; s < nt; ++s) {
                    const T f = sy[s][j] * sz[s][k];
#pragma unroll
                    for (int i = 0; i < P; ++i) acc[i] = fma(f, sx[s][i], acc[i]);
                }
            }
        }
    }
    if (active) {
        T* out = proxy_up + ((int64_t)a.slot[e] * kb + c) * (P * P * P) + (int64_t)P * jk;
#pragma unroll
        for (int i = 0; i < P; ++i) out[i] += acc[i];
    }
}

// ---------------------------------------------------------------------------
// batched contraction with an RHS dimension:
// out[r + R*a] (op)= sum_i M[a + na*i] * in[i + ni*r] for entry ge = e0 + blockIdx.x,
// box eb = ge / rhs, rhs ec = ge % rhs.
// in = in_base + (in_off ? in_off[eb]*rhs + ec*in_unit : blockIdx.x*in_stride), same for out;
// M = mat_base + (mat_off ? mat_off[eb] : 0).
// ---------------------------------------------------------------------------
struct ContractM {
    const void* in;
    const int64_t* in_off;
    int64_t in_stride, in_unit;
    void* out;
    const int64_t* out_off;
    int64_t out_stride, out_unit;
    const void* mat;
    const int64_t* mat_off;
    int ni, na, R, n_entries, rhs;
    int64_t e0;
    int mode;
    double scale;
};

template <typename TO, typename TA>
__device__ __forceinline__ void store_m(TO* p, TA v, int mode, double scale);
template <>
__device__ __forceinline__ void store_m<double, double>(double* p, double v, int mode, double scale) {
    if (mode == kStore) *p = v; else if (mode == kAdd) *p += v; else *p += scale * v;
}
template <>
__device__ __forceinline__ void store_m<double, cd>(double* p, cd v, int mode, double scale) {
    if (mode == kStore) *p = v.x; else if (mode == kAdd) *p += v.x; else *p += scale * v.x;
}
template <>
__device__ __forceinline__ void store_m<cd, cd>(cd* p, cd v, int mode, double) {
    if (mode == kStore) *p = v; else { cd o = *p; *p = cd{o.x + v.x, o.y + v.y}; }
}
template <>
__device__ __forceinline__ void store_m<float, float>(float* p, float v, int mode, double scale) {
    if (mode == kStore) *p = v; else if (mode == kAdd) *p += v; else *p += (float)scale * v;
}
template <>
__device__ __forceinline__ void store_m<float, cf>(float* p, cf v, int mode, double scale) {
    if (mode == kStore) *p = v.x; else if (mode == kAdd) *p += v.x; else *p += (float)scale * v.x;
}
template <>
__device__ __forceinline__ void store_m<cf, cf>(cf* p, cf v, int mode, double) {
    if (mode == kStore) *p = v; else { cf o = *p; *p = cf{o.x + v.x, o.y + v.y}; }
}

template <typename TI, typename TM, typename TO, int RT, int AB>
__global__ void __launch_bounds__(256) k_contract_m(ContractM a) {
    extern __shared__ __align__(16) unsigned char smem_m[];
    using TA = decltype(mac(TM(), TI(), TM()));
    const int ni = a.ni, na = a.na, R = a.R;
    const int e = blockIdx.x, r0 = blockIdx.y * RT;
    const int64_t ge = a.e0 + e;
    const int rhs = a.rhs > 0 ? a.rhs : 1;
    const int64_t eb = ge / rhs, ec = ge % rhs;
    TM* sM = reinterpret_cast<TM*>(smem_m);
    const size_t moff = ((size_t)na * ni * sizeof(TM) + 15) / 16 * 16;
    TI* sIn = reinterpret_cast<TI*>(smem_m + moff);
    const TI* in = reinterpret_cast<const TI*>(a.in) + (a.in_off ? a.in_off[eb] * rhs + ec * a.in_unit : (int64_t)e * a.in_stride);
    TO* out = reinterpret_cast<TO*>(a.out) + (a.out_off ? a.out_off[eb] * rhs + ec * a.out_unit : (int64_t)e * a.out_stride);
    const TM* mat = reinterpret_cast<const TM*>(a.mat) + (a.mat_off ? a.mat_off[eb] : 0);
    for (int idx = threadIdx.x; idx < na * ni; idx += blockDim.x) sM[idx] = mat[idx];
    const int nr = min(RT, R - r0);
    const TI* inb = in + (int64_t)ni * r0;
    for (int idx = threadIdx.x; idx < ni * nr; idx += blockDim.x) {
        const int i = idx % ni, rr = idx / ni;
        sIn[rr + RT * i] = inb[idx];
    }
    __syncthreads();
    const int rr = threadIdx.x % RT, ag = threadIdx.x / RT, nag = blockDim.x / RT;
    if (rr >= nr) return;
    for (int a0 = ag * AB; a0 < na; a0 += nag * AB) {
        TA acc[AB];
#pragma unroll
        for (int b = 0; b < AB; ++b) acc[b] = zero<TA>();
        for (int i = 0; i < ni; ++i) {
            const TI x = sIn[rr + RT * i];
#pragma unroll
            for (int b = 0; b < AB; ++b)
                if (a0 + b < na) acc[b] = mac(sM[a0 + b + na * i], x, acc[b]);
        }
#pragma unroll
        for (int b = 0; b < AB; ++b)
            if (a0 + b < na) store_m<TO, TA>(out + (r0 + rr) + (int64_t)R * (a0 + b), acc[b], a.mode, a.scale);
    }
}

template <typename TI, typename TM, typename TO>
void launch_contract_m(const ContractM& a, cudaStream_t s) {
    constexpr int RT = 32, AB = 4;
    if (a.n_entries <= 0) return;
    const size_t smem = ((size_t)a.na * a.ni * sizeof(TM) + 15) / 16 * 16 + (size_t)a.ni * RT * sizeof(TI);
    static bool configured_dev[64] = {};
    int cur_dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&cur_dev));
    bool& configured = configured_dev[cur_dev & 63];
    if (!configured) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_contract_m<TI, TM, TO, RT, AB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        configured = true;
    }
    if (smem > 200 * 1024) throw std::runtime_error("contraction tile exceeds shared memory");
    const dim3 grid(a.n_entries, (a.R + RT - 1) / RT);
    k_contract_m<TI, TM, TO, RT, AB><<<grid, 256, smem, s>>>(a);
}

// ---------------------------------------------------------------------------
// plane-wave shift: grid (boxes in chunk, mode chunks, rhs)
// ---------------------------------------------------------------------------
// Each thread forms mode m of RB consecutive RHS: the box's (slot, stencil)
// terms sit in shared memory, every term's multiplier is read once for the RB
// RHS, and the RB plane-wave loads of a term are independent.
template <typename T, int RB>
__global__ void __launch_bounds__(256) k_shift_m(const typename Cplx<T>::type* __restrict__ pw_out,
                                                 const T* __restrict__ shift, typename Cplx<T>::type* __restrict__ pw_in,
                                                 int M, const int* __restrict__ term_start,
                                                 const int* __restrict__ term_slot, const int* __restrict__ term_stencil,
                                                 int kb, int e0) {
    using C = typename Cplx<T>::type;
    constexpr int kMaxTerms = 32;  // self + 26 colleagues
    __shared__ int s_slot[kMaxTerms], s_st[kMaxTerms];
    const int e = blockIdx.x, c0 = blockIdx.z * RB;
    const int tb = term_start[e0 + e];
    const int nterm = min(kMaxTerms, term_start[e0 + e + 1] - tb);
    if ((int)threadIdx.x < nterm) {
        s_slot[threadIdx.x] = term_slot[tb + threadIdx.x];
        s_st[threadIdx.x] = term_stencil[tb + threadIdx.x];
    }
    __syncthreads();
    const int m = blockIdx.y * blockDim.x + threadIdx.x;
    if (m >= M) return;
    T ar[RB], ai[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) ar[r] = ai[r] = T(0);
    for (int t = 0; t < nterm; ++t) {
        const T* sh = shift + (int64_t)s_st[t] * 2 * M;
        const T sr = sh[m], si = sh[M + m];
        const C* src = pw_out + ((int64_t)s_slot[t] * kb + c0) * M + m;
        C v[RB];
#pragma unroll
        for (int r = 0; r < RB; ++r) v[r] = (c0 + r < kb) ? src[(int64_t)r * M] : C{T(0), T(0)};
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            ar[r] = fma(v[r].x, sr, fma(-v[r].y, si, ar[r]));
            ai[r] = fma(v[r].x, si, fma(v[r].y, sr, ai[r]));
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r)
        if (c0 + r < kb) pw_in[((int64_t)e * kb + c0 + r) * M + m] = C{ar[r], ai[r]};
}

// ---------------------------------------------------------------------------
// proxy -> leaf targets: grid (leaves, 1, rhs)
// ---------------------------------------------------------------------------
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_eval_m(EvalArgs a, const T* __restrict__ proxy_down, double* __restrict__ pot, int64_t N, int kb) {
    __shared__ T slab[P * P];
    const int e = blockIdx.x, c = blockIdx.z;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const double4 cs = a.center_scale[e];
    const T* C = proxy_down + ((int64_t)a.slot[e] * kb + c) * (P * P * P);
    double* potc = pot + (int64_t)c * N;
    for (int base = 0; base < nt; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const bool act = t < nt;
        T tx[P];
        T y = T(0), z = T(0);
        {
            T x = T(0);
            if (act) {
                const double4 pt = a.trg[t0 + t];
                x = (T)((pt.x - cs.x) * cs.w);
                y = (T)((pt.y - cs.y) * cs.w);
                z = (T)((pt.z - cs.z) * cs.w);
            }
            tx[0] = T(1);
            if (P > 1) tx[1] = x;
#pragma unroll
            for (int n = 2; n < P; ++n) tx[n] = T(2) * x * tx[n - 1] - tx[n - 2];
        }
        T acc = T(0);
        T za = T(1), zb = z;
        for (int k = 0; k < P; ++k) {
            __syncthreads();
            for (int idx = threadIdx.x; idx < P * P; idx += blockDim.x) slab[idx] = C[(int64_t)k * P * P + idx];
            __syncthreads();
            T ya = T(1), yb = y, sk = T(0);
            for (int j = 0; j < P; ++j) {
                T r = T(0);
#pragma unroll
                for (int i = 0; i < P; ++i) r = fma(slab[i + P * j], tx[i], r);
                sk = fma(ya, r, sk);
                const T yn = T(2) * y * yb - ya;
                ya = yb;
                yb = yn;
            }
            acc = fma(za, sk, acc);
            const T zn = T(2) * z * zb - za;
            za = zb;
            zb = zn;
        }
        if (act) potc[t0 + t] += (double)acc;
    }
}

// ---------------------------------------------------------------------------
// residual near field with an RHS block of KB per pass
// ---------------------------------------------------------------------------
struct NearM {
    const int* trg_start;
    const int* trg_count;
    const int* pair_start;
    const int* pair_src_start;
    const int* pair_src_count;
    const double* pair_bsize;
    const int* pair_chunk_base;  // per near pair: first 32-source chunk box of its source box
    const float4* chunk_lo;      // per 32-source chunk: bounding box (rounded outwards)
    const float4* chunk_hi;
    double coef[32];
    int n_leaves;
    int64_t N;
    int kb;
};

// squared gap between a chunk's box and a target box b = (lo xyz, hi xyz)
__device__ __forceinline__ float chunk_gap2(const float4& lo, const float4& hi, const float* b) {
    const float gx = fmaxf(0.0f, fmaxf(lo.x - b[3], b[0] - hi.x));
    const float gy = fmaxf(0.0f, fmaxf(lo.y - b[4], b[1] - hi.y));
    const float gz = fmaxf(0.0f, fmaxf(lo.z - b[5], b[2] - hi.z));
    return fmaf(gx, gx, fmaf(gy, gy, gz * gz));
}

// FP64: positions double4, charges double[s * kb + c]
template <int NC, int KB>
__global__ void __launch_bounds__(128) k_near_m64(NearM a, const double4* __restrict__ trg,
                                                  const double4* __restrict__ src, const double* __restrict__ src_q,
                                                  double* __restrict__ pot) {
    constexpr int TPT = 2;
    __shared__ double4 ss[128];
    __shared__ double sq[128][KB];
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    double c[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) c[i] = a.coef[i];
    for (int cb = 0; cb < a.kb; cb += KB) {
        for (int base = 0; base < nt; base += TPT * 128) {
            double4 tp[TPT];
            double acc[TPT][KB];
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                const int t = base + threadIdx.x + u * 128;
                tp[u] = t < nt ? trg[t0 + t] : make_double4(1e300, 1e300, 1e300, 0.0);
#pragma unroll
                for (int q = 0; q < KB; ++q) acc[u][q] = 0.0;
            }
            for (int pr = a.pair_start[e]; pr < a.pair_start[e + 1]; ++pr) {
                const int s0 = a.pair_src_start[pr], ns = a.pair_src_count[pr];
                const double b = a.pair_bsize[pr];
                const double d2max = b * b, rsc = 2.0 / b, cen = -0.5 * b;
                for (int sb = 0; sb < ns; sb += 128) {
                    __syncthreads();
                    const int js = sb + threadIdx.x;
                    if (js < ns) {
                        ss[threadIdx.x] = src[s0 + js];
#pragma unroll
                        for (int q = 0; q < KB; ++q)
                            sq[threadIdx.x][q] = (cb + q < a.kb) ? src_q[(int64_t)(s0 + js) * a.kb + cb + q] : 0.0;
                    }
                    __syncthreads();
                    const int m = min(128, ns - sb);
                    for (int j = 0; j < m; ++j) {
                        const double4 y = ss[j];
#pragma unroll
                        for (int u = 0; u < TPT; ++u) {
                            const double dx = tp[u].x - y.x, dy = tp[u].y - y.y, dz = tp[u].z - y.z;
                            const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                            if (r2 > 1e-30 && r2 < d2max) {
                                const double rinv = rsqrt_nr(r2);
                                const double x = fma(r2, rinv, cen) * rsc;
                                double pv = c[NC - 1];
#pragma unroll
                                for (int i = NC - 2; i >= 0; --i) pv = fma(pv, x, c[i]);
                                const double w = pv * rinv;
#pragma unroll
                                for (int q = 0; q < KB; ++q) acc[u][q] = fma(w, sq[j][q], acc[u][q]);
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                const int t = base + threadIdx.x + u * 128;
                if (t < nt)
#pragma unroll
                    for (int q = 0; q < KB; ++q)
                        if (cb + q < a.kb) pot[(int64_t)(cb + q) * a.N + t0 + t] += acc[u][q];
            }
        }
    }
}

// FP32: double-float positions, FP32 pair arithmetic, per-box FP32 partial
// sums merged into FP64 accumulators.
template <int NC, int KB>
__global__ void __launch_bounds__(128) k_near_m32(NearM a, const float4* __restrict__ trg_hi,
                                                  const float4* __restrict__ trg_lo, const float4* __restrict__ src_hi,
                                                  const float4* __restrict__ src_lo, const float* __restrict__ src_q,
                                                  double* __restrict__ pot) {
    constexpr int TPT = 2;
    __shared__ float4 sh[128], sl[128];
    __shared__ float sq[128][KB];
    __shared__ float s_wbox[4][6];  // per warp: bounding box of its targets of the pass
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    float c[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) c[i] = (float)a.coef[i];
    for (int cb = 0; cb < a.kb; cb += KB) {
        for (int base = 0; base < nt; base += TPT * 128) {
            float4 th[TPT], tl[TPT];
            double acc[TPT][KB];
            float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                const int t = base + threadIdx.x + u * 128;
                th[u] = t < nt ? trg_hi[t0 + t] : make_float4(1e30f, 1e30f, 1e30f, 0.f);
                tl[u] = t < nt ? trg_lo[t0 + t] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int q = 0; q < KB; ++q) acc[u][q] = 0.0;
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
            __syncthreads();  // the previous pass is done with s_wbox
            if (lane == 0)
                for (int d = 0; d < 3; ++d) {
                    const float pad = 2.5e-7f * fmaxf(fabsf(lo[d]), fabsf(hi[d])) + 1e-30f;
                    s_wbox[warp][d] = lo[d] - pad;
                    s_wbox[warp][3 + d] = hi[d] + pad;
                }
            __syncthreads();
            float wbox[6], cbox[6];
            for (int d = 0; d < 6; ++d) wbox[d] = s_wbox[warp][d];
            for (int d = 0; d < 3; ++d) {
                cbox[d] = fminf(fminf(s_wbox[0][d], s_wbox[1][d]), fminf(s_wbox[2][d], s_wbox[3][d]));
                cbox[3 + d] = fmaxf(fmaxf(s_wbox[0][3 + d], s_wbox[1][3 + d]), fmaxf(s_wbox[2][3 + d], s_wbox[3][3 + d]));
            }
            for (int pr = a.pair_start[e]; pr < a.pair_start[e + 1]; ++pr) {
                const int s0 = a.pair_src_start[pr], ns = a.pair_src_count[pr];
                const double bd = a.pair_bsize[pr];
                const float d2max = (float)(bd * bd), rsc = (float)(2.0 / bd), cen = (float)(-0.5 * bd);
                const float keep2 = d2max * 1.00001f;
                const int cbase = a.pair_chunk_base[pr];
                float part[TPT][KB];
#pragma unroll
                for (int u = 0; u < TPT; ++u)
#pragma unroll
                    for (int q = 0; q < KB; ++q) part[u][q] = 0.f;
                for (int sb = 0; sb < ns; sb += 128) {
                    // 32-source chunks of this block within b of the pass's targets
                    // (the same answer in every thread: the skip is uniform)
                    const int nchk = min(4, (ns - sb + 31) / 32);
                    unsigned need = 0;
                    for (int k = 0; k < nchk; ++k) {
                        const int c = cbase + (sb >> 5) + k;
                        if (chunk_gap2(__ldg(a.chunk_lo + c), __ldg(a.chunk_hi + c), cbox) <= keep2) need |= 1u << k;
                    }
                    if (!need) continue;
                    __syncthreads();
                    const int js = sb + threadIdx.x;
                    if (js < ns && ((need >> (threadIdx.x >> 5)) & 1u)) {
                        sh[threadIdx.x] = src_hi[s0 + js];
                        sl[threadIdx.x] = src_lo[s0 + js];
#pragma unroll
                        for (int q = 0; q < KB; ++q)
                            sq[threadIdx.x][q] = (cb + q < a.kb) ? src_q[(int64_t)(s0 + js) * a.kb + cb + q] : 0.f;
                    }
                    __syncthreads();
                    const int m = min(128, ns - sb);
                    for (int k = 0; k < nchk; ++k) {
                    if (!((need >> k) & 1u)) continue;
                    {
                        const int c = cbase + (sb >> 5) + k;
                        // this warp's targets against the chunk (warp-uniform)
                        if (chunk_gap2(__ldg(a.chunk_lo + c), __ldg(a.chunk_hi + c), wbox) > keep2) continue;
                    }
                    const int je = min(m, 32 * k + 32);
                    for (int j = 32 * k; j < je; ++j) {
                        const float4 yh = sh[j], yl = sl[j];
#pragma unroll
                        for (int u = 0; u < TPT; ++u) {
                            const float dx = (th[u].x - yh.x) + (tl[u].x - yl.x);
                            const float dy = (th[u].y - yh.y) + (tl[u].y - yl.y);
                            const float dz = (th[u].z - yh.z) + (tl[u].z - yl.z);
                            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            if (r2 > 1e-30f && r2 < d2max) {
                                const float rinv = rsqrtf(r2);
                                const float x = fmaf(r2, rinv, cen) * rsc;
                                float pv = c[NC - 1];
#pragma unroll
                                for (int i = NC - 2; i >= 0; --i) pv = fmaf(pv, x, c[i]);
                                const float w = pv * rinv;
#pragma unroll
                                for (int q = 0; q < KB; ++q) part[u][q] = fmaf(w, sq[j][q], part[u][q]);
                            }
                        }
                    }
                    }
                }
#pragma unroll
                for (int u = 0; u < TPT; ++u)
#pragma unroll
                    for (int q = 0; q < KB; ++q) acc[u][q] += (double)part[u][q];
            }
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                const int t = base + threadIdx.x + u * 128;
                if (t < nt)
#pragma unroll
                    for (int q = 0; q < KB; ++q)
                        if (cb + q < a.kb) pot[(int64_t)(cb + q) * a.N + t0 + t] += acc[u][q];
            }
        }
    }
}

template <int KB>
static void launch_near_m64_kb(const NearM& a, const double4* trg, const double4* src, const double* q, double* pot,
                               int nc, cudaStream_t s) {
    switch (nc) {
#define C64(NC) case NC: k_near_m64<NC, KB><<<a.n_leaves, 128, 0, s>>>(a, trg, src, q, pot); break;
        C64(5) C64(6) C64(9) C64(11) C64(12) C64(15) C64(17) C64(18) C64(22) C64(23) C64(25)
#undef C64
        default: throw std::runtime_error("unsupported residual polynomial length");
    }
}

template <int KB>
static void launch_near_m32_kb(const NearM& a, const float4* th, const float4* tl, const float4* sh,
                               const float4* sl, const float* q, double* pot, int nc, cudaStream_t s) {
    switch (nc) {
#define C32(NC) case NC: k_near_m32<NC, KB><<<a.n_leaves, 128, 0, s>>>(a, th, tl, sh, sl, q, pot); break;
        C32(5) C32(6) C32(9) C32(11) C32(12) C32(15) C32(17) C32(18) C32(22) C32(23) C32(25)
#undef C32
        default: throw std::runtime_error("unsupported residual polynomial length");
    }
}

// ---------------------------------------------------------------------------
// fused separable transform out(a,b,c) (+)= sum Ux(a,i) Uy(b,j) Uz(c,k) in(i,j,k)
// for one (box, rhs) entry per CTA, the tensor held in shared memory.
// Matrices U_d column-major P x P at mat + mat_off[eb] + d*P*P.
// ---------------------------------------------------------------------------


// TRI: 0 dense; 1 U(a,i) = 0 for i > a (child -> parent); 2 U(a,i) = 0 for
// i < a (parent -> child).  The skipped entries are rounding-level zeros of
// the reference's triangular Chebyshev translation matrices.
// Column range [lo, hi) that segment s (contracted indices i in [SEG s,
// SEG s + SEG)) touches: all columns, or those a triangular matrix can have
// non-zero (a >= i for TRI 1, a <= i for TRI 2), widened to the segment.
template <int P, int TRI, int SEG>
__device__ __forceinline__ constexpr int seg_lo(int sg) { return TRI == 1 ? SEG * sg : 0; }
template <int P, int TRI, int SEG>
__device__ __forceinline__ constexpr int seg_hi(int sg) {
    return TRI == 2 ? (SEG * sg + SEG < P ? SEG * sg + SEG : P) : P;
}

// dst[r + P*P*a] = sum_i Ut[i*P + a] * src[i + P*r], two columns r per thread.
// The contracted index runs in segments of SEG (segment index unrolled, so
// each segment's column range is a compile-time constant; loop inside a
// segment kept rolled, which bounds the registers).
template <typename T, int P, int TRI>
__device__ __forceinline__ void sep3_step(const T* __restrict__ src, T* __restrict__ dst, const T* __restrict__ Ut,
                                          int nthr) {
    constexpr int SEG = 3, NSEG = (P + SEG - 1) / SEG;
    for (int r = threadIdx.x; r < P * P; r += 2 * nthr) {
        const int r2 = r + nthr;
        const bool two = r2 < P * P;
        T acc0[P], acc1[P];
#pragma unroll
        for (int a = 0; a < P; ++a) acc0[a] = acc1[a] = T(0);
#pragma unroll
        for (int sg = 0; sg < NSEG; ++sg) {
            const int i1 = SEG * sg + SEG < P ? SEG * sg + SEG : P;
#pragma unroll 1
            for (int i = SEG * sg; i < i1; ++i) {
                const T x0 = src[i + P * r];
                const T x1 = two ? src[i + P * r2] : T(0);
#pragma unroll
                for (int a = seg_lo<P, TRI, SEG>(sg); a < seg_hi<P, TRI, SEG>(sg); ++a) {
                    const T u = Ut[i * P + a];
                    acc0[a] = fma(u, x0, acc0[a]);
                    acc1[a] = fma(u, x1, acc1[a]);
                }
            }
        }
#pragma unroll
        for (int a = 0; a < P; ++a) {
            dst[r + P * P * a] = acc0[a];
            if (two) dst[r2 + P * P * a] = acc1[a];
        }
    }
}

template <typename T, int P, int TRI>
__global__ void k_sep3(Sep3 a) {
    extern __shared__ __align__(16) unsigned char smem_s3[];
    constexpr int P3 = P * P * P;
    T* b0 = reinterpret_cast<T*>(smem_s3);
    T* b1 = b0 + P3;
    T* Ut = b1 + P3;  // 3 transposed matrices
    const int64_t ge = a.e0 + blockIdx.x;
    const int rhs = a.rhs > 0 ? a.rhs : 1;
    const int64_t eb = ge / rhs, ec = ge % rhs;
    const T* in = reinterpret_cast<const T*>(a.in) + a.in_off[eb] * rhs + ec * P3;
    T* out = reinterpret_cast<T*>(a.out) + a.out_off[eb] * rhs + ec * P3;
    const T* mat = reinterpret_cast<const T*>(a.mat) + (a.mat_off ? a.mat_off[eb] : 0);
    const int nthr = blockDim.x;
    // input tensor: asynchronous 16-byte copies (all in flight at once) when
    // the source is 16-byte aligned, element loads otherwise
    if ((reinterpret_cast<uintptr_t>(in) & 15) == 0) {
        constexpr int NV = (int)(P3 * sizeof(T) / 16);
        for (int v = threadIdx.x; v < NV; v += nthr)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(b0 + v * (16 / sizeof(T)))),
                         "l"(in + v * (16 / sizeof(T)))
                         : "memory");
        asm volatile("cp.async.commit_group;" ::: "memory");
        for (int idx = NV * (int)(16 / sizeof(T)) + threadIdx.x; idx < P3; idx += nthr) b0[idx] = in[idx];
    } else {
        for (int idx = threadIdx.x; idx < P3; idx += nthr) b0[idx] = in[idx];
    }
    for (int idx = threadIdx.x; idx < 3 * P * P; idx += nthr) {
        const int d = idx / (P * P), w = idx % (P * P);
        const int i = w / P, aa = w % P;
        Ut[d * P * P + i * P + aa] = mat[d * P * P + aa + P * i];
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    sep3_step<T, P, TRI>(b0, b1, Ut, nthr);
    __syncthreads();
    sep3_step<T, P, TRI>(b1, b0, Ut + P * P, nthr);
    __syncthreads();
    // last step straight into the output (coalesced along r); with
    // accumulation all old values are loaded before the first store
    const T* Uz = Ut + 2 * P * P;
    constexpr int SEG = 3, NSEG = (P + SEG - 1) / SEG;
    for (int r = threadIdx.x; r < P * P; r += nthr) {
        T acc[P];
#pragma unroll
        for (int c = 0; c < P; ++c) acc[c] = a.accumulate ? out[r + P * P * c] : T(0);
#pragma unroll
        for (int sg = 0; sg < NSEG; ++sg) {
            const int k1 = SEG * sg + SEG < P ? SEG * sg + SEG : P;
#pragma unroll 1
            for (int k = SEG * sg; k < k1; ++k) {
                const T x = b0[k + P * r];
#pragma unroll
                for (int c = seg_lo<P, TRI, SEG>(sg); c < seg_hi<P, TRI, SEG>(sg); ++c)
                    acc[c] = fma(Uz[k * P + c], x, acc[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < P; ++c) out[r + P * P * c] = acc[c];
    }
}

template <typename T, int P>
static size_t sep3_smem() { return sizeof(T) * (2 * (size_t)P * P * P + 3 * (size_t)P * P); }

template <typename T, int P, int TRI>
static void launch_sep3_t(const Sep3& a, int n_entries, cudaStream_t s) {
    static bool configured_dev[64] = {};
    int cur_dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&cur_dev));
    bool& configured = configured_dev[cur_dev & 63];
    const size_t smem = sep3_smem<T, P>();
    if (!configured) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_sep3<T, P, TRI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = true;
    }
    const int thr = std::max(32, ((P * P + 1) / 2 + 31) / 32 * 32);
    k_sep3<T, P, TRI><<<n_entries, thr, smem, s>>>(a);
}

template <typename T, int P>
static void launch_sep3_p(const Sep3& a, int n_entries, cudaStream_t s) {
    if (P <= 18 && a.tri == 1) return launch_sep3_t<T, P, (P <= 18 ? 1 : 0)>(a, n_entries, s);
    if (P <= 18 && a.tri == 2) return launch_sep3_t<T, P, (P <= 18 ? 2 : 0)>(a, n_entries, s);
    launch_sep3_t<T, P, 0>(a, n_entries, s);
}

// true if the fused kernel handles (T, P) (tensor pair fits in shared memory)
template <typename T>
bool sep3_supported(int p) {
    if (p == 9 || p == 18) return true;
    if (p == 28) return sizeof(T) == 4;
    return false;
}

template <typename T>
void launch_sep3(const Sep3& a, int p, int n_entries, cudaStream_t s) {
    if (n_entries <= 0) return;
    switch (p) {
        case 9: launch_sep3_p<T, 9>(a, n_entries, s); break;
        case 18: launch_sep3_p<T, 18>(a, n_entries, s); break;
        case 28:
            if constexpr (sizeof(T) == 4) {
                launch_sep3_p<T, 28>(a, n_entries, s);
                break;
            }
            [[fallthrough]];
        default: throw std::runtime_error("fused transform not available for this order");
    }
}

template bool sep3_supported<float>(int);
template bool sep3_supported<double>(int);
template void launch_sep3<float>(const Sep3&, int, int, cudaStream_t);
template void launch_sep3<double>(const Sep3&, int, int, cudaStream_t);

// ---------------------------------------------------------------------------
// proxy -> leaf targets, TPT targets per thread: grid (leaves, 1, rhs)
// ---------------------------------------------------------------------------
template <typename T, int P, int TPT>
__device__ __forceinline__ void eval_leaf_g(const EvalArgs& a, int e, int c, const T* __restrict__ proxy_down,
                                            double* __restrict__ pot, int64_t N, int kb, T* slab) {
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const double4 cs = a.center_scale[e];
    const T* C = proxy_down + ((int64_t)a.slot[e] * kb + c) * (P * P * P);
    double* potc = pot + (int64_t)c * N;
    for (int base = 0; base < nt; base += TPT * blockDim.x) {
        T tx[TPT][P], y[TPT], z[TPT];
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
            const int t = base + threadIdx.x + u * blockDim.x;
            T x = T(0);
            y[u] = z[u] = T(0);
            if (t < nt) {
                const double4 pt = a.trg[t0 + t];
                x = (T)((pt.x - cs.x) * cs.w);
                y[u] = (T)((pt.y - cs.y) * cs.w);
                z[u] = (T)((pt.z - cs.z) * cs.w);
            }
            tx[u][0] = T(1);
            if (P > 1) tx[u][1] = x;
#pragma unroll
            for (int n = 2; n < P; ++n) tx[u][n] = T(2) * x * tx[u][n - 1] - tx[u][n - 2];
        }
        T acc[TPT], za[TPT], zb[TPT];
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
            acc[u] = T(0);
            za[u] = T(1);
            zb[u] = z[u];
        }
        for (int k = 0; k < P; ++k) {
            __syncthreads();
            for (int idx = threadIdx.x; idx < P * P; idx += blockDim.x) slab[idx] = C[(int64_t)k * P * P + idx];
            __syncthreads();
            T ya[TPT], yb[TPT], sk[TPT];
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                ya[u] = T(1);
                yb[u] = y[u];
                sk[u] = T(0);
            }
            for (int j = 0; j < P; ++j) {
                T rr[TPT];
#pragma unroll
                for (int u = 0; u < TPT; ++u) rr[u] = T(0);
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    const T cv = slab[i + P * j];
#pragma unroll
                    for (int u = 0; u < TPT; ++u) rr[u] = fma(cv, tx[u][i], rr[u]);
                }
#pragma unroll
                for (int u = 0; u < TPT; ++u) {
                    sk[u] = fma(ya[u], rr[u], sk[u]);
                    const T yn = T(2) * y[u] * yb[u] - ya[u];
                    ya[u] = yb[u];
                    yb[u] = yn;
                }
            }
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
                acc[u] = fma(za[u], sk[u], acc[u]);
                const T zn = T(2) * z[u] * zb[u] - za[u];
                za[u] = zb[u];
                zb[u] = zn;
            }
        }
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
            const int t = base + threadIdx.x + u * blockDim.x;
            if (t < nt) potc[t0 + t] += (double)acc[u];
        }
    }
}

template <typename T, int P, int TPT>
__global__ void __launch_bounds__(128)
    k_eval_g(EvalArgs a, const T* __restrict__ proxy_down, double* __restrict__ pot, int64_t N, int kb) {
    __shared__ T slab[P * P];
    eval_leaf_g<T, P, TPT>(a, blockIdx.x, blockIdx.z, proxy_down, pot, N, kb, slab);
}

// many systems' leaves in one grid (float trees, one RHS): item = (system, leaf)
template <int P, int TPT>
__global__ void __launch_bounds__(128) k_eval_batch(const EvalLeafSys* __restrict__ sys, const int2* __restrict__ items) {
    __shared__ float slab[P * P];
    const int2 it = items[blockIdx.x];
    const EvalLeafSys& S = sys[it.x];
    eval_leaf_g<float, P, TPT>(S.a, it.y, 0, S.proxy_down, S.pot, 0, 1, slab);
}

void launch_batch_eval(const EvalLeafSys* sys, const int2* items, int n_items, int p, cudaStream_t s) {
    if (n_items <= 0) return;
    // one target per thread, 64 threads per leaf: the batch's leaves are small
    // (a 64-thread CTA with 4 targets per thread left most lanes idle: 13.5
    // against 6.6 ms for the 512-system batch at p = 18)
    switch (p) {
        case 9: k_eval_batch<9, 1><<<n_items, 64, 0, s>>>(sys, items); break;
        case 18: k_eval_batch<18, 1><<<n_items, 64, 0, s>>>(sys, items); break;
        default: throw std::runtime_error("batched leaf evaluation: float trees have p = 9 or 18");
    }
    PDMK_CUDA_CHECK(cudaGetLastError());
}

}  // namespace dev

// ===========================================================================
// host side
// ===========================================================================
using dev::cd;
using dev::cf;

struct DeviceTree::MultiState {
    bool fp32 = false;
    int kb = 0;
    std::vector<void*> allocs;
    size_t bytes = 0;
    void* src_q = nullptr;
    void* proxy_up = nullptr;
    void* proxy_down = nullptr;
    void* pw_out = nullptr;
    void* s1 = nullptr;
    void* s2 = nullptr;
    void* pw_in = nullptr;
    int64_t scratch_bytes = 0;
    bool step_scratch = false;  // s1 / s2 hold scratch_bytes (else 256-byte placeholders)
    double* pot = nullptr;
    double* far = nullptr;
    double* q_t = nullptr;
    double* grid = nullptr;
    cd* spec = nullptr;
    cufftHandle fwd = 0, inv = 0;
    // overlapped host evaluates: far field of column chunks on a second stream
    cudaStream_t far_stream = nullptr;
    cufftHandle fwd_c = 0, inv_c = 0;  // batched plans over one chunk of columns
    int chunk_cols = 0;
    std::vector<cudaEvent_t> ev_chunk;  // chunk c's charges are on the device
    cudaEvent_t ev_far0 = nullptr, ev_far = nullptr;  // far-stream work begins / is done
    // FP32 copies of tables and positions
    float* c2p = nullptr;
    float* p2c = nullptr;
    struct Lev {
        cf *poly2pw = nullptr, *poly2pw_half = nullptr, *pw2polyT = nullptr, *pw2polyTw = nullptr;
        float* shift = nullptr;
    };
    std::vector<Lev> lev;
    float4 *src_hi = nullptr, *src_lo = nullptr, *trg_hi = nullptr, *trg_lo = nullptr;
    int* err = nullptr;  // set by tensor-core kernels whose pipeline wait timed out
    double* esw = nullptr;  // NUFFT spreading weights per sorted target (3 x W)
    float* esw32 = nullptr;  // the same in float (mixed-precision state: spreading)

    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        const size_t b = std::max<size_t>(n, 1) * sizeof(T);
        PDMK_CUDA_CHECK(cudaMalloc(&p, b));
        allocs.push_back(p);
        bytes += b;
        return static_cast<T*>(p);
    }
    ~MultiState() {
        if (fwd) cufftDestroy(fwd);
        if (inv) cufftDestroy(inv);
        if (fwd_c) cufftDestroy(fwd_c);
        if (inv_c) cufftDestroy(inv_c);
        if (far_stream) cudaStreamSynchronize(far_stream);
        for (cudaEvent_t e : ev_chunk) cudaEventDestroy(e);
        if (ev_far0) cudaEventDestroy(ev_far0);
        if (ev_far) cudaEventDestroy(ev_far);
        if (far_stream) cudaStreamDestroy(far_stream);
        for (void* p : allocs) cudaFree(p);
    }
};

void DeviceTree::MultiStateDeleter::operator()(MultiState* m) const { delete m; }

int DeviceTree::multi_block(int k, bool fp32) {
    // an existing state of this precision serves every k up to its block size
    const int pi = fp32 ? 1 : 0;
    if (kb_cache_k_[pi] == k && multi_[pi]) return kb_cache_[pi];
    kb_cache_k_[pi] = k;
    kb_cache_[pi] = multi_block_size(k, fp32);
    return kb_cache_[pi];
}

int DeviceTree::multi_block_size(int k, bool fp32) const {
    // bytes per RHS of the per-RHS buffers
    const int64_t ts = fp32 ? 4 : 8;
    const int64_t ncoef = (int64_t)p_ * p_ * p_;
    const int64_t per = ts * ((int64_t)n_all_ + (n_up_ + n_down_) * ncoef + 2 * n_pw_ * (int64_t)M_) +
                        8 * 3 * (int64_t)n_ + 8 * n_grid_ + 16 * n_spec_;
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    const int64_t budget = (int64_t)(0.5 * (double)freeb) - ((int64_t)3 << 30);
    int kb = (int)std::max<int64_t>(1, budget / std::max<int64_t>(per, 1));
    kb = std::min(kb, 64);
    kb = std::min(kb, std::max(1, k));
    return kb;
}

DeviceTree::MultiState& DeviceTree::multi_state(int kb, bool fp32) {
    auto& slot = multi_[fp32 ? 1 : 0];
    if (slot && slot->kb == kb) return *slot;
    slot.reset();
    std::unique_ptr<MultiState, MultiStateDeleter> m(new MultiState);
    m->fp32 = fp32;
    m->kb = kb;
    const int64_t ts = fp32 ? 4 : 8;
    const int64_t ncoef = (int64_t)p_ * p_ * p_;
    m->src_q = m->alloc<unsigned char>((size_t)(ts * n_all_ * kb));
    m->proxy_up = m->alloc<unsigned char>((size_t)(ts * n_up_ * ncoef * kb));
    m->proxy_down = m->alloc<unsigned char>((size_t)(ts * n_down_ * ncoef * kb));
    m->pw_out = m->alloc<unsigned char>((size_t)(2 * ts * n_pw_ * (int64_t)M_ * kb));
    // Scratch: the largest per-entry tensor of any transform step, for at
    // least one box with all kb RHS (the downward pass chunks by box).
    const int64_t per_entry = 2 * ts * std::max<int64_t>({(int64_t)p_ * p_ * npw_, (int64_t)p_ * npw_ * npw_,
                                                          (int64_t)npw_ * npw2_ * p_, (int64_t)npw2_ * p_ * p_,
                                                          (int64_t)M_, ncoef});
    // enough for the largest batched step (all boxes of a group, all kb RHS),
    // capped at 512 MB (larger steps are chunked), never below one box
    int64_t max_boxes = 1;
    for (const auto& g : c2p_groups_) max_boxes = std::max<int64_t>(max_boxes, g.n);
    for (const auto& g : pw_groups_) max_boxes = std::max<int64_t>(max_boxes, g.n);
    for (const auto& E : eval_levels_) max_boxes = std::max<int64_t>({max_boxes, (int64_t)E.n, (int64_t)E.n_p2c});
    m->scratch_bytes = std::max<int64_t>(per_entry * kb, std::min<int64_t>((int64_t)512 << 20, per_entry * kb * max_boxes));
    // s1 / s2 hold step-by-step transform intermediates; the fused transforms need
    // none, but the tensor-core transforms (PDMK_TC_MASK bit 3) run step by step
    // in place of the fused kernels and need them at full size
    const bool fused_all = fp32 ? (dev::sep3_supported<float>(p_) && dev::pw_fused_supported<float>(p_, npw_, npw2_))
                                : (dev::sep3_supported<double>(p_) && dev::pw_fused_supported<double>(p_, npw_, npw2_));
    const bool tc_steps = fp32 && (tc_mask_ & 8);
    const size_t s12 = fused_all && !tc_steps ? 256 : (size_t)m->scratch_bytes;
    m->s1 = m->alloc<unsigned char>(s12);
    m->s2 = m->alloc<unsigned char>(s12);
    m->step_scratch = s12 == (size_t)m->scratch_bytes;
    m->pw_in = m->alloc<unsigned char>((size_t)m->scratch_bytes);
    m->pot = m->alloc<double>((size_t)n_ * kb);
    m->far = m->alloc<double>((size_t)n_ * kb);
    m->q_t = m->alloc<double>((size_t)n_ * kb);
    m->grid = m->alloc<double>((size_t)(n_grid_ * kb));
    m->err = m->alloc<int>(1);
    PDMK_CUDA_CHECK(cudaMemsetAsync(m->err, 0, sizeof(int), stream_));
    m->esw = m->alloc<double>((size_t)n_ * 3 * nufft_.w);
    dev::launch_es_weights(nufft_, n_, m->esw, stream_);
    if (fp32) {
        m->esw32 = m->alloc<float>((size_t)n_ * 3 * nufft_.w);
        dev::launch_to_float(m->esw, m->esw32, (int64_t)n_ * 3 * nufft_.w, stream_);
    }
    m->spec = m->alloc<cd>((size_t)(n_spec_ * kb));
    {
        int dims[3] = {nufft_.n1, nufft_.n2, nufft_.n3};
        const cufftResult r1 =
            cufftPlanMany(&m->fwd, 3, dims, nullptr, 1, (int)n_grid_, nullptr, 1, (int)n_spec_, CUFFT_D2Z, kb);
        const cufftResult r2 =
            cufftPlanMany(&m->inv, 3, dims, nullptr, 1, (int)n_spec_, nullptr, 1, (int)n_grid_, CUFFT_Z2D, kb);
        if (r1 != CUFFT_SUCCESS || r2 != CUFFT_SUCCESS)
            throw std::runtime_error("cuFFT error: batched plan creation failed");
        cufftSetStream(m->fwd, stream_);
        cufftSetStream(m->inv, stream_);
    }
    if (fp32) {
        auto conv = [&](const void* src, int64_t n_doubles) {
            float* d = m->alloc<float>((size_t)n_doubles);
            dev::k_to_float<<<(unsigned)((n_doubles + 255) / 256), 256, 0, stream_>>>(static_cast<const double*>(src), d,
                                                                                      n_doubles);
            return d;
        };
        const int64_t pp = (int64_t)p_ * p_;
        m->c2p = conv(c2p_, 8 * 3 * pp);
        m->p2c = conv(p2c_, 8 * 3 * pp);
        m->lev.resize(lev_.size());
        for (size_t l = 0; l < lev_.size(); ++l) {
            m->lev[l].poly2pw = reinterpret_cast<cf*>(conv(lev_[l].poly2pw, 2 * (int64_t)npw_ * p_));
            m->lev[l].poly2pw_half = reinterpret_cast<cf*>(conv(lev_[l].poly2pw_half, 2 * (int64_t)npw2_ * p_));
            m->lev[l].pw2polyT = reinterpret_cast<cf*>(conv(lev_[l].pw2polyT, 2 * (int64_t)npw_ * p_));
            m->lev[l].pw2polyTw = reinterpret_cast<cf*>(conv(lev_[l].pw2polyTw, 2 * (int64_t)npw2_ * p_));
            m->lev[l].shift = conv(lev_[l].shift, 27 * 2 * (int64_t)M_);
        }
        m->src_hi = m->alloc<float4>(n_all_);
        m->src_lo = m->alloc<float4>(n_all_);
        m->trg_hi = m->alloc<float4>(n_);
        m->trg_lo = m->alloc<float4>(n_);
        dev::k_split_positions<<<(n_all_ + 255) / 256, 256, 0, stream_>>>(src_, m->src_hi, m->src_lo, n_all_);
        dev::k_split_positions<<<(n_ + 255) / 256, 256, 0, stream_>>>(trg_, m->trg_hi, m->trg_lo, n_);
    }
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
    slot = std::move(m);
    return *slot;
}

template <typename T>
void DeviceTree::run_multi_block(MultiState& m, const double* Q, int kvalid, double* pot_user) {
    using C = typename dev::Cplx<T>::type;
    constexpr bool f32 = std::is_same<T, float>::value;
    const int p = p_, n = npw_, n2 = npw2_, M = M_;
    const int64_t ncoef = (int64_t)p * p * p;
    const int kb = m.kb;
    cudaStream_t s = stream_;
    T* src_q = static_cast<T*>(m.src_q);
    T* up = static_cast<T*>(m.proxy_up);
    T* down = static_cast<T*>(m.proxy_down);
    C* pw = static_cast<C*>(m.pw_out);
    const T* c2pm = f32 ? reinterpret_cast<const T*>(m.c2p) : reinterpret_cast<const T*>(c2p_);
    const T* p2cm = f32 ? reinterpret_cast<const T*>(m.p2c) : reinterpret_cast<const T*>(p2c_);
    auto levtab = [&](int l, int which) -> const void* {
        if (f32) {
            const auto& L = m.lev[l];
            return which == 0 ? (const void*)L.poly2pw : which == 1 ? (const void*)L.poly2pw_half
                 : which == 2 ? (const void*)L.pw2polyT : which == 3 ? (const void*)L.pw2polyTw : (const void*)L.shift;
        }
        const auto& L = lev_[l];
        return which == 0 ? (const void*)L.poly2pw : which == 1 ? (const void*)L.poly2pw_half
             : which == 2 ? (const void*)L.pw2polyT : which == 3 ? (const void*)L.pw2polyTw : (const void*)L.shift;
    };
    const int64_t sbytes = m.scratch_bytes;

    // quasi-periodic trees run only the two-column form (qp.cu)
    const bool qp = !f32 && qp_run_;
    if (qp_ && !qp) require_periodic("evaluate_multi");
    if (qp && (kb != 2 || kvalid != 1)) throw std::logic_error("quasi-periodic evaluate: two-column state expected");
    int nl = 0;
    if (far_ext_ && qp) throw std::logic_error("quasi-periodic evaluate with an external far field");
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[0], s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(up, 0, sizeof(T) * std::max<int64_t>(n_up_ * ncoef * kb, 1), s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(down, 0, sizeof(T) * std::max<int64_t>(n_down_ * ncoef * kb, 1), s));
    if (qp) {
        // the phased charges q e^{i bloch.R} per sorted source (two columns, rows
        // per source) and q e^{-i bloch.x} per sorted target for the far field
        dev::launch_qp_charges(reinterpret_cast<double*>(src_q), src_charge_idx_, qp_src_phase_, n_all_, m.q_t,
                               trg_perm_, qp_trg_phase_, n_, Q, s);
        nl += 2;
    } else {
        // charges to row-major (the potential buffer is free until it is zeroed
        // below), then one contiguous row per source
        const int64_t tot = (int64_t)n_all_ * kb;
        const dim3 tgrid((unsigned)((n_ + 31) / 32), (unsigned)((kb + 31) / 32));
        dev::k_transpose_q<<<tgrid, dim3(32, 8), 0, s>>>(Q, m.pot, n_, kb, kvalid); ++nl;
        dev::k_gather_src_rows<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(src_q, src_charge_idx_, m.pot, n_all_,
                                                                                kb); ++nl;
        if (!far_ext_) {
            const int64_t tt = (int64_t)n_ * kb;
            dev::k_gather_trg_m<<<(unsigned)((tt + 255) / 256), 256, 0, s>>>(m.q_t, trg_perm_, Q, n_, kb, kvalid); ++nl;
        }
    }
    PDMK_CUDA_CHECK(cudaMemsetAsync(m.pot, 0, sizeof(double) * n_ * kb, s));
    // proxy moments: tensor-core GEMM (FP32 blocks of >= 16 RHS), else per-RHS CUDA-core kernel
    if (c2x_.n_centers > 0) {
        bool done = false;
        if constexpr (f32) {
            if (tc_mask_ & 1) done = dev::launch_c2proxy_tc(c2x_, src_q, up, kb, p, m.err, s);
        }
        if (done) {
            ++nl;
        } else {
            const dim3 grid(c2x_.n_centers, (p * p + 127) / 128, kb);
            switch (p) {
                case 9: dev::k_c2proxy_m<T, 9><<<grid, 128, 0, s>>>(c2x_, src_q, up, kb); break;
                case 18: dev::k_c2proxy_m<T, 18><<<grid, 128, 0, s>>>(c2x_, src_q, up, kb); break;
                case 28: dev::k_c2proxy_m<T, 28><<<grid, 128, 0, s>>>(c2x_, src_q, up, kb); break;
                case 38: dev::k_c2proxy_m<T, 38><<<grid, 128, 0, s>>>(c2x_, src_q, up, kb); break;
                default: throw std::runtime_error("unsupported expansion order");
            }
            ++nl;
        }
    }
    // Transforms on the tensor cores (FP32 blocks, PDMK_TC_MASK bit 3): every
    // separable step is one tcgen05 contraction (contract_tc.cu); the chunks
    // of (box, RHS) entries are sized so that the step intermediates stay in L2.
    const bool tc_tr = f32 && (tc_mask_ & 8) && m.step_scratch && dev::contract_tc_supported(n, n, 2, 2) &&
                       dev::contract_tc_supported(p, p, 1, 1);
    const int64_t l2_scratch = 64ll << 20;
    // chunked batched contraction helper over (box, rhs) entries
    auto chunked = [&](int n_boxes, int64_t per_entry_bytes, auto&& body) {
        const int64_t total = (int64_t)n_boxes * kb;
        int64_t C = std::max<int64_t>(1, sbytes / std::max<int64_t>(per_entry_bytes, 1));
        if (tc_tr) C = std::max<int64_t>(1, std::min<int64_t>(C, l2_scratch / std::max<int64_t>(per_entry_bytes, 1)));
        for (int64_t e0 = 0; e0 < total; e0 += C) body(e0, (int)std::min<int64_t>(C, total - e0));
    };
    // one contraction step: tensor cores when selected, else the CUDA-core kernel
    // (ci / co: 1 real, 2 complex input / output; cm: complex matrix)
    auto step = [&](const dev::ContractM& c, int ci, int co, bool cm, auto launch_cuda_core) {
        if (tc_tr) {
            dev::ContractTc t{};
            t.in = static_cast<const float*>(c.in); t.in_off = c.in_off; t.in_stride = c.in_stride; t.in_unit = c.in_unit;
            t.out = static_cast<float*>(c.out); t.out_off = c.out_off; t.out_stride = c.out_stride; t.out_unit = c.out_unit;
            t.mat = static_cast<const float*>(c.mat); t.mat_off = c.mat_off; t.mat_complex = cm ? 1 : 0;
            t.ni = c.ni; t.na = c.na; t.R = c.R; t.ci = ci; t.co = co; t.rhs = c.rhs; t.e0 = c.e0;
            t.n_entries = c.n_entries; t.accumulate = c.mode != dev::kStore ? 1 : 0;
            t.scale = c.mode == dev::kAddRealScaled ? (float)c.scale : 1.0f; t.err = m.err;
            dev::launch_contract_tc(t, s);
        } else {
            launch_cuda_core(c);
        }
    };
    const bool fused = dev::sep3_supported<T>(p) && !tc_tr;
    if (!m.step_scratch && (!fused || !dev::pw_fused_supported<T>(p, n, n2)))
        throw std::logic_error("multi-RHS state without step scratch");
    // upward children -> parents
    for (const auto& g : c2p_groups_) {
        const T* mx = c2pm + (int64_t)g.child * 3 * p * p;
        if (fused) {
            dev::Sep3 f{};
            f.in = up; f.in_off = g.in_off; f.out = up; f.out_off = g.out_off; f.mat = mx; f.rhs = kb;
            f.accumulate = 1; f.tri = 1;
            dev::launch_sep3<T>(f, p, g.n * kb, s); ++nl;
            continue;
        }
        chunked(g.n, (int64_t)sizeof(T) * ncoef * 2, [&](int64_t e0, int ne) {
            auto rrr = [&](const dev::ContractM& c) { dev::launch_contract_m<T, T, T>(c, s); };
            dev::ContractM a{};
            a.rhs = kb; a.e0 = e0; a.n_entries = ne;
            a.in = up; a.in_off = g.in_off; a.in_unit = ncoef; a.out = m.s1; a.out_stride = ncoef;
            a.mat = mx; a.ni = p; a.na = p; a.R = p * p; a.mode = dev::kStore;
            step(a, 1, 1, false, rrr); ++nl;
            a.in = m.s1; a.in_off = nullptr; a.in_stride = ncoef; a.out = m.s2; a.mat = mx + p * p;
            step(a, 1, 1, false, rrr); ++nl;
            a.in = m.s2; a.out = up; a.out_off = g.out_off; a.out_unit = ncoef; a.mat = mx + 2 * p * p; a.mode = dev::kAdd;
            step(a, 1, 1, false, rrr); ++nl;
        });
    }
    // outgoing plane waves
    const bool pw_fused = dev::pw_fused_supported<T>(p, n, n2) && !tc_tr;
    for (const auto& g : pw_groups_) {
        if (pw_fused) {
            dev::PwFused f{};
            f.in = up; f.in_off = g.in_off; f.out = pw; f.out_off = g.out_off;
            f.mat_a = levtab(g.level, 0); f.mat_b = levtab(g.level, 1); f.rhs = kb; f.e0 = 0;
            dev::launch_pw_out_fused<T>(f, p, n, n2, g.n * kb, s); ++nl;
            continue;
        }
        const int64_t e1 = (int64_t)p * p * n, e2 = (int64_t)p * n * n;
        chunked(g.n, (int64_t)sizeof(C) * (tc_tr ? e1 + e2 : std::max(e1, e2)), [&](int64_t e0, int ne) {
            auto rcc = [&](const dev::ContractM& c) { dev::launch_contract_m<T, C, C>(c, s); };
            auto ccc = [&](const dev::ContractM& c) { dev::launch_contract_m<C, C, C>(c, s); };
            dev::ContractM a{};
            a.rhs = kb; a.e0 = e0; a.n_entries = ne;
            a.in = up; a.in_off = g.in_off; a.in_unit = ncoef; a.out = m.s1; a.out_stride = e1;
            a.mat = levtab(g.level, 0); a.ni = p; a.na = n; a.R = p * p; a.mode = dev::kStore;
            step(a, 1, 2, true, rcc); ++nl;
            a.in = m.s1; a.in_off = nullptr; a.in_stride = e1; a.out = m.s2; a.out_stride = e2; a.R = p * n;
            step(a, 2, 2, true, ccc); ++nl;
            a.in = m.s2; a.in_stride = e2; a.out = pw; a.out_off = g.out_off; a.out_unit = M;
            a.mat = levtab(g.level, 1); a.na = n2; a.R = n * n;
            step(a, 2, 2, true, ccc); ++nl;
        });
    }
    // downward per level
    for (const auto& E : eval_levels_) {
        const int64_t e1 = (int64_t)n * n2 * p, e2 = (int64_t)n2 * p * p;
        // chunk over boxes (all rhs of a box together): pw_in holds C boxes x kb x M
        const int64_t per_box = (int64_t)sizeof(C) * std::max<int64_t>({(int64_t)M, e1, e2}) * kb;
        const int Cb = (int)std::max<int64_t>(1, sbytes / per_box);
        for (int b0 = 0; b0 < E.n; b0 += Cb) {
            const int nb = std::min(Cb, E.n - b0);
            {
                // eight RHS per thread for wide blocks (each shift weight feeds
                // more products: 85.45 -> 84.95 ms per 64-RHS evaluate), four otherwise
                if (kb >= 8) {
                    const dim3 grid(nb, (M + 255) / 256, (kb + 7) / 8);
                    dev::k_shift_m<T, 8><<<grid, 256, 0, s>>>(pw, static_cast<const T*>(levtab(E.level, 4)),
                                                           static_cast<C*>(m.pw_in), M, E.term_start, E.term_slot,
                                                           E.term_stencil, kb, b0); ++nl;
                } else {
                    const dim3 grid(nb, (M + 255) / 256, (kb + 3) / 4);
                    dev::k_shift_m<T, 4><<<grid, 256, 0, s>>>(pw, static_cast<const T*>(levtab(E.level, 4)),
                                                           static_cast<C*>(m.pw_in), M, E.term_start, E.term_slot,
                                                           E.term_stencil, kb, b0); ++nl;
                }
            }
            if (pw_fused) {
                dev::PwFused f{};
                f.in = m.pw_in; f.in_stride = M; f.out = down; f.out_off = E.down_off;
                f.mat_a = levtab(E.level, 2); f.mat_b = levtab(E.level, 3); f.rhs = kb; f.e0 = (int64_t)b0 * kb;
                dev::launch_pw_in_fused<T>(f, p, n, n2, nb * kb, s); ++nl;
                continue;
            }
            auto ccc = [&](const dev::ContractM& c) { dev::launch_contract_m<C, C, C>(c, s); };
            auto ccr = [&](const dev::ContractM& c) { dev::launch_contract_m<C, C, T>(c, s); };
            dev::ContractM a{};
            a.rhs = kb; a.e0 = (int64_t)b0 * kb; a.n_entries = nb * kb;
            a.in = m.pw_in; a.in_stride = M; a.out = m.s1; a.out_stride = e1;
            a.mat = levtab(E.level, 2); a.ni = n; a.na = p; a.R = n * n2; a.mode = dev::kStore;
            step(a, 2, 2, true, ccc); ++nl;
            a.in = m.s1; a.in_stride = e1; a.out = m.s2; a.out_stride = e2; a.R = n2 * p;
            step(a, 2, 2, true, ccc); ++nl;
            a.in = m.s2; a.in_stride = e2; a.out = down; a.out_off = E.down_off; a.out_unit = ncoef;
            a.mat = levtab(E.level, 3); a.ni = n2; a.R = p * p; a.mode = dev::kAddRealScaled; a.scale = 2.0;
            step(a, 2, 1, true, ccr); ++nl;
        }
        if (E.n_p2c && fused) {
            dev::Sep3 f{};
            f.in = down; f.in_off = E.p2c_in; f.out = down; f.out_off = E.p2c_out; f.mat = p2cm;
            // first write of the children's coefficients (one parent each; their
            // own incoming expansions are added at the next level): store
            f.mat_off = E.p2c_mat; f.rhs = kb; f.accumulate = 0; f.tri = 2;
            dev::launch_sep3<T>(f, p, E.n_p2c * kb, s); ++nl;
        } else if (E.n_p2c) {
            chunked(E.n_p2c, (int64_t)sizeof(T) * ncoef * 2, [&](int64_t e0, int ne) {
                auto rrr = [&](const dev::ContractM& c) { dev::launch_contract_m<T, T, T>(c, s); };
                dev::ContractM b{};
                b.rhs = kb; b.e0 = e0; b.n_entries = ne;
                b.in = down; b.in_off = E.p2c_in; b.in_unit = ncoef; b.out = m.s1; b.out_stride = ncoef;
                b.mat = p2cm; b.mat_off = E.p2c_mat; b.ni = p; b.na = p; b.R = p * p; b.mode = dev::kStore;
                step(b, 1, 1, false, rrr); ++nl;
                b.in = m.s1; b.in_off = nullptr; b.in_stride = ncoef; b.out = m.s2; b.mat = p2cm + p * p;
                b.mat_off = E.p2c_mat;
                step(b, 1, 1, false, rrr); ++nl;
                b.in = m.s2; b.out = down; b.out_off = E.p2c_out; b.out_unit = ncoef; b.mat = p2cm + 2 * p * p;
                b.mode = dev::kAdd;
                step(b, 1, 1, false, rrr); ++nl;
            });
        }
    }
    // leaf evaluation: tensor-core GEMM for FP32 blocks of 16/32/64 RHS, else CUDA cores
    bool eval_done = false;
    if constexpr (f32) {
        if ((tc_mask_ & 4) && eval_.n_leaves > 0) {
            dev::EvalTc t{};
            t.trg = trg_; t.proxy_down = reinterpret_cast<const float*>(down); t.pot = m.pot;
            t.n_leaves = eval_.n_leaves; t.max_trg = eval_max_trg_; t.slot = eval_.slot;
            t.trg_start = eval_.trg_start; t.trg_count = eval_.trg_count; t.center_scale = eval_.center_scale;
            t.N = n_;
            eval_done = dev::launch_eval_tc(t, p, kb, m.err, s);
            if (eval_done) ++nl;
        }
    }
    // leaf evaluation and near field are left to the batch's launches over
    // all systems when deferred (float trees of a batch, one RHS)
    const bool deferred = f32 && defer_near_ && kb == 1;
    if (eval_.n_leaves > 0 && !eval_done && !deferred) {
        const dim3 grid(eval_.n_leaves, 1, kb);
        switch (p) {
            case 9: dev::k_eval_g<T, 9, 4><<<grid, 64, 0, s>>>(eval_, down, m.pot, n_, kb); ++nl; break;
            case 18: dev::k_eval_g<T, 18, 4><<<grid, 64, 0, s>>>(eval_, down, m.pot, n_, kb); ++nl; break;
            case 28: dev::k_eval_g<T, 28, 2><<<grid, 128, 0, s>>>(eval_, down, m.pot, n_, kb); ++nl; break;
            case 38: dev::k_eval_g<T, 38, 2><<<grid, 128, 0, s>>>(eval_, down, m.pot, n_, kb); ++nl; break;
            default: throw std::runtime_error("unsupported expansion order");
        }
    }
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[1], s));
    // near field (left to the batch's queue kernel when deferred)
    if (near_.n_leaves > 0 && !deferred) {
        dev::NearM a{};
        a.trg_start = near_.trg_start; a.trg_count = near_.trg_count; a.pair_start = near_.pair_start;
        a.pair_src_start = near_.pair_src_start; a.pair_src_count = near_.pair_src_count;
        a.pair_bsize = near_.pair_bsize; a.n_leaves = near_.n_leaves; a.N = n_; a.kb = kb;
        a.pair_chunk_base = near_.pair_chunk_base; a.chunk_lo = near_.chunk_lo; a.chunk_hi = near_.chunk_hi;
        for (int i = 0; i < near_.nc; ++i) a.coef[i] = near_.coef[i];
        bool tc_done = false;
        if constexpr (f32) {
            // tensor cores for blocks of 16+ RHS; a single RHS keeps 15/16 of every MMA idle
            // and the CUDA-core kernel's occupancy wins
            if ((tc_mask_ & 2) && kb >= 16 && near_max_pairs_ <= dev::kNearTcMaxPairs &&
                near_max_chunks_ <= dev::kNearTcMaxChunks) {
                dev::NearTc t{};
                t.trg_start = near_.trg_start; t.trg_count = near_.trg_count; t.pair_start = near_.pair_start;
                t.pair_src_start = near_.pair_src_start; t.pair_src_count = near_.pair_src_count;
                t.pair_bsize = near_.pair_bsize; t.n_leaves = near_.n_leaves; t.max_trg = near_max_trg_;
                t.pair_chunk_base = near_pair_chunk_base_; t.chunk_lo = near_chunk_lo_; t.chunk_hi = near_chunk_hi_;
                t.N = n_; t.kb = kb;
                for (int i = 0; i < near_.nc; ++i) t.coef[i] = near_.coef[i];
                // Test hook of the failure detection (never set in normal use):
                // PDMK_TEST_WITHHOLD_NEAR_CHUNK=j makes the first tile withhold
                // chunk j's MMAs and commits; its next pipeline wait then runs
                // out after ~10 ms, the kernel aborts cleanly and sets the error
                // word, and the evaluate returns -2.
                // segment length between FP64 drains (tuning: PDMK_NEAR_SEG)
                t.seg_chunks = 0;
                if (const char* sg = std::getenv("PDMK_NEAR_SEG")) t.seg_chunks = std::atoi(sg);
                t.withhold_chunk = -1;
                t.wait_cycles = 4000000000LL;
                if (const char* w = std::getenv("PDMK_TEST_WITHHOLD_NEAR_CHUNK")) {
                    t.withhold_chunk = std::atoi(w);
                    t.wait_cycles = 20000000LL;
                }
                tc_done = dev::launch_near_tc(t, near_.nc, m.trg_hi, m.trg_lo, m.src_hi, m.src_lo,
                                              reinterpret_cast<const float*>(src_q), m.pot, m.err, s);
            }
        }
        if (tc_done) {
        } else if constexpr (f32) {
            if (kb >= 16)
                dev::launch_near_m32_kb<16>(a, m.trg_hi, m.trg_lo, m.src_hi, m.src_lo, reinterpret_cast<const float*>(src_q),
                                            m.pot, near_.nc, s);
            else if (kb >= 4)
                dev::launch_near_m32_kb<4>(a, m.trg_hi, m.trg_lo, m.src_hi, m.src_lo, reinterpret_cast<const float*>(src_q),
                                           m.pot, near_.nc, s);
            else
                dev::launch_near_m32_kb<1>(a, m.trg_hi, m.trg_lo, m.src_hi, m.src_lo, reinterpret_cast<const float*>(src_q),
                                           m.pot, near_.nc, s);
        } else {
            if (kb >= 8)
                dev::launch_near_m64_kb<8>(a, trg_, src_, reinterpret_cast<const double*>(src_q), m.pot, near_.nc, s);
            else
                dev::launch_near_m64_kb<1>(a, trg_, src_, reinterpret_cast<const double*>(src_q), m.pot, near_.nc, s);
        }
        ++nl;
    }
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[2], s));
    // far field, FP64, all rhs of the block at once (or, in an overlapped host
    // evaluate, already enqueued on the far-field stream by column chunks)
    if (far_ext_)
        PDMK_CUDA_CHECK(cudaStreamWaitEvent(s, far_ext_event_, 0));
    else
        nl += far_columns(m, 0, kb, qp, m.fwd, m.inv, s, /*interp=*/!deferred);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[3], s));
    if (qp) {
        dev::launch_qp_finalize(m.pot, m.far, trg_, trg_perm_, Q, qp_trg_phase_, pot_user, n_, s); ++nl;
    } else if (!deferred) {
        const int64_t tot = (int64_t)n_ * kvalid;
        dev::k_finalize_m<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m.pot, m.far, trg_, trg_perm_, m.q_t, pot_user,
                                                                        n_, kvalid); ++nl;
    }
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[4], s));
    PDMK_CUDA_CHECK(cudaGetLastError());
    multi_launches_ += nl;
}

void DeviceTree::interp_sys(dev::InterpSys& d) const {
    const MultiState* m = multi_[1].get();
    if (!m || m->kb != 1) throw std::logic_error("interp_sys: no single-RHS float state");
    d.a = nufft_;
    d.a.q_sorted = m->q_t;
    d.a.grid = m->grid;
    d.a.far = m->far;
    d.a.rhs_q_stride = n_;
    d.a.rhs_grid_stride = n_grid_;
    d.a.rhs_far_stride = n_;
    d.esw = m->esw;
    d.n = n_;
}

void DeviceTree::eval_leaf_sys(dev::EvalLeafSys& d) const {
    const MultiState* m = multi_[1].get();
    if (!m || m->kb != 1) throw std::logic_error("eval_leaf_sys: no single-RHS float state");
    d.a = eval_;
    d.proxy_down = static_cast<const float*>(m->proxy_down);
    d.pot = m->pot;
}

void DeviceTree::near_leaf_sys(dev::NearLeafSys& d, double* out) const {
    const MultiState* m = multi_[1].get();
    if (!m || m->kb != 1) throw std::logic_error("near_leaf_sys: no single-RHS float state");
    d.trg_start = near_.trg_start;
    d.trg_count = near_.trg_count;
    d.pair_start = near_.pair_start;
    d.pair_src_start = near_.pair_src_start;
    d.pair_src_count = near_.pair_src_count;
    d.pair_bsize = near_.pair_bsize;
    d.pair_chunk_base = near_.pair_chunk_base;
    d.chunk_lo = near_.chunk_lo;
    d.chunk_hi = near_.chunk_hi;
    d.trg_hi = m->trg_hi;
    d.trg_lo = m->trg_lo;
    d.src_hi = m->src_hi;
    d.src_lo = m->src_lo;
    d.src_q = static_cast<const float*>(m->src_q);
    d.pot = m->pot;
    d.far = m->far;
    d.trg = trg_;
    d.perm = trg_perm_;
    d.q_t = m->q_t;
    d.out = out;
}

int DeviceTree::far_columns(MultiState& m, int c0, int cols, bool qp, cufftHandle fwd, cufftHandle inv,
                            cudaStream_t s, bool interp) {
    dev::NufftArgs na = nufft_;
    na.q_sorted = m.q_t + (int64_t)c0 * n_;
    na.grid = m.grid + (int64_t)c0 * n_grid_;
    na.far = m.far + (int64_t)c0 * n_;
    na.rhs_q_stride = n_;
    na.rhs_grid_stride = n_grid_;
    na.rhs_far_stride = n_;
    cd* spec = m.spec + (int64_t)c0 * n_spec_;
    PDMK_CUDA_CHECK(cudaMemsetAsync(na.grid, 0, sizeof(double) * n_grid_ * cols, s));
    // mixed precision: spreading with single-precision taps and partial sums
    // into the FP64 grid; transforms and interpolation stay FP64
    // (single-precision interpolation sums lost accuracy for no speed)
    bool spread32 = false;
    if (m.fp32) spread32 = dev::launch_spread_multi_f32(na, m.esw32, cols, s);
    if (!spread32) dev::launch_spread_multi(na, m.esw, nufft_max_jk_, nufft_max_ex_, cols, s);
    if (cufftExecD2Z(fwd, na.grid, reinterpret_cast<cufftDoubleComplex*>(spec)) != CUFFT_SUCCESS)
        throw std::runtime_error("cuFFT error in the batched forward transform");
    if (qp)
        dev::launch_qp_combine(spec, qp_s_, qp_d_, n_spec_, s);
    else
        dev::launch_multiply(spec, mult_, n_spec_, s, cols);
    if (cufftExecZ2D(inv, reinterpret_cast<cufftDoubleComplex*>(spec), na.grid) != CUFFT_SUCCESS)
        throw std::runtime_error("cuFFT error in the batched inverse transform");
    if (!interp) return 2;
    dev::launch_interp_multi(na, m.esw, n_, cols, s);
    return 3;
}

bool DeviceTree::multi_host_overlapped(int k, bool fp32, double* qd, double* pd,
                                       const std::function<void(int, int)>& upload) {
    constexpr int kChunkCols = 8;
    fp32 = fp32 && mixed_allowed();
    if (!overlap_h2d_ || qp_ || k < 2 * kChunkCols || k % kChunkCols != 0) return false;
    if (multi_block(k, fp32) < k) return false;  // one block of k columns only
    MultiState& m = multi_state(multi_block(k, fp32), fp32);
    if (!m.far_stream) {
        PDMK_CUDA_CHECK(cudaStreamCreateWithFlags(&m.far_stream, cudaStreamNonBlocking));
        PDMK_CUDA_CHECK(cudaEventCreateWithFlags(&m.ev_far, cudaEventDisableTiming));
        PDMK_CUDA_CHECK(cudaEventCreate(&m.ev_far0));
        int dims[3] = {nufft_.n1, nufft_.n2, nufft_.n3};
        const cufftResult r1 = cufftPlanMany(&m.fwd_c, 3, dims, nullptr, 1, (int)n_grid_, nullptr, 1, (int)n_spec_,
                                             CUFFT_D2Z, kChunkCols);
        const cufftResult r2 = cufftPlanMany(&m.inv_c, 3, dims, nullptr, 1, (int)n_spec_, nullptr, 1, (int)n_grid_,
                                             CUFFT_Z2D, kChunkCols);
        if (r1 != CUFFT_SUCCESS || r2 != CUFFT_SUCCESS) throw std::runtime_error("cuFFT error: chunk plan creation failed");
        cufftSetStream(m.fwd_c, m.far_stream);
        cufftSetStream(m.inv_c, m.far_stream);
        m.chunk_cols = kChunkCols;
    }
    const int nch = k / m.chunk_cols;
    while ((int)m.ev_chunk.size() < nch) {
        cudaEvent_t e;
        PDMK_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        m.ev_chunk.push_back(e);
    }
    multi_launches_ = 0;
    // uploads, in order, on the main stream
    for (int c = 0; c < nch; ++c) {
        upload(c * m.chunk_cols, m.chunk_cols);
        PDMK_CUDA_CHECK(cudaEventRecord(m.ev_chunk[c], stream_));
    }
    // the far field of each chunk as soon as it is in
    cudaStream_t fs = m.far_stream;
    for (int c = 0; c < nch; ++c) {
        const int c0 = c * m.chunk_cols, cols = m.chunk_cols;
        PDMK_CUDA_CHECK(cudaStreamWaitEvent(fs, m.ev_chunk[c], 0));
        if (c == 0) PDMK_CUDA_CHECK(cudaEventRecord(m.ev_far0, fs));
        const int64_t tt = (int64_t)n_ * cols;
        dev::k_gather_trg_m<<<(unsigned)((tt + 255) / 256), 256, 0, fs>>>(m.q_t + (int64_t)c0 * n_, trg_perm_,
                                                                          qd + (int64_t)c0 * n_, n_, cols, cols);
        multi_launches_ += 1 + far_columns(m, c0, cols, false, m.fwd_c, m.inv_c, fs);
    }
    PDMK_CUDA_CHECK(cudaEventRecord(m.ev_far, fs));
    // the tree passes, near field and finalize on the main stream
    struct Ext {
        DeviceTree& t;
        Ext(DeviceTree& x, cudaEvent_t e) : t(x) { t.far_ext_ = true; t.far_ext_event_ = e; }
        ~Ext() { t.far_ext_ = false; t.far_ext_event_ = nullptr; }
    } ext(*this, m.ev_far);
    if (fp32)
        run_multi_block<float>(m, qd, k, pd);
    else
        run_multi_block<double>(m, qd, k, pd);
    StageTimes t = last_times();
    float far_ms = 0.0f;
    PDMK_CUDA_CHECK(cudaEventElapsedTime(&far_ms, m.ev_far0, ev_[4]));
    t.nufft_ms = far_ms;  // far-field stream from its first chunk to the finalize (overlaps the rest)
    int err = 0;
    PDMK_CUDA_CHECK(cudaMemcpy(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        PDMK_CUDA_CHECK(cudaMemset(m.err, 0, sizeof(int)));
        throw std::runtime_error("CUDA error: tensor-core pipeline wait timed out in the multi-RHS evaluate");
    }
    last_multi_ = t;
    last_was_multi_ = true;
    return true;
}

void DeviceTree::evaluate_multi_device(const double* Q, int k, double* pot, bool fp32, StageTimes* times) {
    if (k <= 0) throw std::invalid_argument("k must be positive");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    fp32 = fp32 && mixed_allowed();
    const int kb = multi_block(k, fp32);
    MultiState& m = multi_state(kb, fp32);
    StageTimes acc;
    multi_launches_ = 0;
    for (int c0 = 0; c0 < k; c0 += m.kb) {
        const int kv = std::min(m.kb, k - c0);
        if (fp32)
            run_multi_block<float>(m, Q + (int64_t)c0 * n_, kv, pot + (int64_t)c0 * n_);
        else
            run_multi_block<double>(m, Q + (int64_t)c0 * n_, kv, pot + (int64_t)c0 * n_);
        // per-block stage times (the events are reused by the next block)
        const StageTimes t = last_times();
        int err = 0;
        PDMK_CUDA_CHECK(cudaMemcpy(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) {
            PDMK_CUDA_CHECK(cudaMemset(m.err, 0, sizeof(int)));
            throw std::runtime_error("CUDA error: tensor-core pipeline wait timed out in the multi-RHS evaluate");
        }
        acc.dmk_ms += t.dmk_ms;
        acc.direct_ms += t.direct_ms;
        acc.nufft_ms += t.nufft_ms;
        acc.near_ms += t.near_ms;
        acc.finalize_ms += t.finalize_ms;
    }
    if (times) *times = acc;
    last_multi_ = acc;
    last_was_multi_ = true;
}

void DeviceTree::evaluate_complex_device(const double* q, double* pot2, StageTimes* times) {
    if (!qp_) throw std::logic_error("evaluate_complex: bloch not set at construction");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    MultiState& m = multi_state(2, false);
    struct Flag {  // run_multi_block computes the quasi-periodic columns only inside this call
        bool& f;
        explicit Flag(bool& x) : f(x) { f = true; }
        ~Flag() { f = false; }
    } on(qp_run_);
    multi_launches_ = 0;
    run_multi_block<double>(m, q, 1, pot2);
    const StageTimes t = last_times();
    if (times) *times = t;
    last_multi_ = t;
    last_was_multi_ = true;
}

void DeviceTree::evaluate_complex_host(const double* q, double* pot2, StageTimes* times) {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    ensure_stage(2 * (int64_t)n_);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(stage_q_, q, sizeof(double) * n_, cudaMemcpyHostToDevice, stream_));
    evaluate_complex_device(stage_q_, stage_p_, times);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(pot2, stage_p_, sizeof(double) * 2 * (size_t)n_, cudaMemcpyDeviceToHost, stream_));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void DeviceTree::enqueue_multi_device(const double* Q, int k, double* pot, bool fp32) {
    if (k <= 0) throw std::invalid_argument("k must be positive");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    fp32 = fp32 && mixed_allowed();
    const int kb = multi_block(k, fp32);
    MultiState& m = multi_state(kb, fp32);
    multi_launches_ = 0;
    for (int c0 = 0; c0 < k; c0 += m.kb) {
        const int kv = std::min(m.kb, k - c0);
        if (fp32)
            run_multi_block<float>(m, Q + (int64_t)c0 * n_, kv, pot + (int64_t)c0 * n_);
        else
            run_multi_block<double>(m, Q + (int64_t)c0 * n_, kv, pot + (int64_t)c0 * n_);
    }
    last_was_multi_ = true;
}

int* DeviceTree::multi_error_word(bool fp32) const {
    const auto& slot = multi_[fp32 ? 1 : 0];
    return slot ? slot->err : nullptr;
}

void DeviceTree::check_device_error() {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    for (auto& slot : multi_) {
        if (!slot) continue;
        int err = 0;
        PDMK_CUDA_CHECK(cudaMemcpy(&err, slot->err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) {
            PDMK_CUDA_CHECK(cudaMemset(slot->err, 0, sizeof(int)));
            throw std::runtime_error("CUDA error: tensor-core pipeline wait timed out in the multi-RHS evaluate");
        }
    }
}

namespace dev {
__global__ void k_to_float_out(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}
void launch_to_float(const double* in, float* out, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_to_float_out<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n);
}
}  // namespace dev

namespace dev {
__global__ void k_to_double_in(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}
}  // namespace dev

void DeviceTree::ensure_stage(int64_t n) {
    if ((size_t)n <= stage_elems_) return;
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
    if (stage_q_) cudaFree(stage_q_);
    if (stage_p_) cudaFree(stage_p_);
    stage_q_ = stage_p_ = nullptr;
    stage_elems_ = 0;
    PDMK_CUDA_CHECK(cudaMalloc(&stage_q_, sizeof(double) * (size_t)n));
    PDMK_CUDA_CHECK(cudaMalloc(&stage_p_, sizeof(double) * (size_t)n));
    stage_elems_ = (size_t)n;
}

void DeviceTree::evaluate_multi_device_f32(const float* Q, int k, double* pot, bool fp32, StageTimes* times) {
    if (k <= 0) throw std::invalid_argument("k must be positive");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    const int64_t n = (int64_t)n_ * k;
    ensure_stage(n);
    dev::k_to_double_in<<<(unsigned)((n + 255) / 256), 256, 0, stream_>>>(Q, stage_q_, n);
    evaluate_multi_device(stage_q_, k, pot, fp32, times);
}

void DeviceTree::evaluate_multi_host_f32(const float* Q, int k, float* pot, bool fp32) {
    if (k <= 0) throw std::invalid_argument("k must be positive");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    const int64_t n = (int64_t)n_ * k;
    ensure_stage(n);
    // float charges land in the upper half of the potential staging buffer,
    // are widened into the charge staging buffer, and the float potentials
    // are narrowed into the charge buffer after the evaluate
    float* qf = reinterpret_cast<float*>(stage_p_) + n;
    auto upload = [&](int c0, int cols) {
        const int64_t o = (int64_t)c0 * n_, m = (int64_t)cols * n_;
        PDMK_CUDA_CHECK(cudaMemcpyAsync(qf + o, Q + o, sizeof(float) * (size_t)m, cudaMemcpyHostToDevice, stream_));
        dev::k_to_double_in<<<(unsigned)((m + 255) / 256), 256, 0, stream_>>>(qf + o, stage_q_ + o, m);
    };
    if (!multi_host_overlapped(k, fp32, stage_q_, stage_p_, upload)) {
        upload(0, k);
        evaluate_multi_device(stage_q_, k, stage_p_, fp32, nullptr);
    }
    float* pf = reinterpret_cast<float*>(stage_q_);
    dev::k_to_float_out<<<(unsigned)((n + 255) / 256), 256, 0, stream_>>>(stage_p_, pf, n);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(pot, pf, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, stream_));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void DeviceTree::evaluate_multi_host(const double* Q, int k, void* pot, bool pot_float, bool fp32,
                                     StageTimes* times) {
    if (k <= 0) throw std::invalid_argument("k must be positive");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    const int64_t n = (int64_t)n_ * k;
    const size_t bytes = sizeof(double) * (size_t)n;
    ensure_stage(n);
    double* qd = stage_q_;
    double* pd = stage_p_;
    auto upload = [&](int c0, int cols) {
        const int64_t o = (int64_t)c0 * n_;
        PDMK_CUDA_CHECK(cudaMemcpyAsync(qd + o, Q + o, sizeof(double) * (size_t)cols * n_, cudaMemcpyHostToDevice,
                                        stream_));
    };
    // stage times asked for: one upload, then the stages in sequence
    if (times || !multi_host_overlapped(k, fp32, qd, pd, upload)) {
        upload(0, k);
        evaluate_multi_device(qd, k, pd, fp32, times);
    }
    if (pot_float) {
        // reuse the charge buffer for the float copy of the potentials
        float* pf = reinterpret_cast<float*>(qd);
        dev::k_to_float_out<<<(unsigned)((n + 255) / 256), 256, 0, stream_>>>(pd, pf, n);
        PDMK_CUDA_CHECK(cudaMemcpyAsync(pot, pf, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, stream_));
    } else {
        PDMK_CUDA_CHECK(cudaMemcpyAsync(pot, pd, bytes, cudaMemcpyDeviceToHost, stream_));
    }
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

}  // namespace pdmkb
